"""Hamiltonian Monte Carlo problem callables over libeikcuda: the three problem types of
the reference's HMCtraveltimes module (src/HMCtraveltimes.jl:26-283), each a callable
``prob(x, kind)`` that an HMC sampler evaluates model after model:

* ``kind == "nlogpdf"``     -> the misfit 0.5 Σ (t - obs)²/σ² (eikttimemisfit) as a float;
* ``kind == "gradnlogpdf"`` -> its gradient w.r.t. ``x`` as a flat float64 vector.

``EikonalProbVel`` takes the velocity model flattened in column-major order (x fastest,
Julia's ``vec``), ``EikonalProbSrcLoc`` the source coordinates flattened column-major
(all x, then all y(, then all z)), ``EikonalProbVelAndSrcLoc`` the velocity followed by
the source coordinates. With ``logVel=True`` the velocity part of ``x`` is log-velocity:
it is exponentiated before the solve, and the velocity gradient is multiplied by 1/v, as
the reference does (src/HMCtraveltimes.jl:101-104 and 263-266; the exact derivative of the
misfit w.r.t. log-velocity would be v·∂ψ/∂v, the reference's factor is kept so that a
sampler sees the numbers it sees with the reference).

Every evaluation runs on the GPU through one context (``ctx``, by default the device's
default context): the model is uploaded, solved and released in the same call, so a chain
of evaluations keeps no state between calls. The reference's assertions (``whichgrad``
must match the problem type) raise ``AssertionError``; a wrong ``kind`` raises
``RuntimeError`` with the reference's message.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from .api import Context, eikgradient, eikttimemisfit
from .structs import ExtraParams


def _kind(kind) -> str:
    return str(kind).lstrip(":")


def _grid_ok(grd):
    # the reference's fields are typed Union{Grid2DCart,Grid3DCart}
    if type(grd).__name__ not in ("Grid2DCart", "Grid3DCart"):
        raise TypeError(f"grd must be a Grid2DCart or Grid3DCart, not {type(grd).__name__}")


def _velocity(x: np.ndarray, grd, logvel: bool) -> np.ndarray:
    v = np.exp(x) if logvel else x
    return np.reshape(v, tuple(grd.grsize), order="F")


def _coords(x: np.ndarray, nd: int) -> np.ndarray:
    # reshape(inpcoosrc, :, nd): column-major, one row per source
    return np.reshape(x, (-1, nd), order="F")


@dataclass
class EikonalProbVel:
    """Velocity tomography (src/HMCtraveltimes.jl:26-113)."""
    grd: object
    dobs: List[np.ndarray]
    stdobs: List[np.ndarray]
    coordsrc: np.ndarray
    coordrec: List[np.ndarray]
    whichgrad: str
    logVel: bool = False
    extraparams: Optional[ExtraParams] = None
    ctx: Optional[Context] = field(default=None, repr=False, compare=False)

    def __post_init__(self):
        _grid_ok(self.grd)

    def __call__(self, inpvecvel, kind):
        assert _kind(self.whichgrad) == "gradvel", "eikprob.whichgrad==:gradvel"
        x = np.asarray(inpvecvel, dtype=np.float64).ravel()
        velnd = _velocity(x, self.grd, self.logVel)
        k = _kind(kind)
        if k == "nlogpdf":
            return eikttimemisfit(velnd, self.grd, self.coordsrc, self.coordrec, self.dobs, self.stdobs,
                                  extraparams=self.extraparams, ctx=self.ctx)
        if k == "gradnlogpdf":
            grad, _ = eikgradient(velnd, self.grd, self.coordsrc, self.coordrec, self.dobs, self.stdobs, "gradvel",
                                  extraparams=self.extraparams, ctx=self.ctx)
            if self.logVel:
                grad = (1.0 / velnd) * grad
            return np.ravel(grad, order="F")
        raise RuntimeError(f"eikprob::EikonalProbVel(): Wrong argument 'kind': {kind}...")


@dataclass
class EikonalProbSrcLoc:
    """Source location (src/HMCtraveltimes.jl:115-182)."""
    grd: object
    dobs: List[np.ndarray]
    stdobs: List[np.ndarray]
    coordrec: List[np.ndarray]
    velmod: np.ndarray
    whichgrad: str
    extraparams: Optional[ExtraParams] = None
    ctx: Optional[Context] = field(default=None, repr=False, compare=False)

    def __post_init__(self):
        _grid_ok(self.grd)

    def __call__(self, inpcoosrc, kind):
        assert _kind(self.whichgrad) == "gradsrcloc", "eikprob.whichgrad==:gradsrcloc"
        velmod = np.asarray(self.velmod, dtype=np.float64)
        coosrcnd = _coords(np.asarray(inpcoosrc, dtype=np.float64).ravel(), velmod.ndim)
        k = _kind(kind)
        if k == "nlogpdf":
            return eikttimemisfit(velmod, self.grd, coosrcnd, self.coordrec, self.dobs, self.stdobs,
                                  extraparams=self.extraparams, ctx=self.ctx)
        if k == "gradnlogpdf":
            gradsrcloc, _ = eikgradient(velmod, self.grd, coosrcnd, self.coordrec, self.dobs, self.stdobs,
                                        "gradsrcloc", extraparams=self.extraparams, ctx=self.ctx)
            return np.ravel(gradsrcloc, order="F")
        raise RuntimeError(f"eikprob::EikonalProbSrcLoc(): Wrong argument 'kind': {kind}...")


@dataclass
class EikonalProbVelAndSrcLoc:
    """Velocity and source location together (src/HMCtraveltimes.jl:185-283): ``x`` is the
    flattened velocity (prod(grsize) values) followed by the flattened source coordinates."""
    grd: object
    dobs: List[np.ndarray]
    stdobs: List[np.ndarray]
    coordrec: List[np.ndarray]
    whichgrad: str
    logVel: bool = False
    extraparams: Optional[ExtraParams] = None
    ctx: Optional[Context] = field(default=None, repr=False, compare=False)

    def __post_init__(self):
        _grid_ok(self.grd)

    def __call__(self, inppars, kind):
        assert _kind(self.whichgrad) == "gradvelandsrcloc", "eikprob.whichgrad==:gradvelandsrcloc"
        x = np.asarray(inppars, dtype=np.float64).ravel()
        ngridpt = int(np.prod(self.grd.grsize))
        velnd = _velocity(x[:ngridpt], self.grd, self.logVel)
        coosrcnd = _coords(x[ngridpt:], velnd.ndim)
        k = _kind(kind)
        if k == "nlogpdf":
            return eikttimemisfit(velnd, self.grd, coosrcnd, self.coordrec, self.dobs, self.stdobs,
                                  extraparams=self.extraparams, ctx=self.ctx)
        if k == "gradnlogpdf":
            gradvel, gradsrcloc, _ = eikgradient(velnd, self.grd, coosrcnd, self.coordrec, self.dobs, self.stdobs,
                                                 "gradvelandsrcloc", extraparams=self.extraparams, ctx=self.ctx)
            if self.logVel:
                gradvel = (1.0 / velnd) * gradvel
            return np.concatenate([np.ravel(gradvel, order="F"), np.ravel(gradsrcloc, order="F")])
        raise RuntimeError(f"eikprob::EikonalVelAndSrcLocProb(): Wrong argument 'kind': {kind}...")
