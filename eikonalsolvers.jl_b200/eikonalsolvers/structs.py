"""Grid and parameter types of EikonalSolvers.jl, restated for the Python host.

Mirrors ``src/EikSolv/eikstructs.jl``:

* ``Grid2DCart``   (eikstructs.jl:33-55)
* ``Grid3DCart``   (eikstructs.jl:78-103)
* ``Grid2DSphere`` (eikstructs.jl:126-158), θ in degrees, 0 ≤ θ ≤ 180
* ``Grid3DSphere`` (eikstructs.jl:182-219), 5 ≤ θ ≤ 175, 0 ≤ φ ≤ 180
* ``GridRefinementPars`` (eikstructs.jl:230-235)
* ``ExtraParams`` (eikstructs.jl:246-282)

Node coordinates follow Julia's ``range(start=a, step=h, length=n)`` for Float64:
when start and step are small rationals (``Base.rat``), node ``i`` is the correctly
rounded value of ``(start_n + (i-1)*step_n) / den``; otherwise ``a + (i-1)*h`` is
evaluated in double-double and rounded once.  The GPU library receives the same
rational decomposition so both sides compute bit-identical node coordinates.
"""
from __future__ import annotations

import math
from fractions import Fraction
from typing import Tuple

import numpy as np

KIND_2DCART, KIND_3DCART, KIND_2DSPHERE, KIND_3DSPHERE = 0, 1, 2, 3

_F32_MAXINT = 16777216
_F64_MAXINT = 9007199254740992


def _julia_rat(x: float) -> Tuple[int, int]:
    """``Base.rat`` (twiceprecision.jl): bounded continued-fraction approximation."""
    y = x
    a, d, b, c = 1, 1, 0, 0
    m = float(_F32_MAXINT)
    while abs(y) <= m:
        f = int(math.trunc(y))
        y -= f
        a, c = f * a + c, a
        b, d = f * b + d, b
        if not max(abs(a), abs(b)) <= _F32_MAXINT:
            return c, d
        if b != 0 and float(a) / float(b) == x:
            break
        if y == 0.0:
            y = math.inf
        else:
            y = 1.0 / y
    return a, b


class JuliaRange:
    """Float64 ``range(start=a, step=st, length=n)`` with Julia's element values."""

    def __init__(self, start: float, step: float, length: int):
        self.start, self.step, self.length = float(start), float(step), int(length)
        self.rational = False
        self.start_n, self.step_n, self.den = 0, 0, 1
        sn, sd = _julia_rat(self.start)
        tn, td = _julia_rat(self.step)
        if sd != 0 and td != 0 and sn / sd == self.start and tn / td == self.step:
            den = sd // math.gcd(sd, td) * td
            if (abs(den * self.start) <= _F64_MAXINT and abs(den * self.step) <= _F64_MAXINT
                    and den % sd == 0 and den % td == 0):
                self.rational = True
                self.den = den
                self.start_n = sn * (den // sd)
                self.step_n = tn * (den // td)

    def __len__(self) -> int:
        return self.length

    def value(self, i1: int) -> float:
        """1-based element, as ``r[i1]`` in Julia."""
        if self.rational:
            num = self.start_n + (i1 - 1) * self.step_n
            if abs(num) <= 2 ** 53:
                return float(num) / float(self.den)
            return float(Fraction(num, self.den))
        exact = Fraction(self.start) + (i1 - 1) * Fraction(self.step)
        return float(exact)

    def __getitem__(self, idx):
        """0-based Python indexing (``r[0]`` is Julia's ``r[1]``); supports -1."""
        if isinstance(idx, slice):
            return np.array([self[i] for i in range(*idx.indices(self.length))])
        i = int(idx)
        if i < 0:
            i += self.length
        if not 0 <= i < self.length:
            raise IndexError(idx)
        return self.value(i + 1)

    def __array__(self, dtype=None, copy=None):
        arr = np.array([self.value(i) for i in range(1, self.length + 1)], dtype=np.float64)
        return arr if dtype is None else arr.astype(dtype)

    def __iter__(self):
        for i in range(1, self.length + 1):
            yield self.value(i)


class _GridBase:
    kind: int
    ndim: int
    grsize: Tuple[int, ...]
    cooinit: Tuple[float, ...]

    @property
    def spacing(self) -> Tuple[float, ...]:
        raise NotImplementedError

    @property
    def npts(self) -> int:
        return int(np.prod(self.grsize))

    def axis_range(self, d: int) -> JuliaRange:
        return self._axes[d]

    def __repr__(self):
        return f"{type(self).__name__}(spacing={self.spacing}, cooinit={self.cooinit}, grsize={self.grsize})"


class Grid2DCart(_GridBase):
    """2D Cartesian grid (eikstructs.jl:33-55)."""

    kind, ndim = KIND_2DCART, 2

    def __init__(self, *, hgrid: float, cooinit, grsize):
        assert float(hgrid) > 0.0, "hgrid>0.0"
        assert all(int(n) > 0 for n in grsize), "all(grsize.>0)"
        assert len(cooinit) == 2 and len(grsize) == 2
        self.hgrid = float(hgrid)
        self.cooinit = tuple(float(c) for c in cooinit)
        self.grsize = tuple(int(n) for n in grsize)
        self._axes = [JuliaRange(self.cooinit[d], self.hgrid, self.grsize[d]) for d in range(2)]
        self.x, self.y = self._axes
        self.cooend = (self.x[-1], self.y[-1])

    @property
    def spacing(self):
        return (self.hgrid, self.hgrid)


class Grid3DCart(_GridBase):
    """3D Cartesian grid (eikstructs.jl:78-103)."""

    kind, ndim = KIND_3DCART, 3

    def __init__(self, *, hgrid: float, cooinit, grsize):
        assert float(hgrid) > 0.0, "hgrid>0.0"
        assert all(int(n) > 0 for n in grsize), "all(grsize.>0)"
        assert len(cooinit) == 3 and len(grsize) == 3
        self.hgrid = float(hgrid)
        self.cooinit = tuple(float(c) for c in cooinit)
        self.grsize = tuple(int(n) for n in grsize)
        self._axes = [JuliaRange(self.cooinit[d], self.hgrid, self.grsize[d]) for d in range(3)]
        self.x, self.y, self.z = self._axes
        self.cooend = (self.x[-1], self.y[-1], self.z[-1])

    @property
    def spacing(self):
        return (self.hgrid, self.hgrid, self.hgrid)


class Grid2DSphere(_GridBase):
    """2D spherical (polar) grid in (r, θ°) (eikstructs.jl:126-158)."""

    kind, ndim = KIND_2DSPHERE, 2

    def __init__(self, *, Δr: float, Δθ: float, cooinit, grsize):
        assert float(cooinit[0]) >= 0.0, "cooinit[1]>=0.0"
        assert float(Δr) > 0.0, "Δr>0.0"
        assert float(Δθ) > 0.0, "Δθ>0.0"
        assert all(int(n) > 0 for n in grsize), "all(grsize.>0)"
        self.Δr, self.Δθ = float(Δr), float(Δθ)
        self.cooinit = tuple(float(c) for c in cooinit)
        self.grsize = tuple(int(n) for n in grsize)
        self._axes = [JuliaRange(self.cooinit[0], self.Δr, self.grsize[0]),
                      JuliaRange(self.cooinit[1], self.Δθ, self.grsize[1])]
        self.r, self.θ = self._axes
        assert all(0.0 <= t <= 180.0 for t in self.θ), "all(0.0.<=θ.<=180.0)"
        self.cooend = (self.r[-1], self.θ[-1])

    @property
    def spacing(self):
        return (self.Δr, self.Δθ)


class Grid3DSphere(_GridBase):
    """3D spherical grid in (r, θ°, φ°) (eikstructs.jl:182-219)."""

    kind, ndim = KIND_3DSPHERE, 3

    def __init__(self, *, Δr: float, Δθ: float, Δφ: float, cooinit, grsize):
        assert float(cooinit[0]) > 0.0, "cooinit[1]>0.0"
        assert all(int(n) > 0 for n in grsize), "all(grsize.>0)"
        self.Δr, self.Δθ, self.Δφ = float(Δr), float(Δθ), float(Δφ)
        self.cooinit = tuple(float(c) for c in cooinit)
        self.grsize = tuple(int(n) for n in grsize)
        self._axes = [JuliaRange(self.cooinit[0], self.Δr, self.grsize[0]),
                      JuliaRange(self.cooinit[1], self.Δθ, self.grsize[1]),
                      JuliaRange(self.cooinit[2], self.Δφ, self.grsize[2])]
        self.r, self.θ, self.φ = self._axes
        assert all(5.0 <= t <= 175.0 for t in self.θ), "all(5.0.<=θ.<=175.0)"
        assert all(0.0 <= p <= 180.0 for p in self.φ), "all(0.0.<=φ.<=180.0)"
        self.cooend = (self.r[-1], self.θ[-1], self.φ[-1])

    @property
    def spacing(self):
        return (self.Δr, self.Δθ, self.Δφ)


class GridRefinementPars:
    """Refinement around the source (eikstructs.jl:230-235)."""

    def __init__(self, *, downscalefactor: int, noderadius: int):
        self.downscalefactor = int(downscalefactor)
        self.noderadius = int(noderadius)

    def __repr__(self):
        return f"GridRefinementPars(downscalefactor={self.downscalefactor}, noderadius={self.noderadius})"


_PARALLELKINDS = ("serial", "sharedmem", "distribmem")


class ExtraParams:
    """Extra parameters (eikstructs.jl:246-282), same defaults and checks.

    ``parallelkind`` is accepted for compatibility; the GPU path batches all sources
    of a call in one launch regardless of its value.
    """

    def __init__(self, *, refinearoundsrc: bool = True, manualGCtrigger: bool = False,
                 parallelkind: str = "serial", radiussmoothgradsrc: int = 3,
                 smoothgradkern: int = 0, grdrefpars: GridRefinementPars | None = None):
        parallelkind = str(parallelkind).lstrip(":")
        assert int(radiussmoothgradsrc) >= 0, "radiussmoothgradsrc>= 0"
        assert int(smoothgradkern) >= 0, "smoothgradkern>=0"
        if int(smoothgradkern) > 0 and int(smoothgradkern) % 2 == 0:
            raise ValueError("ExtraParams: smoothgradkern must be an odd number")
        if parallelkind not in _PARALLELKINDS:
            raise ValueError("ExtraParams(): 'parallelkind' must be one of :serial, :sharedmem or :distribmem")
        self.refinearoundsrc = bool(refinearoundsrc)
        self.manualGCtrigger = bool(manualGCtrigger)
        self.parallelkind = parallelkind
        self.radiussmoothgradsrc = int(radiussmoothgradsrc)
        self.smoothgradkern = int(smoothgradkern)
        self.grdrefpars = grdrefpars if grdrefpars is not None else GridRefinementPars(
            downscalefactor=5, noderadius=3)

    def __repr__(self):
        return (f"ExtraParams(refinearoundsrc={self.refinearoundsrc}, parallelkind=:{self.parallelkind}, "
                f"radiussmoothgradsrc={self.radiussmoothgradsrc}, smoothgradkern={self.smoothgradkern}, "
                f"grdrefpars={self.grdrefpars})")


WHICHGRAD = {"gradvel": 1, "gradsrcloc": 2, "gradvelandsrcloc": 3}


def normalize_inputs(vel, grd, coordsrc, coordrec):
    """Validate and flatten the reference's argument shapes.

    Returns (vel_colmajor, coordsrc (nsrc x nd C-order), recoff (nsrc+1), rec flat (nrec_tot x nd)).
    """
    vel = np.asarray(vel, dtype=np.float64)
    assert 2 <= vel.ndim <= 3, "2<=ndims(vel)<=3"
    assert vel.ndim == grd.ndim and tuple(vel.shape) == tuple(grd.grsize), "size(vel)==grd.grsize"
    coordsrc = np.ascontiguousarray(np.atleast_2d(np.asarray(coordsrc, dtype=np.float64)))
    assert coordsrc.shape[1] == grd.ndim
    if isinstance(coordrec, np.ndarray) and coordrec.dtype != object:
        coordrec = [coordrec]
    recs = [np.ascontiguousarray(np.atleast_2d(np.asarray(r, dtype=np.float64))) for r in coordrec]
    assert coordsrc.shape[0] == len(recs), "size(coordsrc,1)==length(coordrec)"
    for r in recs:
        assert r.shape[1] == grd.ndim
    recoff = np.zeros(len(recs) + 1, dtype=np.int64)
    for s, r in enumerate(recs):
        recoff[s + 1] = recoff[s] + r.shape[0]
    rec = np.concatenate(recs, axis=0) if recs else np.zeros((0, grd.ndim))
    velf = np.asfortranarray(vel).ravel(order="F")
    return velf, coordsrc, recoff, np.ascontiguousarray(rec)
