"""Differentiable traveltime misfit for PyTorch: the testable counterpart of the
ChainRulesCore `rrule` a Julia caller would put on `eikttimemisfit`
(src/EikSolv/eikmaingrad.jl:1302-1328), with the adjoint of `eikgradient`
(src/EikSolv/eikmaingrad.jl:31-164) as its pullback.

    misfit = eik_misfit(vel, coordsrc, grd, coordrec, pickobs, stdobs)
    misfit.backward()        # vel.grad (and coordsrc.grad if it requires grad)

`vel` is a CUDA float64 tensor shaped like the grid (index [i, j(, k)] as the reference's
arrays), `coordsrc` a (nsrc, ndim) float64 tensor; observations are host arrays or tensors.

Modes:
* "store" (default when a gradient is wanted): one eik_gradient_device call computes the
  misfit and the gradient together; the gradient (one N-sized field, plus nsrc x ndim) is
  kept for backward. Right when every evaluation is differentiated (HMC steps).
* "recompute": forward runs only the traveltime solve; backward runs the gradient call
  (forward again + adjoint). Right when most evaluations are not differentiated (line
  searches), or when the device memory for the adjoint is wanted elsewhere in between.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _lib
from .api import Context, default_context
from .structs import ExtraParams

try:
    import torch
except ImportError:  # pragma: no cover - torch is part of the image
    torch = None


def _flat_obs(coordrec, pickobs, stdobs, device):
    recs = [np.ascontiguousarray(np.atleast_2d(np.asarray(r, dtype=np.float64))) for r in coordrec]
    off = np.zeros(len(recs) + 1, dtype=np.int64)
    for i, r in enumerate(recs):
        off[i + 1] = off[i] + r.shape[0]
    cat = lambda xs: np.ascontiguousarray(np.concatenate([np.asarray(  # noqa: E731
        x.detach().cpu() if torch is not None and isinstance(x, torch.Tensor) else x, dtype=np.float64).ravel()
        for x in xs]))
    rec = torch.from_numpy(np.ascontiguousarray(np.concatenate(recs))).to(device)
    return off, rec, torch.from_numpy(cat(pickobs)).to(device), torch.from_numpy(cat(stdobs)).to(device)


def _gradient(ectx: Context, vel, coordsrc, grd, coordrec, pickobs, stdobs, ep, want_src):
    dev = vel.device
    velf = vel.detach().permute(*reversed(range(vel.dim()))).contiguous()  # column-major order
    off, rec, po, so = _flat_obs(coordrec, pickobs, stdobs, dev)
    cs = coordsrc.detach().to(dev, torch.float64).contiguous()
    torch.cuda.current_stream(dev).synchronize()  # inputs written by torch are visible to the library
    mid = ectx.upload_device(velf.data_ptr(), grd)
    try:
        nsrc, nd = cs.shape
        N = int(np.prod(grd.grsize))
        gv = torch.empty(N, dtype=torch.float64, device=dev)
        gs = torch.zeros(nsrc * nd, dtype=torch.float64, device=dev)
        m = torch.empty(1, dtype=torch.float64, device=dev)
        epc = _lib.extra_struct(ep)
        st = _lib.eik_stats()
        P = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
        rc = ectx.L.eik_gradient_device(ectx.h, C.c_int64(mid), nsrc, P(cs), _lib.ptr(off), P(rec), P(po), P(so),
                                        3 if want_src else 1, C.byref(epc), P(gv), P(gs), P(m), C.byref(st))
        _lib.check(rc, ectx.h)
    finally:
        ectx.release(mid)
    gvel = gv.reshape(tuple(reversed(grd.grsize))).permute(*reversed(range(vel.dim())))
    return m[0], gvel, gs.reshape(nsrc, nd)


def _misfit_only(ectx: Context, vel, coordsrc, grd, coordrec, pickobs, stdobs, ep):
    velf = vel.detach().permute(*reversed(range(vel.dim()))).contiguous()
    torch.cuda.current_stream(vel.device).synchronize()
    mid = ectx.upload_device(velf.data_ptr(), grd)
    try:
        picks = ectx.traveltime(mid, grd, coordsrc.detach().cpu().numpy(), coordrec, extraparams=ep)
    finally:
        ectx.release(mid)
    m = 0.0
    for p, o, s in zip(picks, pickobs, stdobs):
        o = np.asarray(o.detach().cpu() if isinstance(o, torch.Tensor) else o, dtype=np.float64)
        s = np.asarray(s.detach().cpu() if isinstance(s, torch.Tensor) else s, dtype=np.float64)
        d = p - o
        m += float(np.sum(d * d / (s * s)))
    return torch.tensor(0.5 * m, dtype=torch.float64, device=vel.device)


if torch is not None:
    class EikMisfit(torch.autograd.Function):
        @staticmethod
        def forward(fctx, vel, coordsrc, grd, coordrec, pickobs, stdobs, extraparams, ectx, mode):
            want_vel = vel.requires_grad
            want_src = coordsrc.requires_grad
            fctx.args = (vel.detach(), coordsrc.detach(), grd, coordrec, pickobs, stdobs, extraparams, ectx,
                         want_src)
            fctx.src_device = coordsrc.device
            if (want_vel or want_src) and mode == "store":
                m, gv, gs = _gradient(ectx, vel, coordsrc, grd, coordrec, pickobs, stdobs, extraparams, want_src)
                fctx.save_for_backward(gv, gs)
                fctx.stored = True
                return m
            fctx.stored = False
            return _misfit_only(ectx, vel, coordsrc, grd, coordrec, pickobs, stdobs, extraparams)

        @staticmethod
        def backward(fctx, gout):
            if fctx.stored:
                gv, gs = fctx.saved_tensors
            else:
                vel, cs, grd, rec, po, so, ep, ectx, want_src = fctx.args
                _, gv, gs = _gradient(ectx, vel, cs, grd, rec, po, so, ep, want_src)
            gvel = gout * gv if fctx.needs_input_grad[0] else None
            gsrc = (gout * gs).to(fctx.src_device) if fctx.needs_input_grad[1] else None
            return gvel, gsrc, None, None, None, None, None, None, None


def eik_misfit(vel, coordsrc, grd, coordrec, pickobs, stdobs, extraparams: Optional[ExtraParams] = None,
               ctx: Optional[Context] = None, mode: str = "store"):
    """0.5 Σ (t - obs)²/σ² as a differentiable function of `vel` (and `coordsrc`)."""
    if torch is None:
        raise ImportError("torch is required for eik_misfit")
    if mode not in ("store", "recompute"):
        raise ValueError("mode must be 'store' or 'recompute'")
    if not vel.is_cuda or vel.dtype != torch.float64:
        raise TypeError("vel must be a CUDA float64 tensor")
    if not isinstance(coordsrc, torch.Tensor):
        coordsrc = torch.as_tensor(np.asarray(coordsrc, dtype=np.float64))
    ectx = ctx or default_context(vel.device.index or 0)
    return EikMisfit.apply(vel, coordsrc, grd, coordrec, pickobs, stdobs, extraparams, ectx, mode)
