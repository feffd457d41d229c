"""Public API of EikonalSolvers.jl over libeikcuda, with the reference's signatures:

* ``eiktraveltime(vel, grd, coordsrc, coordrec; returntt, extraparams)``
  (src/EikSolv/eikmainfwd.jl:33-143)
* ``eikgradient(vel, grd, coordsrc, coordrec, pickobs, stdobs, whichgrad; extraparams)``
  (src/EikSolv/eikmaingrad.jl:31-164)
* ``eikttimemisfit(velmod, grd, coordsrc, coordrec, ttpicksobs, stdobs; extraparams)``
  (src/EikSolv/eikmaingrad.jl:1302-1328)

Arrays follow the reference: ``vel[i, j(, k)]`` indexed by grid node (x fastest in
memory order is handled here), ``coordsrc`` is (nsrc, ndim), ``coordrec`` a list of
(nrec_s, ndim) arrays, picks are returned as a list of 1-D arrays. Assertion failures of
the reference raise ``AssertionError``; its ``error()`` calls raise ``RuntimeError``.
"""
from __future__ import annotations

import ctypes as C
import threading
import warnings
from typing import Optional

import numpy as np

from . import _lib
from .structs import WHICHGRAD, ExtraParams, normalize_inputs


class EikonalWarning(UserWarning):
    """A condition the reference reports with @warn (the call still returns its result)."""


def _warn(st) -> None:
    for msg in _lib.warn_mask_messages(int(st.warn_mask)):
        warnings.warn(msg, EikonalWarning, stacklevel=3)


class Context:
    """A libeikcuda context on one CUDA device (stream, resident models, HBM budget)."""

    def __init__(self, device: int = 0, hbm_budget: int = 0):
        self.L = _lib.load()
        self.h = C.c_void_p()
        _lib.check(self.L.eik_ctx_create(int(device), C.c_size_t(int(hbm_budget)), C.byref(self.h)))
        self.device = device
        self.last_stats = _lib.eik_stats()

    def set_param(self, name: str, value: float):
        """Scheduling parameter of this context (see eik_ctx_set_param)."""
        _lib.check(self.L.eik_ctx_set_param(self.h, name.encode(), float(value)), self.h)

    def gradient_bytes(self, model: int, nsrc: int, nrec: int, whichgrad="gradvel", extraparams=None,
                       nthreads: int = 1) -> int:
        """Device bytes one gradient pipeline of nsrc sources and nrec receivers in all takes
        from this context's budget (eik_gradient_bytes); larger calls are split into chunks."""
        wg = whichgrad.lstrip(":") if isinstance(whichgrad, str) else whichgrad
        ep = _lib.extra_struct(extraparams, nthreads)
        out = C.c_uint64()
        _lib.check(self.L.eik_gradient_bytes(self.h, C.c_int64(model), int(nsrc), int(nrec), C.byref(ep),
                                             WHICHGRAD[wg], C.byref(out)), self.h)
        return int(out.value)

    def selftest_wait(self, timeout_s: float = 0.2) -> int:
        """Runs one bounded device wait on a flag that nothing sets (eik_selftest_wait) and
        returns its status: EIK_ERR_TIMEOUT (-6) when the wait limit works."""
        return int(self.L.eik_selftest_wait(self.h, float(timeout_s)))
    def close(self):
        if self.h:
            self.L.eik_ctx_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---------------------------------------------------------------- models --
    def upload(self, vel: np.ndarray, grd) -> int:
        """Upload a velocity model (kept resident until ``release``); returns its id."""
        vel = np.asarray(vel, dtype=np.float64)
        assert tuple(vel.shape) == tuple(grd.grsize), "size(vel)==grd.grsize"
        velf = np.ascontiguousarray(np.asfortranarray(vel).ravel(order="F"))
        g = _lib.grid_struct(grd)
        mid = C.c_int64()
        _lib.check(self.L.eik_model_upload(self.h, C.byref(g), _lib.ptr(velf), C.byref(mid)), self.h)
        return mid.value

    def upload_device(self, vel_dev_ptr: int, grd) -> int:
        """Upload a model from a device pointer (column-major FP64) of this context's GPU."""
        g = _lib.grid_struct(grd)
        mid = C.c_int64()
        _lib.check(self.L.eik_model_upload_device(self.h, C.byref(g), C.c_void_p(vel_dev_ptr), C.byref(mid)),
                   self.h)
        return mid.value

    def release(self, model: int):
        _lib.check(self.L.eik_model_release(self.h, C.c_int64(model)), self.h)

    def traveltime_rays(self, model: int, grd, coordsrc, coordrec, steplen: float = 0.01, extraparams=None):
        """Picks and rays in one device pipeline (the traveltime grids never leave the GPU):
        returns (picks, rays) as ``traveltime`` and ``tracerays`` return them."""
        cs, recoff, rec = _ray_inputs(grd, coordsrc, coordrec)
        picks = np.zeros(max(int(recoff[-1]), 1), dtype=np.float64)
        ep = _lib.extra_struct(extraparams)
        st = _lib.eik_stats()

        def call(npts, pts, cap):
            return self.L.eik_traveltime_rays(self.h, C.c_int64(model), cs.shape[0], _lib.ptr(cs), _lib.ptr(recoff),
                                              _lib.ptr(rec), C.byref(ep), float(steplen), _lib.ptr(picks),
                                              _lib.ptr(npts), _lib.ptr(pts), cap, C.byref(st))
        rc, rays = _traced(call, grd, cs, recoff, rec, steplen)
        self.last_stats = st
        _lib.check(rc, self.h)
        return [picks[recoff[s]:recoff[s + 1]].copy() for s in range(cs.shape[0])], rays

    def plan_gradient(self, model: int, grd, coordsrc, coordrec, whichgrad, extraparams=None,
                      nthreads: int = 1) -> "GradientPlan":
        """Captures the gradient pipeline of this workload as a CUDA graph (GradientPlan)."""
        return GradientPlan(self, model, grd, coordsrc, coordrec, whichgrad, extraparams, nthreads)

    def autotune(self, model: int, grd, coordsrc, coordrec, extraparams=None, tuner=None, force: bool = False):
        """Times the forward solve's launch parameters on this workload, keeps the fastest on
        this context and returns the tuner's entry (eikonalsolvers.tune)."""
        from .tune import default_tuner
        return (tuner or default_tuner()).tune(self, model, grd, coordsrc, coordrec, extraparams, force)

    # ------------------------------------------------------------------ calls --
    def traveltime(self, model: int, grd, coordsrc, coordrec, returntt=False, extraparams=None):
        cs = np.ascontiguousarray(np.atleast_2d(np.asarray(coordsrc, dtype=np.float64)))
        if isinstance(coordrec, np.ndarray) and coordrec.dtype != object:
            coordrec = [coordrec]
        recs = [np.ascontiguousarray(np.atleast_2d(np.asarray(r, dtype=np.float64))) for r in coordrec]
        assert cs.shape[0] == len(recs), "size(coordsrc,1)==length(coordrec)"
        recoff = np.zeros(len(recs) + 1, dtype=np.int64)
        for s, r in enumerate(recs):
            recoff[s + 1] = recoff[s] + r.shape[0]
        rec = np.ascontiguousarray(np.concatenate(recs, axis=0)) if recs else np.zeros((0, grd.ndim))
        nsrc = cs.shape[0]
        picks = np.zeros(int(recoff[-1]), dtype=np.float64)
        N = int(np.prod(grd.grsize))
        ttg = np.zeros(nsrc * N, dtype=np.float64) if returntt else None
        ep = _lib.extra_struct(extraparams)
        st = _lib.eik_stats()
        rc = self.L.eik_traveltime(self.h, C.c_int64(model), nsrc, _lib.ptr(cs), _lib.ptr(recoff), _lib.ptr(rec),
                                   C.byref(ep), _lib.ptr(picks), _lib.ptr(ttg), C.byref(st))
        self.last_stats = st
        _lib.check(rc, self.h)
        _warn(st)
        out = [picks[recoff[s]:recoff[s + 1]].copy() for s in range(nsrc)]
        if returntt:
            return out, [ttg[s * N:(s + 1) * N].reshape(grd.grsize, order="F").copy() for s in range(nsrc)]
        return out

    def traveltime_multi(self, requests, returntt=False, extraparams=None):
        """Traveltimes for several models of one dimension in one device pipeline
        (eik_traveltime_multi): ``requests`` is a list of (model, grd, coordsrc, coordrec);
        returns one result per request, each as ``traveltime`` returns it for that request
        alone (bit-identical values)."""
        assert len(requests) > 0, "at least one request"
        ids, offs, css, recs_all, grds = [], [0], [], [], []
        for model, grd, coordsrc, coordrec in requests:
            cs = np.ascontiguousarray(np.atleast_2d(np.asarray(coordsrc, dtype=np.float64)))
            if isinstance(coordrec, np.ndarray) and coordrec.dtype != object:
                coordrec = [coordrec]
            recs = [np.ascontiguousarray(np.atleast_2d(np.asarray(r, dtype=np.float64))) for r in coordrec]
            assert cs.shape[0] == len(recs), "size(coordsrc,1)==length(coordrec)"
            ids.append(int(model))
            offs.append(offs[-1] + cs.shape[0])
            css.append(cs)
            recs_all.extend(recs)
            grds.append(grd)
        nd = grds[0].ndim
        assert all(g.ndim == nd for g in grds), "models of one call have one dimension"
        ids = np.asarray(ids, dtype=np.int64)
        offs = np.asarray(offs, dtype=np.int64)
        cs = np.ascontiguousarray(np.concatenate(css, axis=0))
        recoff = np.zeros(len(recs_all) + 1, dtype=np.int64)
        for s, r in enumerate(recs_all):
            recoff[s + 1] = recoff[s] + r.shape[0]
        rec = np.ascontiguousarray(np.concatenate(recs_all, axis=0)) if recs_all else np.zeros((0, nd))
        picks = np.zeros(max(int(recoff[-1]), 1), dtype=np.float64)
        Ns = [int(np.prod(g.grsize)) for g in grds]
        ttg = None
        if returntt:
            ttg = np.zeros(max(sum(N * (offs[i + 1] - offs[i]) for i, N in enumerate(Ns)), 1), dtype=np.float64)
        ep = _lib.extra_struct(extraparams)
        st = _lib.eik_stats()
        rc = self.L.eik_traveltime_multi(self.h, C.c_int64(len(ids)), _lib.ptr(ids), _lib.ptr(offs), _lib.ptr(cs),
                                         _lib.ptr(recoff), _lib.ptr(rec), C.byref(ep), _lib.ptr(picks),
                                         _lib.ptr(ttg), C.byref(st))
        self.last_stats = st
        _lib.check(rc, self.h)
        _warn(st)
        out, base = [], 0
        for i, g in enumerate(grds):
            srcs = range(int(offs[i]), int(offs[i + 1]))
            pk = [picks[recoff[s]:recoff[s + 1]].copy() for s in srcs]
            if returntt:
                N = Ns[i]
                tts = [ttg[base + k * N:base + (k + 1) * N].reshape(g.grsize, order="F").copy()
                       for k in range(len(srcs))]
                base += N * len(srcs)
                out.append((pk, tts))
            else:
                out.append(pk)
        return out

    def gradient(self, model: int, grd, coordsrc, coordrec, pickobs, stdobs, whichgrad, extraparams=None,
                 nthreads: int = 1):
        """Misfit gradient for all sources in one batched device call.

        ``nthreads`` stands for the caller's ``Threads.nthreads()``: under ``:sharedmem`` the
        reference gives each of min(nsrc, nthreads) consecutive source groups its own gradient
        buffer, which changes the values carried onto source points (eikmaingrad.jl:174-258).
        """
        wg = whichgrad.lstrip(":") if isinstance(whichgrad, str) else whichgrad
        assert wg in WHICHGRAD, "Symbol 'whichgrad' not in (:gradvel, :gradsrcloc, :gradvelandsrcloc)"
        cs = np.ascontiguousarray(np.atleast_2d(np.asarray(coordsrc, dtype=np.float64)))
        if isinstance(coordrec, np.ndarray) and coordrec.dtype != object:
            coordrec = [coordrec]
        recs = [np.ascontiguousarray(np.atleast_2d(np.asarray(r, dtype=np.float64))) for r in coordrec]
        nsrc = cs.shape[0]
        assert len(recs) == len(pickobs), "length(coordrec)==length(pickobs)"
        for r, p, s in zip(recs, pickobs, stdobs):
            assert r.shape[0] == np.asarray(p).shape[0], "size(coordrec[r],1)==size(pickobs[r],1)"
            assert np.asarray(s).shape == np.asarray(p).shape, "size(stdobs[r])==size(pickobs[r])"
        recoff = np.zeros(len(recs) + 1, dtype=np.int64)
        for s, r in enumerate(recs):
            recoff[s + 1] = recoff[s] + r.shape[0]
        rec = np.ascontiguousarray(np.concatenate(recs, axis=0)) if recs else np.zeros((0, grd.ndim))
        po = np.ascontiguousarray(np.concatenate([np.asarray(p, dtype=np.float64).ravel() for p in pickobs]))
        so = np.ascontiguousarray(np.concatenate([np.asarray(p, dtype=np.float64).ravel() for p in stdobs]))
        N = int(np.prod(grd.grsize))
        gv = np.zeros(N, dtype=np.float64) if wg in ("gradvel", "gradvelandsrcloc") else None
        gs = np.zeros(nsrc * grd.ndim, dtype=np.float64) if wg in ("gradsrcloc", "gradvelandsrcloc") else None
        misf = np.zeros(1, dtype=np.float64)
        ep = _lib.extra_struct(extraparams, nthreads)
        st = _lib.eik_stats()
        rc = self.L.eik_gradient(self.h, C.c_int64(model), nsrc, _lib.ptr(cs), _lib.ptr(recoff), _lib.ptr(rec),
                                 _lib.ptr(po), _lib.ptr(so), WHICHGRAD[wg], C.byref(ep), _lib.ptr(gv),
                                 _lib.ptr(gs), _lib.ptr(misf), C.byref(st))
        self.last_stats = st
        _lib.check(rc, self.h)
        _warn(st)
        gradvel = gv.reshape(grd.grsize, order="F") if gv is not None else None
        gradsrc = gs.reshape(nsrc, grd.ndim) if gs is not None else None
        if wg == "gradvel":
            return gradvel, float(misf[0])
        if wg == "gradsrcloc":
            return gradsrc, float(misf[0])
        return gradvel, gradsrc, float(misf[0])

    def gradient_groups(self, model: int, grd, groups, whichgrad, extraparams=None):
        """Several independent gradient evaluations on one model in one device pipeline
        (eik_gradient_groups): ``groups`` is a list of (coordsrc, coordrec, pickobs, stdobs);
        returns one result per group, each as ``gradient`` returns it for that group alone
        with one source group (bit-identical values)."""
        wg = whichgrad.lstrip(":") if isinstance(whichgrad, str) else whichgrad
        assert wg in WHICHGRAD, "Symbol 'whichgrad' not in (:gradvel, :gradsrcloc, :gradvelandsrcloc)"
        assert len(groups) > 0, "at least one group"
        goff, css, recs, pos, sos = [0], [], [], [], []
        for coordsrc, coordrec, pickobs, stdobs in groups:
            cs = np.ascontiguousarray(np.atleast_2d(np.asarray(coordsrc, dtype=np.float64)))
            if isinstance(coordrec, np.ndarray) and coordrec.dtype != object:
                coordrec = [coordrec]
            rr = [np.ascontiguousarray(np.atleast_2d(np.asarray(r, dtype=np.float64))) for r in coordrec]
            assert cs.shape[0] == len(rr) == len(pickobs) == len(stdobs), "one receiver set per source"
            for r, p, q in zip(rr, pickobs, stdobs):
                assert r.shape[0] == np.asarray(p).shape[0], "size(coordrec[r],1)==size(pickobs[r],1)"
                assert np.asarray(q).shape == np.asarray(p).shape, "size(stdobs[r])==size(pickobs[r])"
            goff.append(goff[-1] + cs.shape[0])
            css.append(cs)
            recs.extend(rr)
            pos.extend(np.asarray(p, dtype=np.float64).ravel() for p in pickobs)
            sos.extend(np.asarray(q, dtype=np.float64).ravel() for q in stdobs)
        ng = len(groups)
        goff = np.asarray(goff, dtype=np.int64)
        cs = np.ascontiguousarray(np.concatenate(css, axis=0))
        nsrc = cs.shape[0]
        recoff = np.zeros(nsrc + 1, dtype=np.int64)
        for s, r in enumerate(recs):
            recoff[s + 1] = recoff[s] + r.shape[0]
        rec = np.ascontiguousarray(np.concatenate(recs, axis=0))
        po = np.ascontiguousarray(np.concatenate(pos))
        so = np.ascontiguousarray(np.concatenate(sos))
        N = int(np.prod(grd.grsize))
        gv = np.zeros(ng * N, dtype=np.float64) if wg in ("gradvel", "gradvelandsrcloc") else None
        gs = np.zeros(nsrc * grd.ndim, dtype=np.float64) if wg in ("gradsrcloc", "gradvelandsrcloc") else None
        misf = np.zeros(ng, dtype=np.float64)
        ep = _lib.extra_struct(extraparams)
        st = _lib.eik_stats()
        rc = self.L.eik_gradient_groups(self.h, C.c_int64(model), C.c_int64(ng), _lib.ptr(goff), _lib.ptr(cs),
                                        _lib.ptr(recoff), _lib.ptr(rec), _lib.ptr(po), _lib.ptr(so), WHICHGRAD[wg],
                                        C.byref(ep), _lib.ptr(gv), _lib.ptr(gs), _lib.ptr(misf), C.byref(st))
        self.last_stats = st
        _lib.check(rc, self.h)
        _warn(st)
        out = []
        for g in range(ng):
            gvel = gv[g * N:(g + 1) * N].reshape(grd.grsize, order="F").copy() if gv is not None else None
            gsrc = gs.reshape(nsrc, grd.ndim)[goff[g]:goff[g + 1]].copy() if gs is not None else None
            m = float(misf[g])
            out.append((gvel, m) if wg == "gradvel" else (gsrc, m) if wg == "gradsrcloc" else (gvel, gsrc, m))
        return out


class GradientPlan:
    """A captured eik_gradient pipeline for fixed model, sources, receivers and parameters,
    replayed with new velocities and observations (eik_plan_gradient / eik_plan_run).

    ``run(pickobs, stdobs, vel=None)`` returns what ``Context.gradient`` returns; a ``vel``
    replaces the model's velocity in place (it stays replaced). Results are bit-identical to
    ``Context.gradient`` on the same inputs. Close the plan before releasing its model or
    closing its context."""

    def __init__(self, ctx: "Context", model: int, grd, coordsrc, coordrec, whichgrad, extraparams=None,
                 nthreads: int = 1):
        wg = whichgrad.lstrip(":") if isinstance(whichgrad, str) else whichgrad
        assert wg in WHICHGRAD, "Symbol 'whichgrad' not in (:gradvel, :gradsrcloc, :gradvelandsrcloc)"
        self.ctx, self.grd, self.wg = ctx, grd, wg
        cs = np.ascontiguousarray(np.atleast_2d(np.asarray(coordsrc, dtype=np.float64)))
        if isinstance(coordrec, np.ndarray) and coordrec.dtype != object:
            coordrec = [coordrec]
        recs = [np.ascontiguousarray(np.atleast_2d(np.asarray(r, dtype=np.float64))) for r in coordrec]
        assert cs.shape[0] == len(recs), "size(coordsrc,1)==length(coordrec)"
        self.nsrc = cs.shape[0]
        self.nrec = [r.shape[0] for r in recs]
        recoff = np.zeros(len(recs) + 1, dtype=np.int64)
        for s, r in enumerate(recs):
            recoff[s + 1] = recoff[s] + r.shape[0]
        rec = np.ascontiguousarray(np.concatenate(recs, axis=0))
        ep = _lib.extra_struct(extraparams, nthreads)
        self.h = C.c_void_p()
        _lib.check(ctx.L.eik_plan_gradient(ctx.h, C.c_int64(model), self.nsrc, _lib.ptr(cs), _lib.ptr(recoff),
                                           _lib.ptr(rec), WHICHGRAD[wg], C.byref(ep), C.byref(self.h)), ctx.h)
        self.last_stats = _lib.eik_stats()

    def run(self, pickobs, stdobs, vel=None):
        assert len(pickobs) == self.nsrc and len(stdobs) == self.nsrc, "length(coordrec)==length(pickobs)"
        for n, p, s in zip(self.nrec, pickobs, stdobs):
            assert np.asarray(p).shape[0] == n, "size(coordrec[r],1)==size(pickobs[r],1)"
            assert np.asarray(s).shape == np.asarray(p).shape, "size(stdobs[r])==size(pickobs[r])"
        po = np.ascontiguousarray(np.concatenate([np.asarray(p, dtype=np.float64).ravel() for p in pickobs]))
        so = np.ascontiguousarray(np.concatenate([np.asarray(p, dtype=np.float64).ravel() for p in stdobs]))
        velf = None
        if vel is not None:
            vel = np.asarray(vel, dtype=np.float64)
            assert tuple(vel.shape) == tuple(self.grd.grsize), "size(vel)==grd.grsize"
            velf = np.ascontiguousarray(np.asfortranarray(vel).ravel(order="F"))
        N = int(np.prod(self.grd.grsize))
        nd = self.grd.ndim
        gv = np.zeros(N, dtype=np.float64) if self.wg != "gradsrcloc" else None
        gs = np.zeros(self.nsrc * nd, dtype=np.float64) if self.wg != "gradvel" else None
        misf = np.zeros(1, dtype=np.float64)
        st = _lib.eik_stats()
        rc = self.ctx.L.eik_plan_run(self.h, _lib.ptr(velf), _lib.ptr(po), _lib.ptr(so), _lib.ptr(gv), _lib.ptr(gs),
                                     _lib.ptr(misf), C.byref(st))
        self.last_stats = st
        _lib.check(rc, self.ctx.h)
        gradvel = gv.reshape(self.grd.grsize, order="F") if gv is not None else None
        gradsrc = gs.reshape(self.nsrc, nd) if gs is not None else None
        if self.wg == "gradvel":
            return gradvel, float(misf[0])
        if self.wg == "gradsrcloc":
            return gradsrc, float(misf[0])
        return gradvel, gradsrc, float(misf[0])

    def close(self):
        if self.h:
            self.ctx.L.eik_plan_destroy(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def _ray_inputs(grd, coordsrc, coordrec):
    cs = np.ascontiguousarray(np.atleast_2d(np.asarray(coordsrc, dtype=np.float64)))
    if isinstance(coordrec, np.ndarray) and coordrec.dtype != object:
        coordrec = [coordrec]
    recs = [np.ascontiguousarray(np.atleast_2d(np.asarray(r, dtype=np.float64))) for r in coordrec]
    assert cs.shape[0] == len(recs), "size(coordsrc,1)==length(coordrec)"
    recoff = np.zeros(len(recs) + 1, dtype=np.int64)
    for s, r in enumerate(recs):
        recoff[s + 1] = recoff[s] + r.shape[0]
    rec = np.ascontiguousarray(np.concatenate(recs, axis=0)) if recs else np.zeros((0, grd.ndim))
    return cs, recoff, rec


def _ray_capacity(grd, cs, recoff, rec, steplen) -> int:
    """A generous first guess of the points of all rays (3x the straight-line distance)."""
    rstep = steplen * grd.spacing[0] if grd.kind in (0, 1) else steplen
    cap = 0
    for s in range(cs.shape[0]):
        for r in range(recoff[s], recoff[s + 1]):
            if grd.kind in (0, 1):
                d = float(np.linalg.norm(rec[r] - cs[s]))
            else:  # polar coordinates, degrees
                a, b = rec[r], cs[s]
                d = float(np.sqrt(max(a[0] ** 2 + b[0] ** 2 - 2 * a[0] * b[0] * np.cos(np.deg2rad(a[1] - b[1])), 0)))
            cap += int(3.0 * d / rstep) + 16
    return cap


def _split_rays(npts, pts, recoff, nd):
    out, k = [], 0
    for s in range(len(recoff) - 1):
        rays = []
        for r in range(recoff[s], recoff[s + 1]):
            n = int(npts[r])
            rays.append(pts[k * nd:(k + n) * nd].reshape(n, nd).copy())
            k += n
        out.append(rays)
    return out


def _traced(call, grd, cs, recoff, rec, steplen):
    """Runs a ray-tracing entry point, again with the exact size when the first guess was short."""
    npts = np.zeros(max(int(recoff[-1]), 1), dtype=np.int64)
    cap = _ray_capacity(grd, cs, recoff, rec, steplen)
    pts = np.zeros(cap * grd.ndim, dtype=np.float64)
    rc = call(npts, pts, cap)
    if rc == -5:  # EIK_ERR_OUT_OF_BUDGET: the rays are longer than the guess
        cap = int(npts[:recoff[-1]].sum())
        pts = np.zeros(cap * grd.ndim, dtype=np.float64)
        rc = call(npts, pts, cap)
    return rc, _split_rays(npts, pts, recoff, grd.ndim)


def tracerays(grd, ttime, coordsrc, coordrec, steplen: float = 0.01, ctx: Optional[Context] = None):
    """Rays from every receiver to its source through the traveltime grids ``ttime`` (one per
    source, as ``eiktraveltime(...; returntt=true)`` returns them) (eikutils.jl:201-213).
    Returns, per source, a list of (npoints, ndim) arrays, receiver first, source last."""
    ctx = ctx or default_context()
    cs, recoff, rec = _ray_inputs(grd, coordsrc, coordrec)
    assert len(ttime) == cs.shape[0], "length(ttime)==size(coordsrc,1)"
    for t in ttime:
        assert tuple(np.shape(t)) == tuple(grd.grsize), "size(ttime[s])==grd.grsize"
    tt = np.ascontiguousarray(np.concatenate([np.asarray(t, dtype=np.float64).ravel(order="F") for t in ttime]))
    g = _lib.grid_struct(grd)
    st = _lib.eik_stats()

    def call(npts, pts, cap):
        return ctx.L.eik_tracerays(ctx.h, C.byref(g), cs.shape[0], _lib.ptr(tt), _lib.ptr(cs), _lib.ptr(recoff),
                                   _lib.ptr(rec), float(steplen), _lib.ptr(npts), _lib.ptr(pts), cap, C.byref(st))
    rc, rays = _traced(call, grd, cs, recoff, rec, steplen)
    ctx.last_stats = st
    _lib.check(rc, ctx.h)
    return rays


_default: dict = {}
_dlock = threading.Lock()


def default_context(device: int = 0) -> Context:
    with _dlock:
        if device not in _default:
            _default[device] = Context(device)
        return _default[device]


def _with_model(vel, grd, fn, ctx: Optional[Context] = None):
    ctx = ctx or default_context()
    mid = ctx.upload(vel, grd)
    try:
        return fn(ctx, mid)
    finally:
        ctx.release(mid)


def eiktraveltime(vel, grd, coordsrc, coordrec, returntt: bool = False,
                  extraparams: Optional[ExtraParams] = None, ctx: Optional[Context] = None):
    """Traveltimes at the receivers (and optionally on the whole grid) for every source."""
    vel = np.asarray(vel, dtype=np.float64)
    assert 2 <= vel.ndim <= 3, "2<=ndims(vel)<=3"
    return _with_model(vel, grd, lambda c, m: c.traveltime(m, grd, coordsrc, coordrec, returntt, extraparams), ctx)


def eikgradient(vel, grd, coordsrc, coordrec, pickobs, stdobs, whichgrad,
                extraparams: Optional[ExtraParams] = None, ctx: Optional[Context] = None,
                nthreads: int = 1):
    """Gradient of the misfit w.r.t. velocity and/or source location, plus the misfit."""
    vel = np.asarray(vel, dtype=np.float64)
    assert 2 <= vel.ndim <= 3, "2<=ndims(vel)<=3"
    return _with_model(vel, grd, lambda c, m: c.gradient(m, grd, coordsrc, coordrec, pickobs, stdobs,
                                                         whichgrad, extraparams, nthreads), ctx)


def eikttimemisfit(velmod, grd, coordsrc, coordrec, ttpicksobs, stdobs,
                   extraparams: Optional[ExtraParams] = None, ctx: Optional[Context] = None) -> float:
    """0.5 * Σ_s Σ_r (t - obs)² / σ² through eiktraveltime (eikmaingrad.jl:1302-1328)."""
    picks = eiktraveltime(velmod, grd, coordsrc, coordrec, extraparams=extraparams, ctx=ctx)
    misf = 0.0
    for s in range(len(picks)):
        d = picks[s] - np.asarray(ttpicksobs[s])
        misf += float(np.sum(d * d / np.asarray(stdobs[s]) ** 2))
    return 0.5 * misf
