"""ctypes binding of the oracle (CPU restatement of EikonalSolvers.jl 0.15.3).

TEST INFRASTRUCTURE ONLY. Imported by ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` as the checker / timed CPU reference; the GPU product
path never imports it.

Parity status: the reference is Julia and no Julia toolchain exists here, so the
oracle is pinned through the reference's own known-answer and finite-difference tests
(test/test_cartesian_2D.jl, test/test_cartesian_3D.jl), ported in tests/test_oracle_*.py.
Bitwise agreement with the Julia implementation itself is unverified ("parity unpinned"
at the bit level; pinned at the reference tests' tolerances).

Grids are duck-typed: any object with ``kind``, ``ndim``, ``grsize``, ``spacing`` and
``cooinit`` (the classes of ``eikonalsolvers.structs`` qualify).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import List, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

WHICHGRAD = {"gradvel": 1, "gradsrcloc": 2, "gradvelandsrcloc": 3}
_PK = {"serial": 0, "sharedmem": 1, "distribmem": 2}


class OracleError(RuntimeError):
    pass


class OracleAssertionError(OracleError, AssertionError):
    pass


def build() -> str:
    """Compile the oracle library in place (make) and return its path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "libeikoracle.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libeikoracle.so")
        srcs = [os.path.join(_HERE, f) for f in ("fwd.cpp", "grad.cpp", "rays.cpp", "capi.cpp", "eikoracle.hpp")]
        if not os.path.exists(path) or any(os.path.getmtime(s) > os.path.getmtime(path) for s in srcs if os.path.exists(s)):
            build()
        L = C.CDLL(path)
        P = C.c_void_p
        L.eikor_traveltime.argtypes = [C.c_int, P, P, P, P, C.c_int64, P, P, P, C.c_int, C.c_int64,
                                       C.c_int64, C.c_int, C.c_int, P, P, P, C.c_char_p, C.c_int]
        L.eikor_traveltime.restype = C.c_int
        L.eikor_gradient.argtypes = [C.c_int, P, P, P, P, C.c_int64, P, P, P, P, P, C.c_int, C.c_int,
                                     C.c_int64, C.c_int64, C.c_int64, C.c_int64, C.c_int, C.c_int,
                                     P, P, P, P, C.c_char_p, C.c_int]
        L.eikor_gradient.restype = C.c_int
        L.eikor_forward_debug.argtypes = [C.c_int, P, P, P, P, P, C.c_int, C.c_int64, C.c_int64, P,
                                          P, P, P, C.c_int64, P, P, C.c_int64, P, P, P, P, P,
                                          C.c_char_p, C.c_int]
        L.eikor_forward_debug.restype = C.c_int
        L.eikor_range_value.argtypes = [C.c_double, C.c_double, C.c_int64, C.c_int64]
        L.eikor_range_value.restype = C.c_double
        L.eikor_smoothgradient.argtypes = [C.c_int, P, P, P, C.c_int64, P, C.c_char_p, C.c_int]
        L.eikor_smoothgradient.restype = C.c_int
        L.eikor_tracerays.argtypes = [C.c_int, P, P, P, P, C.c_int64, P, P, P, C.c_double, C.c_int64, P, P,
                                      C.c_int64, P, C.c_char_p, C.c_int]
        L.eikor_tracerays.restype = C.c_int
        _LIB = L
    return _LIB


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def _grid_arrays(grd):
    nd = grd.ndim
    gs = np.array(list(grd.grsize) + [1] * (3 - nd), dtype=np.int64)
    sp = np.array(list(grd.spacing) + [0.0] * (3 - nd), dtype=np.float64)
    co = np.array(list(grd.cooinit) + [0.0] * (3 - nd), dtype=np.float64)
    return gs, sp, co


def _check(rc: int, buf):
    if rc == 0:
        return
    msg = buf.value.decode(errors="replace")
    if rc == 1:
        raise OracleAssertionError(msg)
    raise OracleError(msg)


def _flatten(vel, grd, coordsrc, coordrec):
    vel = np.asarray(vel, dtype=np.float64)
    assert tuple(vel.shape) == tuple(grd.grsize)
    velf = np.ascontiguousarray(np.asfortranarray(vel).ravel(order="F"))
    cs = np.ascontiguousarray(np.atleast_2d(np.asarray(coordsrc, dtype=np.float64)))
    if isinstance(coordrec, np.ndarray) and coordrec.dtype != object:
        coordrec = [coordrec]
    recs = [np.ascontiguousarray(np.atleast_2d(np.asarray(r, dtype=np.float64))) for r in coordrec]
    assert cs.shape[0] == len(recs), "size(coordsrc,1)==length(coordrec)"
    recoff = np.zeros(len(recs) + 1, dtype=np.int64)
    for s, r in enumerate(recs):
        recoff[s + 1] = recoff[s] + r.shape[0]
    rec = np.ascontiguousarray(np.concatenate(recs, axis=0)) if recs else np.zeros((0, grd.ndim))
    return velf, cs, recoff, rec


def _ep(extraparams):
    if extraparams is None:
        return dict(refine=1, ds=5, nr=3, rs=3, kern=0, pk=0)
    return dict(refine=int(extraparams.refinearoundsrc), ds=extraparams.grdrefpars.downscalefactor,
                nr=extraparams.grdrefpars.noderadius, rs=extraparams.radiussmoothgradsrc,
                kern=extraparams.smoothgradkern, pk=_PK[extraparams.parallelkind])


def eiktraveltime(vel, grd, coordsrc, coordrec, returntt: bool = False, extraparams=None,
                  nthreads: int = 1, return_warn: bool = False):
    """Oracle of ``eiktraveltime`` (eikmainfwd.jl:33-143)."""
    L = lib()
    velf, cs, recoff, rec = _flatten(vel, grd, coordsrc, coordrec)
    gs, sp, co = _grid_arrays(grd)
    nsrc = cs.shape[0]
    ep = _ep(extraparams)
    picks = np.zeros(int(recoff[-1]), dtype=np.float64)
    N = int(np.prod(grd.grsize))
    ttg = np.zeros(nsrc * N, dtype=np.float64) if returntt else None
    warn = np.zeros(1, dtype=np.uint32)
    buf = C.create_string_buffer(512)
    rc = L.eikor_traveltime(grd.kind, _p(gs), _p(sp), _p(co), _p(velf), nsrc, _p(cs), _p(recoff),
                            _p(rec), ep["refine"], ep["ds"], ep["nr"], ep["pk"], int(nthreads),
                            _p(picks), _p(ttg) if ttg is not None else None, _p(warn), buf, 512)
    _check(rc, buf)
    pk = [picks[recoff[s]:recoff[s + 1]].copy() for s in range(nsrc)]
    out = [pk]
    if returntt:
        out.append([ttg[s * N:(s + 1) * N].reshape(grd.grsize, order="F").copy() for s in range(nsrc)])
    if return_warn:
        out.append(int(warn[0]))
    return out[0] if len(out) == 1 else tuple(out)


def eikgradient(vel, grd, coordsrc, coordrec, pickobs, stdobs, whichgrad, extraparams=None,
                nthreads: int = 1, return_warn: bool = False):
    """Oracle of ``eikgradient`` (eikmaingrad.jl:31-164)."""
    L = lib()
    wg = whichgrad.lstrip(":") if isinstance(whichgrad, str) else whichgrad
    assert wg in WHICHGRAD, "Symbol 'whichgrad' not in (:gradvel, :gradsrcloc, :gradvelandsrcloc)"
    velf, cs, recoff, rec = _flatten(vel, grd, coordsrc, coordrec)
    gs, sp, co = _grid_arrays(grd)
    nsrc = cs.shape[0]
    assert len(pickobs) == nsrc and len(stdobs) == nsrc
    po = np.ascontiguousarray(np.concatenate([np.asarray(p, dtype=np.float64).ravel() for p in pickobs]))
    so = np.ascontiguousarray(np.concatenate([np.asarray(p, dtype=np.float64).ravel() for p in stdobs]))
    assert po.size == recoff[-1] and so.size == recoff[-1]
    ep = _ep(extraparams)
    N = int(np.prod(grd.grsize))
    gv = np.zeros(N, dtype=np.float64)
    gsrc = np.zeros(nsrc * grd.ndim, dtype=np.float64)
    misf = np.zeros(1, dtype=np.float64)
    warn = np.zeros(1, dtype=np.uint32)
    buf = C.create_string_buffer(512)
    rc = L.eikor_gradient(grd.kind, _p(gs), _p(sp), _p(co), _p(velf), nsrc, _p(cs), _p(recoff), _p(rec),
                          _p(po), _p(so), WHICHGRAD[wg], ep["refine"], ep["ds"], ep["nr"], ep["rs"],
                          ep["kern"], ep["pk"], int(nthreads), _p(gv), _p(gsrc), _p(misf), _p(warn),
                          buf, 512)
    _check(rc, buf)
    gradvel = gv.reshape(grd.grsize, order="F")
    gradsrc = gsrc.reshape(nsrc, grd.ndim)
    res = {"gradvel": (gradvel, misf[0]), "gradsrcloc": (gradsrc, misf[0]),
           "gradvelandsrcloc": (gradvel, gradsrc, misf[0])}[wg]
    if return_warn:
        return res + (int(warn[0]),)
    return res


def eikttimemisfit(velmod, grd, coordsrc, coordrec, ttpicksobs, stdobs, extraparams=None,
                   nthreads: int = 1) -> float:
    """Oracle of ``eikttimemisfit`` (eikmaingrad.jl:1302-1328)."""
    picks = eiktraveltime(velmod, grd, coordsrc, coordrec, extraparams=extraparams, nthreads=nthreads)
    misf = 0.0
    for s in range(len(picks)):
        d = picks[s] - np.asarray(ttpicksobs[s])
        misf += float(np.sum(d * d / (np.asarray(stdobs[s]) ** 2)))
    return 0.5 * misf


def forward_debug(vel, grd, src, extraparams=None):
    """One-source forward with adjoint bookkeeping; returns a dict of the FMM state."""
    L = lib()
    velf, cs, _, _ = _flatten(vel, grd, np.atleast_2d(src), [np.zeros((1, grd.ndim)) + np.asarray(grd.cooinit)])
    gs, sp, co = _grid_arrays(grd)
    ep = _ep(extraparams)
    N = int(np.prod(grd.grsize))
    tt = np.zeros(N)
    codes = np.zeros(N * grd.ndim, dtype=np.int8)
    fmmpos = np.zeros(N, dtype=np.int32)
    srcpts = np.zeros(max(N, 1), dtype=np.int64)
    stats = np.zeros(5, dtype=np.int64)
    fine_n = np.zeros(3, dtype=np.int64)
    cap = 200000
    fine_tt = np.zeros(cap)
    fine_status = np.zeros(cap, dtype=np.uint8)
    fine_pos = np.zeros(cap, dtype=np.int32)
    fine_nacc = np.zeros(1, dtype=np.int64)
    batch = np.zeros(N, dtype=np.int32)
    buf = C.create_string_buffer(512)
    src = np.ascontiguousarray(np.asarray(src, dtype=np.float64).ravel())
    rc = L.eikor_forward_debug(grd.kind, _p(gs), _p(sp), _p(co), _p(velf), _p(src), ep["refine"], ep["ds"],
                               ep["nr"], _p(tt), _p(codes), _p(fmmpos), _p(srcpts), srcpts.size, _p(stats),
                               _p(fine_n), cap, _p(fine_tt), _p(fine_status), _p(fine_pos), _p(fine_nacc),
                               _p(batch), buf, 512)
    _check(rc, buf)
    out = dict(tt=tt.reshape(grd.grsize, order="F"), codes=codes.reshape(N, grd.ndim),
               fmmpos=fmmpos, srcpts=srcpts[:stats[3]].copy(), pops=int(stats[0]),
               nonmonotone=int(stats[1]), max_batch=int(stats[2]), warn=int(stats[4]),
               batch=batch.reshape(grd.grsize, order="F"))
    if ep["refine"]:
        fn = tuple(int(x) for x in fine_n[:grd.ndim])
        nf = int(np.prod(fn))
        out.update(fine_n=fn, fine_nacc=int(fine_nacc[0]))
        if nf <= cap:
            out.update(fine_tt=fine_tt[:nf].reshape(fn, order="F").copy(),
                       fine_status=fine_status[:nf].reshape(fn, order="F").copy(),
                       fine_fmmpos=fine_pos[:nf].reshape(fn, order="F").copy())
    return out


def range_value(start: float, step: float, length: int, i1: int) -> float:
    return lib().eikor_range_value(start, step, length, i1)


def smoothgradient(l: int, grd, grad) -> np.ndarray:
    L = lib()
    gs, sp, co = _grid_arrays(grd)
    g = np.ascontiguousarray(np.asfortranarray(np.asarray(grad, dtype=np.float64)).ravel(order="F"))
    buf = C.create_string_buffer(512)
    _check(L.eikor_smoothgradient(grd.kind, _p(gs), _p(sp), _p(co), int(l), _p(g), buf, 512), buf)
    return g.reshape(grd.grsize, order="F")


def tracerays(grd, ttime, coordsrc, coordrec, steplen: float = 0.01, max_steps: int = 1 << 24):
    """Oracle of ``tracerays`` (eikutils.jl:201-328): per source, per receiver, the ray as an
    (npoints, ndim) array from the receiver to the source."""
    L = lib()
    cs = np.ascontiguousarray(np.atleast_2d(np.asarray(coordsrc, dtype=np.float64)))
    nsrc = cs.shape[0]
    recs = [np.ascontiguousarray(np.atleast_2d(np.asarray(r, dtype=np.float64))) for r in coordrec]
    recoff = np.zeros(nsrc + 1, dtype=np.int64)
    for i, r in enumerate(recs):
        recoff[i + 1] = recoff[i] + r.shape[0]
    rec = np.ascontiguousarray(np.concatenate(recs))
    tt = np.ascontiguousarray(np.concatenate([np.asarray(t, dtype=np.float64).ravel(order="F") for t in ttime]))
    gs, sp, co = _grid_arrays(grd)
    npts = np.zeros(int(recoff[-1]), dtype=np.int64)
    total = np.zeros(1, dtype=np.int64)
    buf = C.create_string_buffer(512)
    _check(L.eikor_tracerays(grd.kind, _p(gs), _p(sp), _p(co), _p(tt), nsrc, _p(cs), _p(recoff), _p(rec),
                             float(steplen), int(max_steps), _p(npts), None, 0, _p(total), buf, 512), buf)
    pts = np.zeros(int(total[0]) * grd.ndim, dtype=np.float64)
    _check(L.eikor_tracerays(grd.kind, _p(gs), _p(sp), _p(co), _p(tt), nsrc, _p(cs), _p(recoff), _p(rec),
                             float(steplen), int(max_steps), _p(npts), _p(pts), int(total[0]), _p(total), buf,
                             512), buf)
    out, k = [], 0
    for s in range(nsrc):
        rays = []
        for r in range(recoff[s], recoff[s + 1]):
            n = int(npts[r])
            rays.append(pts[k * grd.ndim:(k + n) * grd.ndim].reshape(n, grd.ndim).copy())
            k += n
        out.append(rays)
    return out
