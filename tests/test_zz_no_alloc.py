"""GPU test of eik_ttimemisfit_noalloc, the misfit entry point that allocates no device
memory. It exists for host programs that own all device memory and do not let an
operator call cudaMalloc (a framework op under the framework's own allocator, a sampler
callback that must not change the device's memory map); its scratch is a fixed array
inside the library that every call reuses.

The checks: on the same traveltime grids and observations its misfit equals the misfit of
the regular entry points (eik_traveltime's picks summed on the host, and eik_gradient's
misfit) within the misfit tolerance of the gradient tests, on two calls in a row (the
second with fewer sources and other observations, so stale scratch from the first call
would show); calls beyond its fixed capacity and receivers outside the grid are refused.

This file is collected last on purpose, so that a run stopping at the first failure has
already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from eikonalsolvers import Context, Grid2DSphere, Grid3DCart, Grid3DSphere, _lib
from eikonalsolvers import configs as CF

pytestmark = pytest.mark.gpu
MISFIT_RTOL = 1e-9
MAX_SOURCES = 65536  # the fixed scratch's capacity stated in include/eikcuda.h
CODE = {name: code for code, name in _lib.ERRORS.items()}


def _host_misfit(picks, pobs, sobs):
    m = 0.0
    for p, o, s in zip(picks, pobs, sobs):
        d = np.asarray(p) - np.asarray(o)
        m += float(np.sum(d * d / np.asarray(s) ** 2))
    return 0.5 * m


def _case(kind):
    if kind == "2D":
        w = CF.cfg2(scale=0.125, nsrc=5)
        return w.grd, w.vel, w.coordsrc, w.coordrec
    if kind == "sphere2D":
        # polar grid; receivers include the last node of both axes (the i == n corner rule)
        grd = Grid2DSphere(Δr=2.0, Δθ=0.25, cooinit=(5800.0, 10.0), grsize=(40, 50))
        r = np.array(grd.r)[:, None]
        vel = np.ascontiguousarray(np.broadcast_to(5.0 + 0.01 * (6000.0 - r), grd.grsize))
        cs = np.array([[5800.0 + 17.3 * 2.0, 10.0 + 21.4 * 0.25], [5800.0 + 9.0 * 2.0, 10.0 + 30.6 * 0.25],
                       [5800.0 + 25.5 * 2.0, 10.0 + 7.2 * 0.25]])
        th = np.linspace(10.5, grd.θ[-1], 9)
        rec = np.column_stack([np.full(9, grd.r[-1]), th])
        rec = np.vstack([rec, [[5830.3, grd.θ[-1]], [grd.r[-1], grd.θ[-1]]]])
        return grd, vel, cs, [rec.copy() for _ in range(3)]
    if kind == "sphere3D":
        grd = Grid3DSphere(Δr=2.0, Δθ=0.25, Δφ=0.3, cooinit=(5800.0, 40.0, 10.0), grsize=(18, 20, 22))
        r = np.array(grd.r)[:, None, None]
        vel = np.ascontiguousarray(np.broadcast_to(5.0 + 0.01 * (6000.0 - r), grd.grsize))
        cs = np.array([[5800.0 + 8.3 * 2.0, 40.0 + 9.4 * 0.25, 10.0 + 10.6 * 0.3],
                       [5800.0 + 4.6 * 2.0, 40.0 + 12.2 * 0.25, 10.0 + 6.3 * 0.3],
                       [5800.0 + 12.1 * 2.0, 40.0 + 5.7 * 0.25, 10.0 + 15.2 * 0.3]])
        th = np.linspace(40.3, grd.θ[-1], 4)
        ph = np.linspace(10.4, grd.φ[-1], 4)
        rec = np.array([[grd.r[-1], a, b] for a in th for b in ph] + [[5810.7, grd.θ[-1], grd.φ[-1]]])
        return grd, vel, cs, [rec.copy() for _ in range(3)]
    grd = Grid3DCart(hgrid=0.1, cooinit=(0.0, 0.0, 0.0), grsize=(24, 20, 18))
    vel = CF.layered_3d(grd.grsize, seed=5)
    rng = np.random.default_rng(21)
    cs = np.column_stack([rng.uniform(0.3, 2.0, 4), rng.uniform(0.3, 1.6, 4), rng.uniform(0.9, 1.5, 4)])
    xr, yr = np.linspace(0.0, grd.x[-1], 5), np.linspace(0.0, grd.y[-1], 4)
    rec = np.array([[a, b, 0.0] for b in yr for a in xr])
    return grd, vel, cs, [rec.copy() for _ in range(4)]


def _flat(recs, pobs, sobs):
    off = np.zeros(len(recs) + 1, dtype=np.int64)
    for i, r in enumerate(recs):
        off[i + 1] = off[i] + r.shape[0]
    return (off, np.ascontiguousarray(np.concatenate(recs)), np.ascontiguousarray(np.concatenate(pobs)),
            np.ascontiguousarray(np.concatenate(sobs)))


def _noalloc(L, torch, grd, tt, recs, pobs, sobs):
    """Calls the entry point through the C ABI with every array in device memory."""
    dev = torch.device("cuda", 0)
    ttg = torch.from_numpy(np.ascontiguousarray(np.stack([t.ravel(order="F") for t in tt]))).to(dev)
    off, rec, po, so = _flat(recs, pobs, sobs)
    d_rec, d_po, d_so = (torch.from_numpy(a).to(dev) for a in (rec, po, so))
    out = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
    g = _lib.grid_struct(grd)
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    P = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    rc = L.eik_ttimemisfit_noalloc(C.byref(g), len(tt), P(ttg), _lib.ptr(off), P(d_rec), P(d_po), P(d_so),
                                   P(out), stream)
    return rc, float(out.item())


@pytest.mark.parametrize("kind", ["2D", "3D", "sphere2D", "sphere3D"])
def test_noalloc_misfit_matches_regular_entry_points(kind):
    torch = pytest.importorskip("torch")
    grd, vel, cs, recs = _case(kind)
    ctx = Context(0)
    L = ctx.L
    try:
        mid = ctx.upload(vel, grd)
        mobs = ctx.upload(vel * 1.03, grd)
        picks, tt = ctx.traveltime(mid, grd, cs, recs, returntt=True)
        rng = np.random.default_rng(5)
        pobs = [p + rng.normal(0.0, 0.01, p.shape) for p in ctx.traveltime(mobs, grd, cs, recs)]
        sobs = [0.01 * np.ones(p.shape) for p in pobs]
        # call 1: every source, against eik_traveltime's picks and eik_gradient's misfit
        rc, m1 = _noalloc(L, torch, grd, tt, recs, pobs, sobs)
        assert rc == 0, _lib.load().eik_last_error(None)
        ref1 = _host_misfit(picks, pobs, sobs)
        _, mg = ctx.gradient(mid, grd, cs, recs, pobs, sobs, "gradvel")  # gradvel runs on every grid kind
        assert abs(m1 - ref1) <= MISFIT_RTOL * abs(ref1), (m1, ref1)
        assert abs(m1 - mg) <= MISFIT_RTOL * abs(mg), (m1, mg)
        # call 2, right after: fewer sources and other observations
        k = max(1, len(tt) - 2)
        pobs2 = [o + 0.02 for o in pobs[:k]]
        sobs2 = [2.0 * s for s in sobs[:k]]
        rc, m2 = _noalloc(L, torch, grd, tt[:k], recs[:k], pobs2, sobs2)
        assert rc == 0, _lib.load().eik_last_error(None)
        ref2 = _host_misfit(picks[:k], pobs2, sobs2)
        assert abs(m2 - ref2) <= MISFIT_RTOL * abs(ref2), (m2, ref2)
        assert m2 != m1
        ctx.release(mobs)
        ctx.release(mid)
    finally:
        ctx.close()


def test_noalloc_misfit_refuses_what_it_cannot_hold():
    torch = pytest.importorskip("torch")
    L = _lib.load()
    grd, vel, cs, recs = _case("2D")
    g = _lib.grid_struct(grd)
    off = np.zeros(MAX_SOURCES + 2, dtype=np.int64)
    one = torch.zeros(1, dtype=torch.float64, device="cuda:0")
    P = C.c_void_p(one.data_ptr())
    rc = L.eik_ttimemisfit_noalloc(C.byref(g), MAX_SOURCES + 1, P, _lib.ptr(off), P, P, P, P, None)
    assert rc == CODE["EIK_ERR_OUT_OF_BUDGET"]
    assert b"fixed scratch" in L.eik_last_error(None)
    # a receiver outside the grid is reported, nothing is read out of bounds
    ctx = Context(0)
    try:
        mid = ctx.upload(vel, grd)
        picks, tt = ctx.traveltime(mid, grd, cs[:1], recs[:1], returntt=True)
        ctx.release(mid)
    finally:
        ctx.close()
    bad = recs[0].copy()
    bad[0, 0] = grd.x[-1] + 1.0
    rc, _ = _noalloc(L, torch, grd, tt, [bad], [picks[0]], [np.ones(picks[0].shape)])
    assert rc == CODE["EIK_ERR_ASSERT"]
    assert b"outside the grid" in L.eik_last_error(None)
