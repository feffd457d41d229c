"""GPU ray tracing (eik_tracerays / eik_traveltime_rays) against the oracle's tracerays on
the same traveltime grids. Cartesian rays are bit-identical (the kernels do the oracle's
arithmetic operation for operation); on a Grid2DSphere the step also calls sin, cos and
atan2, whose last bits may differ between CUDA and the host library, so the rays agree to
1e-9 relative and in length to one point."""
import numpy as np
import pytest

import eikoracle as O
import refcases as RC
from eikonalsolvers import Context, ExtraParams, Grid2DSphere, Grid3DSphere, tracerays
from eikonalsolvers import configs as CF

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = Context(0)
    yield c
    c.close()


def _cart_cases():
    c2 = [c for c in RC.all_forward_cases() if c["name"] == "2Dlingrad0"][0]
    w3 = CF.cfg3(scale=0.125, nsrc=3, nrec_side=4)
    w2 = CF.cfg2(scale=0.125, nsrc=3)
    return [("2Dlingrad", c2["vel"], c2["grd"], c2["coordsrc"], c2["coordrec"]),
            ("cfg2-small", w2.vel, w2.grd, w2.coordsrc, [r[::20] for r in w2.coordrec]),
            ("cfg3-small", w3.vel, w3.grd, w3.coordsrc, w3.coordrec)]


@pytest.mark.parametrize("case", _cart_cases(), ids=lambda c: c[0])
def test_cartesian_rays_are_bit_identical_to_the_oracle(ctx, case):
    _, vel, grd, cs, rec = case
    _, tt = O.eiktraveltime(vel, grd, cs, rec, returntt=True, extraparams=ExtraParams())
    got = tracerays(grd, tt, cs, rec, steplen=0.01, ctx=ctx)
    want = O.tracerays(grd, tt, cs, rec, steplen=0.01)
    assert len(got) == len(want)
    for gs, ws in zip(got, want):
        assert len(gs) == len(ws)
        for g, w in zip(gs, ws):
            assert g.shape == w.shape and np.array_equal(g, w)


def test_traveltime_rays_keeps_the_grids_on_the_device(ctx):
    """Picks and rays from one device pipeline equal eik_traveltime's picks and the rays of
    its returned grids."""
    w = CF.cfg3(scale=0.125, nsrc=3, nrec_side=4)
    mid = ctx.upload(w.vel, w.grd)
    try:
        picks, rays = ctx.traveltime_rays(mid, w.grd, w.coordsrc, w.coordrec, steplen=0.02)
        p2, tt = ctx.traveltime(mid, w.grd, w.coordsrc, w.coordrec, returntt=True)
    finally:
        ctx.release(mid)
    assert all(np.array_equal(a, b) for a, b in zip(picks, p2))
    r2 = tracerays(w.grd, tt, w.coordsrc, w.coordrec, steplen=0.02, ctx=ctx)
    for a, b in zip(rays, r2):
        assert all(np.array_equal(x, y) for x, y in zip(a, b))


def test_polar_rays_match_the_oracle(ctx):
    # spacings of about 2 km on both axes: with a much coarser θ axis the reference's descent
    # can circle a source it cannot resolve to within Δr·sqrt(2) and never stop
    g = Grid2DSphere(Δr=2.0, Δθ=0.02, cooinit=(5800.0, 10.0), grsize=(40, 60))
    r = np.array(g.r)[:, None]
    vel = np.ascontiguousarray(np.broadcast_to(5.0 + 0.01 * (6000.0 - r), g.grsize))
    cs = np.array([[5800.0 + 17.3 * 2.0, 10.0 + 31.4 * 0.02]])
    rec = [np.vstack([np.column_stack([np.full(6, 5878.0), np.linspace(10.1, 11.1, 6)]),
                      [[5806.0, 10.2], [5860.0, 11.15]]])]
    _, tt = O.eiktraveltime(vel, g, cs, rec, returntt=True)
    got = tracerays(g, tt, cs, rec, steplen=0.5, ctx=ctx)[0]
    want = O.tracerays(g, tt, cs, rec, steplen=0.5)[0]
    for a, b in zip(got, want):
        assert abs(a.shape[0] - b.shape[0]) <= 1
        n = min(a.shape[0], b.shape[0]) - 1
        assert np.allclose(a[:n], b[:n], rtol=1e-9, atol=0)
        assert np.array_equal(a[-1], b[-1])


def test_ray_errors(ctx):
    g3 = Grid3DSphere(Δr=2.0, Δθ=0.25, Δφ=0.3, cooinit=(5800.0, 40.0, 10.0), grsize=(8, 8, 8))
    with pytest.raises(RuntimeError, match="not yet implemented"):
        tracerays(g3, [np.ones(g3.grsize)], np.array([[5806.0, 41.0, 11.0]]), [np.array([[5810.0, 41.5, 11.5]])],
                  ctx=ctx)


def test_rays_that_outgrow_their_room_are_traced_again(ctx):
    """ray_room 0 gives every ray a room of 16 points in the single pass, so the long ones take
    the second pass: same rays as with the default room."""
    w = CF.cfg3(scale=0.125, nsrc=2, nrec_side=3)
    _, tt = O.eiktraveltime(w.vel, w.grd, w.coordsrc, w.coordrec, returntt=True)
    want = tracerays(w.grd, tt, w.coordsrc, w.coordrec, steplen=0.02, ctx=ctx)
    ctx.set_param("ray_room", 0.0)
    try:
        got = tracerays(w.grd, tt, w.coordsrc, w.coordrec, steplen=0.02, ctx=ctx)
    finally:
        ctx.set_param("ray_room", 3.0)
    for a, b in zip(got, want):
        assert all(np.array_equal(x, y) for x, y in zip(a, b))


def test_polar_traveltime_rays(ctx):
    """Picks and rays in one device pipeline on a Grid2DSphere model equal eik_traveltime's
    picks and the rays of its returned grids."""
    g = Grid2DSphere(Δr=2.0, Δθ=0.02, cooinit=(5800.0, 10.0), grsize=(40, 60))
    r = np.array(g.r)[:, None]
    vel = np.ascontiguousarray(np.broadcast_to(5.0 + 0.01 * (6000.0 - r), g.grsize))
    cs = np.array([[5800.0 + 17.3 * 2.0, 10.0 + 31.4 * 0.02]])
    rec = [np.column_stack([np.full(4, 5878.0), np.linspace(10.1, 11.1, 4)])]
    mid = ctx.upload(vel, g)
    try:
        picks, rays = ctx.traveltime_rays(mid, g, cs, rec, steplen=0.5)
        p2, tt = ctx.traveltime(mid, g, cs, rec, returntt=True)
    finally:
        ctx.release(mid)
    assert all(np.array_equal(a, b) for a, b in zip(picks, p2))
    r2 = tracerays(g, tt, cs, rec, steplen=0.5, ctx=ctx)
    assert all(np.array_equal(x, y) for x, y in zip(rays[0], r2[0]))
