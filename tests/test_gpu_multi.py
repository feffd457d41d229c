"""Traveltimes of several models with grids of different sizes in one device pipeline
(eik_traveltime_multi): every source's picks and traveltime grid equal, bit for bit, what
eik_traveltime gives for its model alone (whose parity with the oracle the forward tests
pin). Covers 2D and 3D, Cartesian and spherical grids side by side, the refined start-up
and the plain one, a model with no sources, and the argument checks."""
import numpy as np
import pytest

from eikonalsolvers import Context, ExtraParams, _lib
from eikonalsolvers import configs as CF

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = Context(0)
    yield c
    c.close()


def _workloads_2d():
    a = CF.cfg1()
    b = CF.cfg2(scale=0.25, nsrc=5)
    c = CF.cfg1()
    c.coordsrc, c.coordrec = c.coordsrc[:0], []
    return [a, b, c]


def _workloads_3d():
    a = CF.cfg3(scale=0.25, nsrc=3, nrec_side=5)
    b = CF.cfg4(scale=0.2, nsrc=2)
    c = CF.cfg3(scale=0.125, nsrc=2, nrec_side=4)
    return [a, b, c]


def _check(ctx, ws, ep):
    ids = [ctx.upload(w.vel, w.grd) for w in ws]
    try:
        reqs = [(m, w.grd, w.coordsrc, w.coordrec) for m, w in zip(ids, ws)]
        multi = ctx.traveltime_multi(reqs, returntt=True, extraparams=ep)
        stats = ctx.last_stats
        assert stats.fwd_rounds > 0
        for m, w, (pk, tt) in zip(ids, ws, multi):
            assert len(pk) == len(w.coordsrc) and len(tt) == len(w.coordsrc)
            if len(w.coordsrc) == 0:
                continue
            apk, att = ctx.traveltime(m, w.grd, w.coordsrc, w.coordrec, returntt=True, extraparams=ep)
            for s in range(len(att)):
                assert tt[s].shape == att[s].shape
                assert int((tt[s] != att[s]).sum()) == 0, (w.name, s)
                assert np.array_equal(pk[s], apk[s]), (w.name, s)
        picks_only = ctx.traveltime_multi(reqs, extraparams=ep)
        for a, (pk, _) in zip(picks_only, multi):
            assert all(np.array_equal(x, y) for x, y in zip(a, pk))
    finally:
        for m in ids:
            ctx.release(m)


@pytest.mark.parametrize("refine", [True, False], ids=["refined", "plain"])
def test_multi_2d_equals_separate_calls(ctx, refine):
    _check(ctx, _workloads_2d(), ExtraParams(refinearoundsrc=refine))


@pytest.mark.parametrize("refine", [True, False], ids=["refined", "plain"])
def test_multi_3d_cartesian_and_spherical_equal_separate_calls(ctx, refine):
    _check(ctx, _workloads_3d(), ExtraParams(refinearoundsrc=refine))


def test_multi_rejects_mixed_dimensions(ctx):
    a, b = CF.cfg1(), CF.cfg3(scale=0.125, nsrc=1, nrec_side=3)
    ia, ib = ctx.upload(a.vel, a.grd), ctx.upload(b.vel, b.grd)
    try:
        with pytest.raises(AssertionError, match="one dimension"):
            ctx.traveltime_multi([(ia, a.grd, a.coordsrc, a.coordrec), (ib, b.grd, b.coordsrc, b.coordrec)])
        # the context stays usable
        ctx.traveltime(ia, a.grd, a.coordsrc, a.coordrec)
    finally:
        ctx.release(ia)
        ctx.release(ib)


def test_multi_checks_positions_per_model(ctx):
    a, b = CF.cfg1(), CF.cfg2(scale=0.25, nsrc=2)
    ia, ib = ctx.upload(a.vel, a.grd), ctx.upload(b.vel, b.grd)
    try:
        far = b.coordsrc.copy()
        far[1, 0] = a.grd.x[-1] + 1.0  # inside model a's grid, outside model b's
        assert far[1, 0] > b.grd.x[-1]
        with pytest.raises(AssertionError, match="source 1 outside"):
            ctx.traveltime_multi([(ia, a.grd, a.coordsrc, a.coordrec), (ib, b.grd, far, b.coordrec)])
    finally:
        ctx.release(ia)
        ctx.release(ib)
