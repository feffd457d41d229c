"""Failure detection on the GPU without faulting it: every device wait of the persistent
solves is bounded (global timer) and every round loop has a limit; running out of either
stops the kernel, which returns, and the call reports an error status while the context
stays usable. The reference's @warn sites come back as Python warnings.

* a round limit of 3 makes the forward solve stop: EIK_ERR_NOT_CONVERGED, then the same
  context with the limit lifted gives the oracle's traveltimes;
* a bounded wait on a flag that nothing sets (eik_selftest_wait) runs out after its limit:
  EIK_ERR_TIMEOUT, then the context still solves;
* a source exactly halfway between two nodes is shifted as the reference does
  (eikmainfwd.jl:1259-1319) and reported as a warning.
"""
import time

import numpy as np
import pytest

import eikoracle as O
from eikonalsolvers import Context, EikonalWarning, ExtraParams, Grid2DCart, _lib
from eikonalsolvers import configs as CF

pytestmark = pytest.mark.gpu
CODE = {name: code for code, name in _lib.ERRORS.items()}


@pytest.fixture(scope="module")
def ctx():
    c = Context(0)
    yield c
    c.close()


def _small():
    return CF.cfg3(scale=0.125, nsrc=2, nrec_side=4)


def _solve(ctx, w):
    mid = ctx.upload(w.vel, w.grd)
    try:
        return ctx.traveltime(mid, w.grd, w.coordsrc, w.coordrec, returntt=True)
    finally:
        ctx.release(mid)


def test_round_limit_reports_not_converged_and_the_context_recovers(ctx):
    w = _small()
    ctx.set_param("max_rounds", 3)
    try:
        with pytest.raises(_lib.EikError) as ei:
            _solve(ctx, w)
        assert ei.value.code == CODE["EIK_ERR_NOT_CONVERGED"]
        assert ctx.last_stats.err_mask != 0
    finally:
        ctx.set_param("max_rounds", 0)
    picks, tt = _solve(ctx, w)
    op, ott = O.eiktraveltime(w.vel, w.grd, w.coordsrc, w.coordrec, returntt=True, extraparams=ExtraParams())
    for a, b in zip(tt, ott):
        assert np.array_equal(a, b)


def test_bounded_wait_runs_out_and_the_context_recovers(ctx):
    t0 = time.perf_counter()
    rc = ctx.selftest_wait(0.25)
    dt = time.perf_counter() - t0
    assert rc == CODE["EIK_ERR_TIMEOUT"]
    assert 0.2 <= dt < 10.0
    assert b"wait ran out" in _lib.load().eik_last_error(None)
    assert ctx.selftest_wait(100.0) == CODE["EIK_ERR_ASSERT"]  # limits outside [1 ms, 10 s] are refused
    w = _small()
    picks, tt = _solve(ctx, w)
    assert all(np.isfinite(t).all() for t in tt)


def test_halfway_source_is_shifted_and_warned(ctx):
    grd = Grid2DCart(hgrid=0.5, cooinit=(0.0, 0.0), grsize=(40, 30))
    vel = np.full(grd.grsize, 2.0)
    cs = np.array([[10.25, 7.0]])  # halfway between x nodes 10.0 and 10.5
    rec = [np.array([[1.0, 1.0], [18.0, 13.0]])]
    mid = ctx.upload(vel, grd)
    try:
        with pytest.warns(EikonalWarning, match="halfway"):
            picks = ctx.traveltime(mid, grd, cs, rec)
    finally:
        ctx.release(mid)
    op, warn = O.eiktraveltime(vel, grd, cs, rec, extraparams=ExtraParams(), return_warn=True)
    assert warn & 0x2
    assert np.array_equal(picks[0], op[0])


def test_automatic_round_limit_reruns_the_call():
    """A forward solve that stops at the automatic round limit (no max_rounds set) is run
    once more with wider rounds and the full limit: the call succeeds, bit-identical to the
    oracle, and eik_stats.retries says so; with max_rounds set the limit is a hard stop."""
    import eikoracle as O
    from eikonalsolvers import Context
    from eikonalsolvers import configs as CF
    c = Context(0)
    try:
        w = CF.cfg1()
        mid = c.upload(w.vel, w.grd)
        op = O.eiktraveltime(w.vel, w.grd, w.coordsrc, w.coordrec, extraparams=w.extraparams)
        for cl in (1.0, 0.0):
            c.set_param("cluster_solve", cl)
            c.set_param("auto_round_limit", 5)
            pk = c.traveltime(mid, w.grd, w.coordsrc, w.coordrec)
            assert c.last_stats.retries == 1
            assert all(np.array_equal(a, b) for a, b in zip(pk, op))
            c.set_param("auto_round_limit", 0)
            c.traveltime(mid, w.grd, w.coordsrc, w.coordrec)
            assert c.last_stats.retries == 0
        po = [p + 0.01 for p in op]
        so = [0.01 * np.ones(p.shape) for p in op]
        g0 = c.gradient(mid, w.grd, w.coordsrc, w.coordrec, po, so, "gradvel")
        c.set_param("auto_round_limit", 5)
        g1 = c.gradient(mid, w.grd, w.coordsrc, w.coordrec, po, so, "gradvel")
        assert c.last_stats.retries == 1
        assert np.array_equal(g0[0], g1[0]) and g0[1] == g1[1]
        c.set_param("auto_round_limit", 0)
        c.release(mid)
    finally:
        c.close()
