"""GPU forward parity: libeikcuda (through the C ABI) against the oracle on the same
inputs. Contract: traveltimes within 1e-6 relative of the reference's FP64 result; the
Cartesian cases are expected to agree bit for bit (same operations, same order)."""
import numpy as np
import pytest

import eikoracle as O
import refcases as RC
from eikonalsolvers import Context, ExtraParams, GridRefinementPars
from eikonalsolvers import configs as CF

pytestmark = pytest.mark.gpu
RTOL = 1e-6


@pytest.fixture(scope="module")
def ctx():
    c = Context(0)
    yield c
    c.close()


def _run(ctx, vel, grd, cs, rec, ep):
    mid = ctx.upload(vel, grd)
    try:
        picks, tt = ctx.traveltime(mid, grd, cs, rec, returntt=True, extraparams=ep)
    finally:
        ctx.release(mid)
    return picks, tt


def _compare(picks, tt, opicks, ott, bitwise):
    for s in range(len(tt)):
        rel = np.abs(tt[s] - ott[s]) / np.abs(ott[s])
        rel[ott[s] == 0] = np.abs(tt[s] - ott[s])[ott[s] == 0]
        assert rel.max() <= RTOL, (s, rel.max(), int((tt[s] != ott[s]).sum()))
        prel = np.abs(picks[s] - opicks[s]) / np.abs(opicks[s])
        assert prel.max() <= RTOL
        if bitwise:
            assert int((tt[s] != ott[s]).sum()) == 0, f"{int((tt[s] != ott[s]).sum())} nodes differ"
            assert np.array_equal(picks[s], opicks[s])


@pytest.mark.parametrize("case", RC.all_forward_cases(), ids=lambda c: c["name"])
def test_reference_cases(ctx, case):
    picks, tt = _run(ctx, case["vel"], case["grd"], case["coordsrc"], case["coordrec"], case["extraparams"])
    op, ott = O.eiktraveltime(case["vel"], case["grd"], case["coordsrc"], case["coordrec"], returntt=True,
                              extraparams=case["extraparams"])
    _compare(picks, tt, op, ott, bitwise=True)
    # and the reference's own known-answer bound
    d = tt[0] - case["analytic"]
    assert np.abs(d).max() <= case["tolerr"] and np.linalg.norm(d) <= case["tolnorm"]


def test_cfg1_full(ctx):
    w = CF.cfg1()
    picks, tt = _run(ctx, w.vel, w.grd, w.coordsrc, w.coordrec, w.extraparams)
    op, ott = O.eiktraveltime(w.vel, w.grd, w.coordsrc, w.coordrec, returntt=True, extraparams=w.extraparams)
    _compare(picks, tt, op, ott, bitwise=True)


@pytest.mark.parametrize("refine", [True, False])
def test_cfg2_small(ctx, refine):
    w = CF.cfg2(scale=0.25, nsrc=6)
    ep = ExtraParams(refinearoundsrc=refine)
    picks, tt = _run(ctx, w.vel, w.grd, w.coordsrc, w.coordrec, ep)
    op, ott = O.eiktraveltime(w.vel, w.grd, w.coordsrc, w.coordrec, returntt=True, extraparams=ep)
    _compare(picks, tt, op, ott, bitwise=True)


@pytest.mark.parametrize("refine", [True, False])
def test_cfg3_small(ctx, refine):
    w = CF.cfg3(scale=0.25, nsrc=3, nrec_side=5)
    ep = ExtraParams(refinearoundsrc=refine)
    picks, tt = _run(ctx, w.vel, w.grd, w.coordsrc, w.coordrec, ep)
    op, ott = O.eiktraveltime(w.vel, w.grd, w.coordsrc, w.coordrec, returntt=True, extraparams=ep)
    _compare(picks, tt, op, ott, bitwise=True)


def test_refinement_params(ctx):
    w = CF.cfg3(scale=0.125, nsrc=2, nrec_side=4)
    ep = ExtraParams(grdrefpars=GridRefinementPars(downscalefactor=3, noderadius=2))
    picks, tt = _run(ctx, w.vel, w.grd, w.coordsrc, w.coordrec, ep)
    op, ott = O.eiktraveltime(w.vel, w.grd, w.coordsrc, w.coordrec, returntt=True, extraparams=ep)
    _compare(picks, tt, op, ott, bitwise=True)


def test_asserts_mirror_reference(ctx):
    import refcases
    c = RC.fwd_2D_constvel()[0]
    bad = c["vel"].copy()
    bad[3, 4] = 0.0
    with pytest.raises(AssertionError):
        _run(ctx, bad, c["grd"], c["coordsrc"], c["coordrec"], c["extraparams"])
    out = c["coordsrc"].copy()
    out[0, 0] = -1.0
    with pytest.raises(AssertionError):
        _run(ctx, c["vel"], c["grd"], out, c["coordrec"], c["extraparams"])


@pytest.mark.parametrize("which", ["3Dconst1", "3Dlingrad3", "2Dconst3", "cfg3"])
def test_refined_startup_fixed_point_equals_heap_replay(ctx, which):
    """The refined window solved as a fixed point with its stop reconstructed from keys gives
    the same traveltimes as the exact heap replay (sources with a tied stop are replayed)."""
    if which == "cfg3":
        w = CF.cfg3(scale=0.25, nsrc=6, nrec_side=5)
        vel, grd, cs, rec, ep = w.vel, w.grd, w.coordsrc, w.coordrec, ExtraParams()
    else:
        c = [c for c in RC.all_forward_cases() if c["name"] == which][0]
        vel, grd, cs, rec, ep = c["vel"], c["grd"], c["coordsrc"], c["coordrec"], c["extraparams"]
    out = []
    for mode in (1, 0):
        ctx.set_param("fine_replay", mode)
        out.append(_run(ctx, vel, grd, cs, rec, ep))
    ctx.set_param("fine_replay", 0)
    for a, b in zip(out[0][1], out[1][1]):
        assert np.array_equal(a, b)


def test_many_sources_batched_at_128cubed_match_the_oracle(ctx):
    """16 sources of the 3D layered workload at 128^3 in one call (many sources in flight in
    every round): the sources checked are bit-identical to the oracle's FMM."""
    w = CF.cfg3(scale=0.5, nsrc=16, nrec_side=5)
    picks, tt = _run(ctx, w.vel, w.grd, w.coordsrc, w.coordrec, ExtraParams())
    for s in (0, 7, 15):
        op, ott = O.eiktraveltime(w.vel, w.grd, w.coordsrc[s:s + 1], w.coordrec[s:s + 1], returntt=True,
                                  extraparams=ExtraParams())
        assert int((tt[s] != ott[0]).sum()) == 0, s
        assert np.array_equal(picks[s], op[0])


@pytest.mark.parametrize("which", ["2d_cluster", "3d_global"])
def test_visit_counts_add_up(ctx, which):
    """Without the refined start-up every list entry of the coarse solve is visited once, with
    one outcome: the outcome counts sum to the list entries, and the three outcomes that
    follow an evaluation of the order rule sum to the evaluations."""
    w = CF.cfg2(scale=0.125, nsrc=3) if which == "2d_cluster" else CF.cfg3(scale=0.125, nsrc=3, nrec_side=3)
    _run(ctx, w.vel, w.grd, w.coordsrc, w.coordrec, ExtraParams(refinearoundsrc=False))
    st = ctx.last_stats
    vis = [int(v) for v in st.fwd_visits]
    assert st.node_evals > 0 and st.retries == 0
    assert sum(vis) == int(st.tile_activations), vis
    assert vis[4] + vis[5] + vis[6] == int(st.node_evals), vis
