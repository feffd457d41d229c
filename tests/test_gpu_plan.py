"""GPU tests of captured gradient plans (eik_plan_gradient / eik_plan_run): the replayed
CUDA graph gives bit-identical results to eik_gradient on the same inputs, across replays
with new velocities (in place) and new observations; the plan pins its model and context."""
import numpy as np
import pytest

import refcases as RC
from eikonalsolvers import Context, ExtraParams
from eikonalsolvers import configs as CF

pytestmark = pytest.mark.gpu


def _same(a, b):
    if isinstance(a, tuple):
        return all(_same(x, y) for x, y in zip(a, b))
    if isinstance(a, float):
        return a == b
    return np.array_equal(a, b)


def _reference(vel, grd, cs, rec, po, so, which, ep):
    """eik_gradient on a fresh context and model: what every replay must reproduce."""
    c = Context(0)
    try:
        mid = c.upload(vel, grd)
        out = c.gradient(mid, grd, cs, rec, po, so, which, extraparams=ep)
        st = c.last_stats
        c.release(mid)
        return out, st
    finally:
        c.close()


def _obs(vel, grd, cs, rec, ep, seed):
    c = Context(0)
    try:
        mid = c.upload(vel, grd)
        picks = c.traveltime(mid, grd, cs, rec, extraparams=ep)
        c.release(mid)
    finally:
        c.close()
    rng = np.random.default_rng(seed)
    return [p + rng.normal(0.0, 0.01, p.shape) for p in picks], [0.01 * np.ones(p.shape) for p in picks]


def _cases():
    w2 = CF.cfg2(scale=0.125, nsrc=5)
    w3 = CF.cfg3(scale=0.125, nsrc=3, nrec_side=5)
    c = [c for c in RC.all_forward_cases() if c["name"] == "2Dconst3"][0]
    return [
        ("2D-refined", w2.vel, w2.grd, w2.coordsrc, w2.coordrec, ExtraParams(), "gradvelandsrcloc"),
        ("3D-refined-smoothed", w3.vel, w3.grd, w3.coordsrc, w3.coordrec, ExtraParams(smoothgradkern=3),
         "gradvelandsrcloc"),
        ("3D-plain", w3.vel, w3.grd, w3.coordsrc, w3.coordrec, ExtraParams(refinearoundsrc=False), "gradvel"),
        ("2D-constant-ties", c["vel"], c["grd"], c["coordsrc"], [c["coordrec"][0]] * len(c["coordsrc"]),
         c["extraparams"], "gradvel"),
    ]


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_plan_replays_match_eik_gradient(case):
    _, vel, grd, cs, rec, ep, which = case
    rng = np.random.default_rng(3)
    vel2 = vel * (1.0 + 0.02 * rng.uniform(-1.0, 1.0, vel.shape))
    po, so = _obs(vel * 1.03, grd, cs, rec, ep, 1)
    po2, so2 = _obs(vel * 0.98, grd, cs, rec, ep, 2)
    ctx = Context(0)
    mid = ctx.upload(vel, grd)
    plan = ctx.plan_gradient(mid, grd, cs, rec, which, extraparams=ep)
    try:
        runs = [(None, po, so, vel), (None, po2, so2, vel), (vel2, po, so, vel2), (None, po2, so2, vel2),
                (vel, po, so, vel)]
        for k, (v, p, s, vref) in enumerate(runs):
            got = plan.run(p, s, vel=v)
            want, st = _reference(vref, grd, cs, rec, p, s, which, ep)
            assert _same(got, want), (k, which)
            assert plan.last_stats.fine_replays == st.fine_replays
            assert plan.last_stats.err_mask == 0
        # the model kept the last velocity: an ordinary call on it sees it
        assert _same(ctx.gradient(mid, grd, cs, rec, po, so, which, extraparams=ep),
                     _reference(vel, grd, cs, rec, po, so, which, ep)[0])
    finally:
        plan.close()
        ctx.release(mid)
        ctx.close()


def test_plan_pins_model_and_context_and_checks_velocity():
    w = CF.cfg2(scale=0.125, nsrc=2)
    ctx = Context(0)
    mid = ctx.upload(w.vel, w.grd)
    po, so = _obs(w.vel, w.grd, w.coordsrc, w.coordrec, ExtraParams(), 4)
    plan = ctx.plan_gradient(mid, w.grd, w.coordsrc, w.coordrec, "gradvel")
    try:
        with pytest.raises(AssertionError, match="plan"):
            ctx.release(mid)
        assert ctx.L.eik_ctx_destroy(ctx.h) == -1  # EIK_ERR_ASSERT: the context stays alive
        assert b"plan" in ctx.L.eik_last_error(None)
        first = plan.run(po, so)
        bad = w.vel.copy()
        bad[3, 4] = 0.0
        with pytest.raises(AssertionError, match="vel"):
            plan.run(po, so, vel=bad)
        assert _same(plan.run(po, so), first)  # the refused velocity was not taken
    finally:
        plan.close()
    ctx.release(mid)
    ctx.close()


def test_plan_on_a_spherical_grid():
    """A plan on a Grid3DSphere model: replays with new velocities equal eik_gradient."""
    from eikonalsolvers import Grid3DSphere
    grd = Grid3DSphere(Δr=2.0, Δθ=0.25, Δφ=0.3, cooinit=(5800.0, 40.0, 10.0), grsize=(18, 20, 22))
    r = np.array(grd.r)[:, None, None]
    vel = np.ascontiguousarray(np.broadcast_to(5.0 + 0.01 * (6000.0 - r), grd.grsize))
    cs = np.array([[5800.0 + 8.3 * 2.0, 40.0 + 9.4 * 0.25, 10.0 + 10.6 * 0.3]])
    th, ph = np.linspace(40.3, 44.5, 3), np.linspace(10.4, 16.0, 3)
    rec = [np.array([[5800.0 + 17 * 2.0, a, b] for a in th for b in ph])]
    ep = ExtraParams()
    po, so = _obs(vel * 1.02, grd, cs, rec, ep, 5)
    vel2 = vel * (1.0 + 0.01 * np.random.default_rng(8).uniform(-1.0, 1.0, vel.shape))
    ctx = Context(0)
    mid = ctx.upload(vel, grd)
    plan = ctx.plan_gradient(mid, grd, cs, rec, "gradvel", extraparams=ep)
    try:
        for v, vref in ((None, vel), (vel2, vel2), (vel, vel)):
            assert _same(plan.run(po, so, vel=v), _reference(vref, grd, cs, rec, po, so, "gradvel", ep)[0])
    finally:
        plan.close()
        ctx.release(mid)
        ctx.close()
