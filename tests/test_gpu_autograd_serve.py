"""GPU tests of the differentiable misfit (torch autograd over eik_gradient_device) and of
the serving loop (every result identical alone and in a concurrent, batched mix)."""
import numpy as np
import pytest

import refcases as RC
from eikonalsolvers import Context, ExtraParams
from eikonalsolvers import configs as CF

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _case():
    c = RC.gradsrc_2D()[1]  # refined start-up, smoothing off
    grd, rec, ep = c["grd"], c["coordrec"], c["extraparams"]
    ctx = Context(0)
    mid = ctx.upload(c["velmod"], grd)
    pobs = ctx.traveltime(mid, grd, c["coordsrc1"], rec, extraparams=ep)
    ctx.release(mid)
    sobs = [0.0001 * np.ones(p.shape) for p in pobs]
    return c, grd, rec, ep, pobs, sobs, ctx


def test_autograd_matches_eikgradient_and_modes_agree():
    from eikonalsolvers.autograd import eik_misfit
    c, grd, rec, ep, pobs, sobs, ctx = _case()
    mid = ctx.upload(c["vel0"], grd)
    gv, gs, m = ctx.gradient(mid, grd, c["coordsrc2"], rec, pobs, sobs, "gradvelandsrcloc", extraparams=ep)
    ctx.release(mid)
    out = {}
    for mode in ("store", "recompute"):
        vel = torch.tensor(c["vel0"], dtype=torch.float64, device="cuda", requires_grad=True)
        cs = torch.tensor(c["coordsrc2"], dtype=torch.float64, requires_grad=True)
        mis = eik_misfit(vel, cs, grd, rec, pobs, sobs, extraparams=ep, ctx=ctx, mode=mode)
        (2.0 * mis).backward()
        out[mode] = (float(mis), vel.grad.cpu().numpy(), cs.grad.numpy())
    for mode, (mm, g, s) in out.items():
        assert abs(mm - m) <= 1e-9 * abs(m), (mode, mm, m)
        assert np.array_equal(g, 2.0 * gv), mode
        assert np.array_equal(s, 2.0 * gs), mode
    ctx.close()


def test_autograd_velocity_gradient_against_central_differences():
    """A few cells of d(misfit)/d(vel) against central differences of the forward-only
    misfit, at the reference testset's step and error bound (test_cartesian_2D.jl:168-254)."""
    from eikonalsolvers.autograd import eik_misfit
    c = RC.gradvel_2D()[1]
    grd, rec, ep = c["grd"], c["coordrec"], c["extraparams"]
    ctx = Context(0)
    mid = ctx.upload(c["velmod"], grd)
    pobs = ctx.traveltime(mid, grd, c["coordsrc1"], rec, extraparams=ep)
    ctx.release(mid)
    sobs = [0.0001 * np.ones(p.shape) for p in pobs]
    vel = torch.tensor(c["vel0"], dtype=torch.float64, device="cuda", requires_grad=True)
    cs = torch.tensor(c["coordsrc2"], dtype=torch.float64)
    eik_misfit(vel, cs, grd, rec, pobs, sobs, extraparams=ep, ctx=ctx).backward()
    g = vel.grad.cpu().numpy()
    dh = c["dh"]
    for (i, j) in [(25, 3), (10, 4), (40, 5), (25, 15), (5, 20)]:
        mp, mm = [], []
        for sgn, acc in ((1.0, mp), (-1.0, mm)):
            v = torch.tensor(c["vel0"], dtype=torch.float64, device="cuda")
            v[i, j] += sgn * dh
            acc.append(float(eik_misfit(v, cs, grd, rec, pobs, sobs, extraparams=ep, ctx=ctx, mode="recompute")))
        fd = (mp[0] - mm[0]) / (2 * dh)
        assert abs(fd - g[i, j]) <= 1.015 * c["tolerr"], (i, j, fd, g[i, j])
    ctx.close()


def test_serving_results_alone_equal_results_in_the_mix():
    from eikonalsolvers.serve import Request, Server
    models, reqs = CF.serving_requests(n=14, rate=1000.0, seed=9, scale=0.1, nmodels=4, max_sources=5)

    def make(r):
        return Request(model=r["model"], kind=r["kind"], coordsrc=r["coordsrc"], coordrec=r["coordrec"],
                       pickobs=r.get("pickobs"), stdobs=r.get("stdobs"))

    alone = []
    with Server(slots=1) as srv:
        for k, (vel, grd, _) in models.items():
            srv.register_model(k, vel, grd)
        for r in reqs:
            alone.append(srv.submit(make(r)).result(timeout=300))
    with Server(slots=3) as srv:
        for k, (vel, grd, _) in models.items():
            srv.register_model(k, vel, grd)
        futs = [srv.submit(make(r)) for r in reqs]
        mixed = [f.result(timeout=300) for f in futs]
        st = srv.stats()
    assert st["requests"] == len(reqs) and st["p99_ms"] >= st["p50_ms"]
    for r, a, b in zip(reqs, alone, mixed):
        if r["kind"] == "traveltime":
            assert len(a) == len(b) and all(np.array_equal(x, y) for x, y in zip(a, b))
        else:
            assert np.array_equal(a[0], b[0]) and a[1] == b[1]
