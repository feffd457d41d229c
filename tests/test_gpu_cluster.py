"""The forward solve of small problems in one thread-block cluster each (state in
distributed shared memory, rounds separated by the cluster barrier) against the persistent
global solve: picks, traveltime grids and gradients bit-identical with the context parameter
cluster_solve forced on (2: any dimension) and off, for the refined windows (always small) and for coarse grids that
fit a cluster, on 2D and 3D Cartesian and spherical grids. The oracle parity of the default
path, which now takes the cluster solve on these sizes, is in test_gpu_forward.py and
test_gpu_gradient.py. A round limit stops the cluster solve with EIK_ERR_NOT_CONVERGED and
leaves the context usable. By default (1) only 2D problems take the cluster."""
import numpy as np
import pytest

import eikoracle as O
from eikonalsolvers import Context, ExtraParams, _lib
from eikonalsolvers import configs as CF

pytestmark = pytest.mark.gpu

CASES = {
    "cfg1 300x220 x4": lambda: CF.cfg1(),
    "2D 128x80 x3": lambda: CF.cfg2(scale=0.125, nsrc=3),
    "3D 32^3 x3": lambda: CF.cfg3(scale=0.125, nsrc=3, nrec_side=4),
    "3D 44^3 x2": lambda: CF.cfg3(scale=44 / 256, nsrc=2, nrec_side=4),
    "sphere 30x27x27 x2": lambda: CF.cfg4(scale=0.15, nsrc=2),
    "3D 64^3 x2 (too large: windows only)": lambda: CF.cfg3(scale=0.25, nsrc=2, nrec_side=4),
}


@pytest.fixture(scope="module")
def ctx():
    c = Context(0)
    yield c
    c.close()


def _tt(ctx, w, ep, on):
    ctx.set_param("cluster_solve", 2.0 if on else 0.0)
    mid = ctx.upload(w.vel, w.grd)
    try:
        return ctx.traveltime(mid, w.grd, w.coordsrc, w.coordrec, returntt=True, extraparams=ep), ctx.last_stats.launches
    finally:
        ctx.release(mid)
        ctx.set_param("cluster_solve", 1.0)


@pytest.mark.parametrize("refine", [True, False], ids=["refined", "plain"])
@pytest.mark.parametrize("name", list(CASES))
def test_cluster_solve_equals_global_solve(ctx, name, refine):
    w = CASES[name]()
    ep = ExtraParams(refinearoundsrc=refine)
    (pk1, tt1), n1 = _tt(ctx, w, ep, True)
    (pk0, tt0), n0 = _tt(ctx, w, ep, False)
    for s in range(len(tt0)):
        assert int((tt1[s] != tt0[s]).sum()) == 0, (name, s)
        assert np.array_equal(pk1[s], pk0[s])
    if "too large" not in name or refine:
        assert n1 < n0  # the cluster path launched (fewer kernels: no separate init and seeding)


def test_cluster_solve_matches_the_oracle_on_config_1(ctx):
    w = CF.cfg1()
    (pk, tt), _ = _tt(ctx, w, w.extraparams, True)
    op, ott = O.eiktraveltime(w.vel, w.grd, w.coordsrc, w.coordrec, returntt=True, extraparams=w.extraparams)
    for s in range(len(tt)):
        assert int((tt[s] != ott[s]).sum()) == 0
        assert np.array_equal(pk[s], op[s])


@pytest.mark.parametrize("name,which", [("cfg1 300x220 x4", "gradvel"), ("3D 32^3 x3", "gradvelandsrcloc")])
def test_cluster_solve_gradients_equal_global_solve(ctx, name, which):
    w = CASES[name]()
    rng = np.random.default_rng(2)
    po = [np.full(r.shape[0], 1.0) + 0.1 * rng.standard_normal(r.shape[0]) for r in w.coordrec]
    so = [0.05 * np.ones(p.shape) for p in po]
    mid = ctx.upload(w.vel, w.grd)
    try:
        out = []
        for on in (2.0, 0.0):
            ctx.set_param("cluster_solve", on)
            out.append(ctx.gradient(mid, w.grd, w.coordsrc, w.coordrec, po, so, which))
    finally:
        ctx.set_param("cluster_solve", 1.0)
        ctx.release(mid)
    for a, b in zip(*out):
        if isinstance(a, float):
            assert a == b
        else:
            assert np.array_equal(a, b)


def test_cluster_solve_round_limit(ctx):
    w = CF.cfg1()
    mid = ctx.upload(w.vel, w.grd)
    try:
        ctx.set_param("max_rounds", 3)
        with pytest.raises(_lib.EikError) as ei:
            ctx.traveltime(mid, w.grd, w.coordsrc, w.coordrec)
        assert "EIK_ERR_NOT_CONVERGED" in str(ei.value)
        ctx.set_param("max_rounds", 0)
        pk = ctx.traveltime(mid, w.grd, w.coordsrc, w.coordrec)
        op = O.eiktraveltime(w.vel, w.grd, w.coordsrc, w.coordrec, extraparams=w.extraparams)
        assert all(np.array_equal(a, b) for a, b in zip(pk, op))
    finally:
        ctx.set_param("max_rounds", 0)
        ctx.release(mid)


def test_default_takes_clusters_in_2d_only(ctx):
    w2, w3 = CF.cfg1(), CF.cfg3(scale=0.125, nsrc=3, nrec_side=4)
    launches = {}
    for name, w in (("2d", w2), ("3d", w3)):
        for mode in (1.0, 0.0):
            ctx.set_param("cluster_solve", mode)
            mid = ctx.upload(w.vel, w.grd)
            try:
                ctx.traveltime(mid, w.grd, w.coordsrc, w.coordrec)
                launches[name, mode] = ctx.last_stats.launches
            finally:
                ctx.release(mid)
    ctx.set_param("cluster_solve", 1.0)
    assert launches["2d", 1.0] < launches["2d", 0.0]
    assert launches["3d", 1.0] == launches["3d", 0.0]
