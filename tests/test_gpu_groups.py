"""Several gradient evaluations on one model in one pipeline with per-group outputs
(eik_gradient_groups, the serving loop's merged gradient call): every group's gradient
field, source-location gradient and misfit equal, bit for bit, eik_gradient of that group's
sources alone with one source group. Groups carry over between co-located sources only
within themselves (eikmaingrad.jl:182-190): a co-located pair split across two groups and
one kept inside a group are both covered, with the smoothing around sources, the Gaussian
smoothing of the field, 2D and 3D Cartesian grids and a spherical grid."""
import numpy as np
import pytest

from eikonalsolvers import Context, ExtraParams
from eikonalsolvers import configs as CF

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    c = Context(0)
    yield c
    c.close()


def _groups(w, sizes, seed):
    rng = np.random.default_rng(seed)
    cs, recs = w.coordsrc, w.coordrec
    out, s = [], 0
    for n in sizes:
        po = [np.full(recs[s + k].shape[0], 1.0) + 0.1 * rng.standard_normal(recs[s + k].shape[0]) for k in range(n)]
        so = [0.05 * np.ones(p.shape) for p in po]
        out.append((cs[s:s + n].copy(), [recs[s + k] for k in range(n)], po, so))
        s += n
    return out


def _check(ctx, w, groups, which, ep):
    mid = ctx.upload(w.vel, w.grd)
    try:
        merged = ctx.gradient_groups(mid, w.grd, groups, which, extraparams=ep)
        for g, (cs, rec, po, so) in enumerate(groups):
            alone = ctx.gradient(mid, w.grd, cs, rec, po, so, which, extraparams=ep)
            for a, b in zip(merged[g], alone):
                if isinstance(a, float):
                    assert a == b, (g, a, b)
                else:
                    assert np.array_equal(a, b), (g, float(np.abs(a - b).max()))
    finally:
        ctx.release(mid)


@pytest.mark.parametrize("smooth", [0, 5], ids=["plain", "smoothgradkern5"])
def test_groups_3d_equal_calls_alone(ctx, smooth):
    w = CF.cfg3(scale=0.25, nsrc=6, nrec_side=5)
    w.coordsrc[2] = w.coordsrc[1]  # co-located pair inside the first group
    w.coordsrc[3] = w.coordsrc[2]  # and across the boundary to the second
    groups = _groups(w, [3, 1, 2], 4)
    _check(ctx, w, groups, "gradvelandsrcloc", ExtraParams(smoothgradkern=smooth))


def test_groups_2d_equal_calls_alone(ctx):
    w = CF.cfg2(scale=0.25, nsrc=7)
    _check(ctx, w, _groups(w, [2, 4, 1], 5), "gradvelandsrcloc", ExtraParams())


@pytest.mark.parametrize("refine", [True, False], ids=["refined", "plain"])
def test_groups_sphere_equal_calls_alone(ctx, refine):
    w = CF.cfg4(scale=0.15, nsrc=4)
    _check(ctx, w, _groups(w, [1, 3], 6), "gradvel", ExtraParams(refinearoundsrc=refine))


def test_groups_reject_an_empty_group(ctx):
    w = CF.cfg2(scale=0.125, nsrc=2)
    mid = ctx.upload(w.vel, w.grd)
    try:
        groups = _groups(w, [1, 1], 7)
        groups.insert(1, (np.zeros((0, 2)), [], [], []))
        with pytest.raises(AssertionError, match="at least one source"):
            ctx.gradient_groups(mid, w.grd, groups, "gradvel")
    finally:
        ctx.release(mid)
