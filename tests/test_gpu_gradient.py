"""GPU gradient parity: eik_gradient (through the C ABI) against the oracle on the same
inputs. Contract: velocity and source-location gradients within 1e-4 relative L2 of the
reference's FP64 result, misfit within 1e-9 relative. The forward traveltimes are
bit-identical to the oracle's, so the remaining differences are the summation orders of
the adjoint solve (observed ~1e-13)."""
import numpy as np
import pytest

import eikoracle as O
import refcases as RC
from eikonalsolvers import Context, ExtraParams, GridRefinementPars
from eikonalsolvers import Grid2DSphere, Grid3DSphere
from eikonalsolvers import configs as CF

pytestmark = pytest.mark.gpu
GRAD_RTOL = 1e-4
MISFIT_RTOL = 1e-9


@pytest.fixture(scope="module")
def ctx():
    c = Context(0)
    yield c
    c.close()


def _gpu_grad(ctx, vel, grd, cs, rec, pobs, sobs, which, ep, nthreads=1):
    mid = ctx.upload(vel, grd)
    try:
        return ctx.gradient(mid, grd, cs, rec, pobs, sobs, which, extraparams=ep, nthreads=nthreads)
    finally:
        ctx.release(mid)


def _rel_l2(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def _check(res_gpu, res_ora, which):
    if which == "gradvelandsrcloc":
        gv, gs, m = res_gpu
        ov, os_, om = res_ora
        assert _rel_l2(gv, ov) <= GRAD_RTOL, _rel_l2(gv, ov)
        assert _rel_l2(gs, os_) <= GRAD_RTOL, _rel_l2(gs, os_)
    else:
        g, m = res_gpu
        o, om = res_ora
        assert g.shape == o.shape
        assert _rel_l2(g, o) <= GRAD_RTOL, _rel_l2(g, o)
    assert abs(m - om) <= MISFIT_RTOL * abs(om), (m, om)


def _obs(vel, grd, cs, rec, ep, sigma=0.0001):
    picks = O.eiktraveltime(vel, grd, cs, rec, extraparams=ep)
    return picks, [sigma * np.ones(p.shape) for p in picks]


@pytest.mark.parametrize("case", RC.gradvel_2D() + RC.gradvel_3D() + RC.gradsrc_2D() + RC.gradsrc_3D(),
                         ids=lambda c: c["name"])
@pytest.mark.parametrize("which", ["gradvel", "gradsrcloc", "gradvelandsrcloc"])
def test_reference_gradient_cases(ctx, case, which):
    grd, rec, ep = case["grd"], case["coordrec"], case["extraparams"]
    pobs, sobs = _obs(case["velmod"], grd, case["coordsrc1"], rec, ep)
    g = _gpu_grad(ctx, case["vel0"], grd, case["coordsrc2"], rec, pobs, sobs, which, ep)
    o = O.eikgradient(case["vel0"], grd, case["coordsrc2"], rec, pobs, sobs, which, extraparams=ep)
    _check(g, o, which)


@pytest.mark.parametrize("refine", [True, False])
@pytest.mark.parametrize("radius", [0, 3])
def test_cfg2_small_multisource(ctx, refine, radius):
    """Several sources in one call: carry-over onto source points and the smoothing
    around each source, summed in source order."""
    w = CF.cfg2(scale=0.25, nsrc=5, forward=lambda v, g, c, r, e: O.eiktraveltime(v, g, c, r, extraparams=e))
    ep = ExtraParams(refinearoundsrc=refine, radiussmoothgradsrc=radius)
    g = _gpu_grad(ctx, w.vel, w.grd, w.coordsrc, w.coordrec, w.pickobs, w.stdobs, "gradvelandsrcloc", ep)
    o = O.eikgradient(w.vel, w.grd, w.coordsrc, w.coordrec, w.pickobs, w.stdobs, "gradvelandsrcloc", extraparams=ep)
    _check(g, o, "gradvelandsrcloc")


@pytest.mark.parametrize("refine", [True, False])
def test_cfg3_small(ctx, refine):
    w = CF.cfg3(scale=0.125, nsrc=3, nrec_side=5,
                forward=lambda v, g, c, r, e: O.eiktraveltime(v, g, c, r, extraparams=e))
    ep = ExtraParams(refinearoundsrc=refine)
    g = _gpu_grad(ctx, w.vel, w.grd, w.coordsrc, w.coordrec, w.pickobs, w.stdobs, "gradvelandsrcloc", ep)
    o = O.eikgradient(w.vel, w.grd, w.coordsrc, w.coordrec, w.pickobs, w.stdobs, "gradvelandsrcloc", extraparams=ep)
    _check(g, o, "gradvelandsrcloc")


def _stacked_sources(nsrc=7):
    """Sources stacked upwards under the receivers: each one sits in the ray fan of the one
    before, so the value carried onto its source points is not zero."""
    w = CF.cfg2(scale=0.125, nsrc=2)
    h = w.grd.hgrid
    x0 = w.coordsrc[0][0]
    cs = np.array([[x0 + 0.37 * h * k, (60 - 6.3 * k) * h + 0.011] for k in range(nsrc)])
    return w, cs, [w.coordrec[0]] * nsrc


@pytest.mark.parametrize("refine", [True, False])
@pytest.mark.parametrize("nthreads", [1, 3])
def test_sharedmem_groups(ctx, refine, nthreads):
    """:sharedmem with 3 threads: 7 sources in groups of 3, 2, 2, each group with its own
    gradient buffer (changes the result by ~1e-2 relative for these sources)."""
    w, cs, rec = _stacked_sources()
    ep = ExtraParams(parallelkind="sharedmem", radiussmoothgradsrc=0, refinearoundsrc=refine)
    pobs, sobs = _obs(w.vel * 1.02, w.grd, cs, rec, ep, sigma=0.01)
    g = _gpu_grad(ctx, w.vel, w.grd, cs, rec, pobs, sobs, "gradvel", ep, nthreads=nthreads)
    o = O.eikgradient(w.vel, w.grd, cs, rec, pobs, sobs, "gradvel", extraparams=ep, nthreads=nthreads)
    _check(g, o, "gradvel")


@pytest.mark.parametrize("refine", [True, False])
def test_colocated_sources(ctx, refine):
    """Three sources at one position: the value carried onto the shared source points is a
    recurrence over all of them."""
    w = CF.cfg2(scale=0.125, nsrc=2)
    cs = np.vstack([w.coordsrc[0], w.coordsrc[0], w.coordsrc[1], w.coordsrc[0]])
    rec = [w.coordrec[0]] * 4
    ep = ExtraParams(refinearoundsrc=refine)
    pobs, sobs = _obs(w.vel * 1.02, w.grd, cs, rec, ep, sigma=0.01)
    g = _gpu_grad(ctx, w.vel, w.grd, cs, rec, pobs, sobs, "gradvel", ep)
    o = O.eikgradient(w.vel, w.grd, cs, rec, pobs, sobs, "gradvel", extraparams=ep)
    _check(g, o, "gradvel")


def _sphere2d():
    grd = Grid2DSphere(Δr=2.0, Δθ=0.25, cooinit=(5800.0, 10.0), grsize=(40, 50))
    r = np.array(grd.r)[:, None]
    vel = np.ascontiguousarray(np.broadcast_to(5.0 + 0.01 * (6000.0 - r), grd.grsize))
    cs = np.array([[5800.0 + 17.3 * 2.0, 10.0 + 21.4 * 0.25]])
    rec = [np.column_stack([np.full(9, 5800.0 + 39 * 2.0), np.linspace(10.5, 21.5, 9)])]
    return grd, vel, cs, rec


def _sphere3d():
    grd = Grid3DSphere(Δr=2.0, Δθ=0.25, Δφ=0.3, cooinit=(5800.0, 40.0, 10.0), grsize=(18, 20, 22))
    r = np.array(grd.r)[:, None, None]
    vel = np.ascontiguousarray(np.broadcast_to(5.0 + 0.01 * (6000.0 - r), grd.grsize))
    cs = np.array([[5800.0 + 8.3 * 2.0, 40.0 + 9.4 * 0.25, 10.0 + 10.6 * 0.3]])
    th = np.linspace(40.3, 44.5, 4)
    ph = np.linspace(10.4, 16.0, 4)
    rec = [np.array([[5800.0 + 17 * 2.0, a, b] for a in th for b in ph])]
    return grd, vel, cs, rec


@pytest.mark.parametrize("maker", [_sphere2d, _sphere3d], ids=["sphere2D", "sphere3D"])
@pytest.mark.parametrize("refine", [True, False])
def test_spherical_gradvel(ctx, maker, refine):
    grd, vel, cs, rec = maker()
    ep = ExtraParams(refinearoundsrc=refine)
    pobs, sobs = _obs(vel * 1.03, grd, cs, rec, ep, sigma=0.01)
    g = _gpu_grad(ctx, vel, grd, cs, rec, pobs, sobs, "gradvel", ep)
    o = O.eikgradient(vel, grd, cs, rec, pobs, sobs, "gradvel", extraparams=ep)
    _check(g, o, "gradvel")


def test_spherical_gradsrcloc_errors(ctx):
    grd, vel, cs, rec = _sphere2d()
    pobs, sobs = _obs(vel, grd, cs, rec, ExtraParams())
    with pytest.raises(Exception, match="hgrid"):
        _gpu_grad(ctx, vel, grd, cs, rec, pobs, sobs, "gradsrcloc", ExtraParams())


def test_gradsrcloc_fd_on_gpu(ctx):
    """Source-location gradient against central differences of the GPU's own misfit
    (the reference's gradsrcloc 2D testset, refined)."""
    case = RC.gradsrc_2D()[1]
    grd, rec, ep = case["grd"], case["coordrec"], case["extraparams"]
    pobs, sobs = _obs(case["velmod"], grd, case["coordsrc1"], rec, ep)
    gs, _ = _gpu_grad(ctx, case["vel0"], grd, case["coordsrc2"], rec, pobs, sobs, "gradsrcloc", ep)
    mid = ctx.upload(case["vel0"], grd)
    try:
        def picks_src(c):
            return ctx.traveltime(mid, grd, c, rec, extraparams=ep)
        fd = RC.fd_gradsrc(picks_src, case["coordsrc2"], case["dh"], pobs, sobs)
    finally:
        ctx.release(mid)
    d = np.abs(gs - fd)
    assert d.max() <= 1.015 * case["tolerr"] and np.linalg.norm(d) <= 1.015 * case["tolnorm"], (gs, fd)


@pytest.mark.parametrize("kind,l", [("2D", 5), ("3D", 3), ("3D", 23)])
def test_smoothgradkern(ctx, kind, l):
    """ExtraParams.smoothgradkern = l: the summed gradient is smoothed on the device. The
    smoothed GPU gradient is bit-identical to the oracle's smoothgradient applied to the
    GPU's unsmoothed gradient (same weights, same summation order; 3D with l = 23 takes the
    unstaged kernel), and within the gradient tolerance of the oracle's eikgradient."""
    if kind == "2D":
        w = CF.cfg2(scale=0.125, nsrc=3, forward=lambda v, g, c, r, e: O.eiktraveltime(v, g, c, r, extraparams=e))
    else:
        w = CF.cfg3(scale=0.125, nsrc=2, nrec_side=5,
                    forward=lambda v, g, c, r, e: O.eiktraveltime(v, g, c, r, extraparams=e))
    ep = ExtraParams(smoothgradkern=l)
    g, m = _gpu_grad(ctx, w.vel, w.grd, w.coordsrc, w.coordrec, w.pickobs, w.stdobs, "gradvel", ep)
    g0, m0 = _gpu_grad(ctx, w.vel, w.grd, w.coordsrc, w.coordrec, w.pickobs, w.stdobs, "gradvel", ExtraParams())
    assert m == m0
    assert np.array_equal(g, O.smoothgradient(l, w.grd, g0))
    o = O.eikgradient(w.vel, w.grd, w.coordsrc, w.coordrec, w.pickobs, w.stdobs, "gradvel", extraparams=ep)
    _check((g, m), o, "gradvel")


@pytest.mark.parametrize("maker", [_sphere2d, _sphere3d], ids=["sphere2D", "sphere3D"])
def test_spherical_smoothgradkern(ctx, maker):
    """Gaussian smoothing of the summed gradient on spherical grids (index-space smoothing,
    as the reference's smoothgradient): bit-identical to the oracle's smoothing of the GPU's
    unsmoothed gradient and within the gradient tolerance of the oracle's eikgradient."""
    grd, vel, cs, rec = maker()
    pobs, sobs = _obs(vel * 1.03, grd, cs, rec, ExtraParams(), sigma=0.01)
    ep = ExtraParams(smoothgradkern=3)
    g, m = _gpu_grad(ctx, vel, grd, cs, rec, pobs, sobs, "gradvel", ep)
    g0, _ = _gpu_grad(ctx, vel, grd, cs, rec, pobs, sobs, "gradvel", ExtraParams())
    assert np.array_equal(g, O.smoothgradient(3, grd, g0))
    o = O.eikgradient(vel, grd, cs, rec, pobs, sobs, "gradvel", extraparams=ep)
    _check((g, m), o, "gradvel")
