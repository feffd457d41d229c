"""HMC problem callables (src/HMCtraveltimes.jl:26-283).

CPU: the callables' own logic (flattening orders, the split of the parameter vector, the
log-velocity transform and the reference's 1/v factor on the velocity gradient, the
assertions and the error on a wrong ``kind``) with the solver calls routed to the oracle.
GPU: the same callables on libeikcuda against the oracle-backed ones, misfit within 1e-9
and gradients within 1e-4 relative L2.
"""
import numpy as np
import pytest

import eikoracle as O
import refcases as RC
from eikonalsolvers import ExtraParams, Grid2DSphere
from eikonalsolvers import hmc as H

GRAD_RTOL = 1e-4
MISFIT_RTOL = 1e-9


def _case():
    c = RC.gradsrc_2D()[0]
    grd, rec = c["grd"], c["coordrec"]
    ep = ExtraParams(refinearoundsrc=False)
    picks = O.eiktraveltime(c["velmod"], grd, c["coordsrc1"], rec, extraparams=ep)
    sobs = [0.01 * np.ones(p.shape) for p in picks]
    return c, grd, rec, ep, picks, sobs


def _on_oracle(monkeypatch):
    monkeypatch.setattr(H, "eikgradient",
                        lambda *a, ctx=None, **k: O.eikgradient(*a, **k))
    monkeypatch.setattr(H, "eikttimemisfit",
                        lambda *a, ctx=None, **k: O.eikttimemisfit(*a, **k))


def _probs(c, grd, rec, ep, picks, sobs, logvel, ctx=None):
    pv = H.EikonalProbVel(grd=grd, dobs=picks, stdobs=sobs, coordsrc=c["coordsrc2"], coordrec=rec,
                          whichgrad="gradvel", logVel=logvel, extraparams=ep, ctx=ctx)
    ps = H.EikonalProbSrcLoc(grd=grd, dobs=picks, stdobs=sobs, coordrec=rec, velmod=c["vel0"],
                             whichgrad=":gradsrcloc", extraparams=ep, ctx=ctx)
    pb = H.EikonalProbVelAndSrcLoc(grd=grd, dobs=picks, stdobs=sobs, coordrec=rec,
                                   whichgrad="gradvelandsrcloc", logVel=logvel, extraparams=ep, ctx=ctx)
    return pv, ps, pb


def _x(c, logvel):
    v = np.ravel(c["vel0"], order="F")
    xv = np.log(v) if logvel else v
    xs = np.ravel(c["coordsrc2"], order="F")
    return xv, xs, np.concatenate([xv, xs])


@pytest.mark.parametrize("logvel", [False, True])
def test_callables_on_the_oracle(monkeypatch, logvel):
    _on_oracle(monkeypatch)
    c, grd, rec, ep, picks, sobs = _case()
    pv, ps, pb = _probs(c, grd, rec, ep, picks, sobs, logvel)
    xv, xs, xb = _x(c, logvel)
    # the velocity the callables solve on: exp(log v) is v only to rounding
    vel0 = np.reshape(np.exp(xv), grd.grsize, order="F") if logvel else c["vel0"]
    m_ref = O.eikttimemisfit(vel0, grd, c["coordsrc2"], rec, picks, sobs, extraparams=ep)
    assert abs(pv(xv, "nlogpdf") - m_ref) <= 1e-12 * m_ref
    m_src = O.eikttimemisfit(c["vel0"], grd, c["coordsrc2"], rec, picks, sobs, extraparams=ep)
    assert abs(ps(xs, ":nlogpdf") - m_src) <= 1e-12 * m_src
    assert abs(pb(xb, "nlogpdf") - m_ref) <= 1e-12 * m_ref
    gv, gs, _ = O.eikgradient(vel0, grd, c["coordsrc2"], rec, picks, sobs, "gradvelandsrcloc", extraparams=ep)
    gv_want = (1.0 / vel0) * gv if logvel else gv
    assert np.allclose(pv(xv, "gradnlogpdf"), np.ravel(gv_want, order="F"), rtol=1e-12, atol=0)
    _, gs0, _ = O.eikgradient(c["vel0"], grd, c["coordsrc2"], rec, picks, sobs, "gradvelandsrcloc", extraparams=ep)
    assert np.allclose(ps(xs, "gradnlogpdf"), np.ravel(gs0, order="F"), rtol=1e-12, atol=0)
    gb = pb(xb, "gradnlogpdf")
    assert gb.shape == xb.shape
    assert np.allclose(gb, np.concatenate([np.ravel(gv_want, order="F"), np.ravel(gs, order="F")]),
                       rtol=1e-12, atol=0)


def test_callables_refuse_what_the_reference_refuses(monkeypatch):
    _on_oracle(monkeypatch)
    c, grd, rec, ep, picks, sobs = _case()
    pv, ps, pb = _probs(c, grd, rec, ep, picks, sobs, False)
    xv, xs, xb = _x(c, False)
    with pytest.raises(RuntimeError, match="Wrong argument 'kind'"):
        pv(xv, "logpdf")
    with pytest.raises(RuntimeError, match="Wrong argument 'kind'"):
        ps(xs, "grad")
    bad = H.EikonalProbVel(grd=grd, dobs=picks, stdobs=sobs, coordsrc=c["coordsrc2"], coordrec=rec,
                           whichgrad="gradsrcloc")
    with pytest.raises(AssertionError):
        bad(xv, "nlogpdf")
    sph = Grid2DSphere(Δr=2.0, Δθ=0.25, cooinit=(5800.0, 10.0), grsize=(10, 10))
    with pytest.raises(TypeError):
        H.EikonalProbVel(grd=sph, dobs=picks, stdobs=sobs, coordsrc=c["coordsrc2"], coordrec=rec,
                         whichgrad="gradvel")


@pytest.mark.gpu
@pytest.mark.parametrize("logvel", [False, True])
def test_callables_on_the_gpu_match_the_oracle(monkeypatch, logvel):
    from eikonalsolvers import Context
    c, grd, rec, ep, picks, sobs = _case()
    xv, xs, xb = _x(c, logvel)
    ctx = Context(0)
    try:
        gpu = [p(x, k) for p, x in zip(_probs(c, grd, rec, ep, picks, sobs, logvel, ctx=ctx), (xv, xs, xb))
               for k in ("nlogpdf", "gradnlogpdf")]
    finally:
        ctx.close()
    _on_oracle(monkeypatch)
    ora = [p(x, k) for p, x in zip(_probs(c, grd, rec, ep, picks, sobs, logvel), (xv, xs, xb))
           for k in ("nlogpdf", "gradnlogpdf")]
    for g, o in zip(gpu, ora):
        if np.ndim(o) == 0:
            assert abs(g - o) <= MISFIT_RTOL * abs(o), (g, o)
        else:
            assert np.linalg.norm(g - o) <= GRAD_RTOL * np.linalg.norm(o)
