"""A gradient call larger than the context's HBM budget runs as several pipelines over
consecutive chunks of its sources (recomputing their traveltimes rather than keeping all of
them at once): the result equals the one-pipeline result bit for bit. The chunks cut through
source groups (:sharedmem with several groups, and :serial), through a pair of co-located
sources whose shared source points carry the gradient from one source to the next
(eikmaingrad.jl:182-190, 242-246), and run with the smoothing around sources and the Gaussian
smoothing of the sum."""
import numpy as np
import pytest

from eikonalsolvers import Context, ExtraParams, _lib
from eikonalsolvers import configs as CF

pytestmark = pytest.mark.gpu


def _workload():
    w = CF.cfg3(scale=0.25, nsrc=7, nrec_side=6)
    cs = w.coordsrc.copy()
    cs[3] = cs[2]  # co-located pair on both sides of the first chunk boundary
    rng = np.random.default_rng(3)
    recs = w.coordrec
    pobs = [np.full(r.shape[0], 2.0) + 0.1 * rng.standard_normal(r.shape[0]) for r in recs]
    sobs = [0.05 * np.ones(r.shape[0]) for r in recs]
    return w, cs, recs, pobs, sobs


def _run(ctx, w, cs, recs, pobs, sobs, ep, nthreads):
    mid = ctx.upload(w.vel, w.grd)
    try:
        out = ctx.gradient(mid, w.grd, cs, recs, pobs, sobs, "gradvelandsrcloc", extraparams=ep, nthreads=nthreads)
        return out, ctx.last_stats.chunks
    finally:
        ctx.release(mid)


def _budget_for(w, cs, recs, ep, nthreads, per_chunk):
    """A budget that holds the model, the chunk state and `per_chunk` sources, but not the call."""
    c = Context(0)
    try:
        mid = c.upload(w.vel, w.grd)
        nrec = sum(r.shape[0] for r in recs)
        b1 = c.gradient_bytes(mid, 1, nrec, "gradvelandsrcloc", ep, nthreads)
        b2 = c.gradient_bytes(mid, 2, nrec, "gradvelandsrcloc", ep, nthreads)
        bn = c.gradient_bytes(mid, len(cs), nrec, "gradvelandsrcloc", ep, nthreads)
        c.release(mid)
    finally:
        c.close()
    per, fix = b2 - b1, 2 * b1 - b2
    N = int(np.prod(w.grd.grsize))
    budget = fix + 3 * 8 * N + 64 + per * per_chunk + per // 2
    assert budget < bn
    return budget + 2 * 8 * N  # the resident model (velocity and slowness)


@pytest.mark.parametrize("parallelkind,nthreads,smooth", [("sharedmem", 3, 0), ("serial", 1, 5)],
                         ids=["sharedmem3", "serial-smooth"])
def test_chunked_gradient_equals_one_pipeline(parallelkind, nthreads, smooth):
    w, cs, recs, pobs, sobs = _workload()
    ep = ExtraParams(parallelkind=parallelkind, smoothgradkern=smooth)
    full = Context(0)
    try:
        ref, nch = _run(full, w, cs, recs, pobs, sobs, ep, nthreads)
    finally:
        full.close()
    assert nch == 0
    small = Context(0, hbm_budget=_budget_for(w, cs, recs, ep, nthreads, per_chunk=3))
    try:
        got, nch = _run(small, w, cs, recs, pobs, sobs, ep, nthreads)
    finally:
        small.close()
    assert nch == 3  # chunks of 3, 3 and 1 sources
    assert np.array_equal(got[0], ref[0])
    assert np.array_equal(got[1], ref[1])
    assert got[2] == ref[2]


def test_a_budget_below_one_source_is_refused():
    w, cs, recs, pobs, sobs = _workload()
    N = int(np.prod(w.grd.grsize))
    ctx = Context(0, hbm_budget=2 * 8 * N + 4096)
    try:
        with pytest.raises(_lib.EikError) as ei:
            _run(ctx, w, cs, recs, pobs, sobs, ExtraParams(), 1)
        assert ei.value.code == -5  # EIK_ERR_OUT_OF_BUDGET
    finally:
        ctx.close()
