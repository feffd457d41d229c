"""CPU tests of the serving loop's host logic (admission order, batching of traveltime
requests on one model, splitting of results, failure isolation), with a stand-in for the
device context that records the calls it receives."""
import threading
import time

import numpy as np
import pytest

from eikonalsolvers import Grid2DCart, Grid3DCart
from eikonalsolvers.serve import Request, Server


class FakeContext:
    """Answers traveltime with picks = source x-coordinate + receiver index, gradient with
    a field of the source count; records every call."""
    calls = []
    lock = threading.Lock()

    def __init__(self):
        self.params = {}
        self.next_id = 0

    def set_param(self, k, v):
        self.params[k] = v

    def upload(self, vel, grd):
        self.next_id += 1
        return self.next_id

    def release(self, mid):
        pass

    def close(self):
        pass

    def traveltime(self, mid, grd, cs, recs, extraparams=None):
        time.sleep(0.01)
        with self.lock:
            self.calls.append(("traveltime", len(cs)))
        return [cs[s][0] + np.arange(len(recs[s]), dtype=float) for s in range(len(cs))]

    def traveltime_multi(self, reqs, extraparams=None):
        time.sleep(0.01)
        with self.lock:
            self.calls.append(("traveltime_multi", tuple(len(cs) for (_, _, cs, _) in reqs)))
        return [[cs[s][0] + np.arange(len(recs[s]), dtype=float) for s in range(len(cs))]
                for (_, _, cs, recs) in reqs]

    def gradient(self, mid, grd, cs, recs, po, so, which, extraparams=None):
        time.sleep(0.01)
        if np.any(np.isnan(cs)):
            raise RuntimeError("bad source")
        with self.lock:
            self.calls.append(("gradient", len(cs)))
        return np.full(grd.grsize, float(len(cs))), 1.0

    def gradient_groups(self, mid, grd, groups, which, extraparams=None):
        time.sleep(0.01)
        if any(np.any(np.isnan(g[0])) for g in groups):
            raise RuntimeError("bad source")
        with self.lock:
            self.calls.append(("gradient_groups", tuple(len(g[0]) for g in groups)))
        return [(np.full(grd.grsize, float(len(g[0]))), 1.0) for g in groups]


@pytest.fixture
def grd():
    return Grid2DCart(hgrid=1.0, cooinit=(0.0, 0.0), grsize=(8, 8))


def _req(kind, xs, model="a"):
    cs = np.array([[x, 1.0] for x in xs])
    recs = [np.zeros((3, 2)) for _ in xs]
    return Request(model=model, kind=kind, coordsrc=cs, coordrec=recs,
                   pickobs=[np.zeros(3)] * len(xs), stdobs=[np.ones(3)] * len(xs))


def test_traveltime_requests_are_batched_across_models_and_split(grd):
    FakeContext.calls = []
    grd3 = Grid3DCart(hgrid=1.0, cooinit=(0.0, 0.0, 0.0), grsize=(4, 4, 4))
    srv = Server(slots=1, max_batch_sources=10, context_factory=FakeContext)
    srv.register_model("a", np.ones(grd.grsize), grd)
    srv.register_model("b", np.ones((6, 5)), Grid2DCart(hgrid=1.0, cooinit=(0.0, 0.0), grsize=(6, 5)))
    srv.register_model("c", np.ones(grd3.grsize), grd3)
    blocker = srv.submit(_req("gradient", [9.0]))  # keeps the only slot busy
    futs = [srv.submit(_req("traveltime", [1.0, 2.0])), srv.submit(_req("traveltime", [3.0], model="b")),
            srv.submit(_req("traveltime", [4.0, 5.0, 6.0])),
            srv.submit(Request(model="c", kind="traveltime", coordsrc=np.array([[7.0, 1.0, 1.0]]),
                               coordrec=[np.zeros((2, 3))]))]
    blocker.result(timeout=10)
    res = [f.result(timeout=10) for f in futs]
    srv.close()
    assert [float(p[0]) for p in res[0]] == [1.0, 2.0]
    assert [float(p[0]) for p in res[2]] == [4.0, 5.0, 6.0]
    assert [float(p[0]) for p in res[1]] == [3.0]
    assert [float(p[0]) for p in res[3]] == [7.0]
    # the 2D requests ran as one call: model "a" (5 sources) beside model "b"; 3D alone
    assert ("traveltime_multi", (5, 1)) in FakeContext.calls and ("traveltime", 1) in FakeContext.calls
    st = srv.stats()
    assert st["requests"] == 5 and st["p99_ms"] >= st["p50_ms"] > 0


def test_gradient_requests_on_one_model_share_a_call_and_failures_stay_local(grd):
    FakeContext.calls = []
    srv = Server(slots=1, context_factory=FakeContext)
    srv.register_model("a", np.ones(grd.grsize), grd)
    srv.register_model("b", np.ones(grd.grsize), grd)
    blocker = srv.submit(_req("traveltime", [9.0]))  # keeps the only slot busy
    good = [srv.submit(_req("gradient", [1.0, 2.0])) for _ in range(3)]
    other = srv.submit(_req("gradient", [1.0], model="b"))
    bad = srv.submit(_req("gradient", [np.nan]))
    blocker.result(timeout=10)
    for f in good:
        g, m = f.result(timeout=10)
        assert g[0, 0] == 2.0
    assert other.result(timeout=10)[0][0, 0] == 1.0
    with pytest.raises(RuntimeError, match="bad source"):
        bad.result(timeout=10)
    srv.close()
    # one merged call failed on the bad request; each request then ran alone
    assert FakeContext.calls.count(("gradient", 2)) == 3
    assert ("gradient", 1) in FakeContext.calls  # model "b" is never merged with "a"


def test_gradient_groups_merge_without_failures(grd):
    FakeContext.calls = []
    srv = Server(slots=1, context_factory=FakeContext)
    srv.register_model("a", np.ones(grd.grsize), grd)
    blocker = srv.submit(_req("traveltime", [9.0]))
    futs = [srv.submit(_req("gradient", [1.0] * (k + 1))) for k in range(3)]
    blocker.result(timeout=10)
    assert [f.result(timeout=10)[0][0, 0] for f in futs] == [1.0, 2.0, 3.0]
    srv.close()
    assert ("gradient_groups", (1, 2, 3)) in FakeContext.calls


def test_slots_get_an_sm_share_and_unknown_models_are_refused(grd):
    srv = Server(slots=4, context_factory=FakeContext)
    assert all(c.params["sm_fraction"] == 0.25 for c in srv._ctx)
    with pytest.raises(KeyError):
        srv.submit(_req("traveltime", [1.0], model="zzz"))
    srv.close()


def test_admission_by_device_memory(grd):
    """With a server-wide HBM budget that holds one gradient batch but not two, gradients run
    one at a time while the slots still take them; a request larger than the whole budget fails
    alone; everything else completes."""
    from eikonalsolvers.serve import request_bytes
    one = request_bytes(grd, 1, "gradient")
    srv = Server(slots=3, context_factory=FakeContext, hbm_budget=int(1.5 * one))
    try:
        srv.register_model("a", np.ones(grd.grsize), grd)
        futs = [srv.submit(_req("gradient", [1.0 + i])) for i in range(6)]
        big = srv.submit(_req("gradient", [1.0, 2.0]))  # two sources: about twice the budget / 1.5
        for f in futs:
            g, m = f.result(timeout=10)
            assert g.shape == grd.grsize
        with pytest.raises(MemoryError):
            big.result(timeout=10)
        assert 0 < srv.max_inflight_seen <= srv.hbm_budget
        assert srv.max_inflight_seen < 2 * one  # never two gradients in flight at once
    finally:
        srv.close()


def test_request_bytes_scales_with_work(grd):
    from eikonalsolvers import ExtraParams
    from eikonalsolvers.serve import request_bytes
    t1 = request_bytes(grd, 1, "traveltime")
    assert request_bytes(grd, 4, "traveltime") == 4 * t1
    assert request_bytes(grd, 1, "gradient") > t1
    assert request_bytes(grd, 1, "traveltime", ExtraParams(refinearoundsrc=False)) < t1


def test_traveltime_batches_are_capped_by_the_memory_budget(grd):
    """Several 1-source traveltime requests on one model whose sum exceeds the server's budget
    while each fits alone: they are merged only as far as the budget allows, so none fails."""
    from eikonalsolvers.serve import request_bytes
    FakeContext.calls = []
    one = request_bytes(grd, 1, "traveltime")
    srv = Server(slots=1, max_batch_sources=64, context_factory=FakeContext, hbm_budget=int(2.5 * one))
    try:
        srv.register_model("a", np.ones(grd.grsize), grd)
        assert request_bytes(grd, 1, "gradient") <= srv.hbm_budget
        blocker = srv.submit(_req("gradient", [9.0]))  # keeps the only slot busy meanwhile
        futs = [srv.submit(_req("traveltime", [1.0 + i])) for i in range(5)]
        blocker.result(timeout=10)
        res = [f.result(timeout=10) for f in futs]
        assert [float(p[0][0]) for p in res] == [1.0 + i for i in range(5)]
        sizes = [n for (k, n) in FakeContext.calls if k == "traveltime"]
        assert sum(sizes) == 5 and max(sizes) <= 2
        assert srv.max_inflight_seen <= srv.hbm_budget
    finally:
        srv.close()


def test_a_full_queue_refuses_arrivals(grd):
    from eikonalsolvers.serve import ServerOverloaded
    FakeContext.calls = []
    srv = Server(slots=1, context_factory=FakeContext, max_queue=2)
    srv.register_model("a", np.ones(grd.grsize), grd)
    blocker = srv.submit(_req("gradient", [9.0]))
    t0 = time.perf_counter()
    while srv._queue and time.perf_counter() - t0 < 5.0:  # until the slot has taken it
        time.sleep(0.0005)
    queued = [srv.submit(_req("traveltime", [1.0])), srv.submit(_req("traveltime", [2.0]))]
    refused = srv.submit(_req("traveltime", [3.0]))
    with pytest.raises(ServerOverloaded):
        refused.result(timeout=10)
    blocker.result(timeout=10)
    assert [float(f.result(timeout=10)[0][0]) for f in queued] == [1.0, 2.0]
    st = srv.stats()
    srv.close()
    assert st["refused"] == 1 and st["requests"] == 3


def test_cancelled_requests_never_run(grd):
    FakeContext.calls = []
    srv = Server(slots=1, context_factory=FakeContext)
    srv.register_model("a", np.ones(grd.grsize), grd)
    blocker = srv.submit(_req("gradient", [9.0]))
    t0 = time.perf_counter()
    while srv._queue and time.perf_counter() - t0 < 5.0:  # until the slot has taken it
        time.sleep(0.0005)
    keep = srv.submit(_req("traveltime", [1.0]))
    drop = [srv.submit(_req("traveltime", [2.0])), srv.submit(_req("gradient", [3.0]))]
    assert all(f.cancel() for f in drop)
    blocker.result(timeout=10)
    assert float(keep.result(timeout=10)[0][0]) == 1.0
    st = srv.stats()
    srv.close()
    assert st["cancelled"] == 2 and st["requests"] == 2
    assert ("gradient", 1) in FakeContext.calls and ("traveltime", 1) in FakeContext.calls
    assert len(FakeContext.calls) == 2  # the blocker and the kept request only
