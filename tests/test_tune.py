"""Autotuner of the forward launch parameters (eikonalsolvers/tune.py).

CPU: with a stand-in context whose timings depend on the parameters, the tuner picks the
fastest pair, applies it, reuses the table entry for a workload of the same class, keeps the
table in a JSON file, and raises when a candidate returns different picks. GPU: on a real
context every candidate returns the same picks (the tuner checks it) and the tuned context
gives the picks of an untuned one.
"""
import json

import numpy as np
import pytest

from eikonalsolvers import ExtraParams, Grid2DCart, Grid3DCart
from eikonalsolvers import configs as CF
from eikonalsolvers.tune import Tuner, workload_key


class _Stats:
    device_ms = 0.0


class FakeContext:
    def __init__(self, cost, picks_for=None):
        self.params = {}
        self.cost = cost
        self.picks_for = picks_for or (lambda p: [np.arange(3.0)])
        self.calls = 0
        self.last_stats = _Stats()

    def set_param(self, name, value):
        self.params[name] = value

    def traveltime(self, model, grd, coordsrc, coordrec, extraparams=None):
        self.calls += 1
        self.last_stats = _Stats()
        self.last_stats.device_ms = self.cost(self.params["round_gate"], self.params["ctas_per_sm"])
        return self.picks_for(self.params)


GRD = Grid2DCart(hgrid=0.5, cooinit=(0.0, 0.0), grsize=(100, 60))
CS = np.array([[10.0, 10.0], [20.0, 12.0]])
REC = [np.array([[1.0, 1.0]])] * 2


def test_tuner_picks_the_fastest_and_reuses_it(tmp_path):
    path = str(tmp_path / "tune.json")
    t = Tuner(path=path, candidates={"round_gate": (1.0, 2.0, 3.0), "ctas_per_sm": (2, 3, 4)}, repeats=2,
              shipped=None)
    ctx = FakeContext(lambda g, c: 1.0 + abs(g - 2.0) + 0.5 * abs(c - 3))
    e = t.tune(ctx, 0, GRD, CS, REC)
    assert (e["round_gate"], e["ctas_per_sm"]) == (2.0, 3)
    assert ctx.params == {"round_gate": 2.0, "ctas_per_sm": 3.0}
    assert ctx.calls == 9 * 2 and len(e["timings"]) == 9
    # same class (node count and sources rounded up to powers of two): no timing
    grd2 = Grid2DCart(hgrid=0.5, cooinit=(0.0, 0.0), grsize=(101, 61))
    assert workload_key(grd2, 2) == workload_key(GRD, 2)
    ctx2 = FakeContext(lambda g, c: 1.0)
    assert t.tune(ctx2, 0, grd2, CS, REC) == e and ctx2.calls == 0
    assert ctx2.params == {"round_gate": 2.0, "ctas_per_sm": 3.0}
    # another class is timed again; the file keeps both
    assert workload_key(GRD, 5) != workload_key(GRD, 2)
    assert workload_key(GRD, 2, ExtraParams(refinearoundsrc=False)) != workload_key(GRD, 2)
    assert workload_key(Grid3DCart(hgrid=1.0, cooinit=(0, 0, 0), grsize=(8, 8, 8)), 2) != workload_key(GRD, 2)
    t.tune(FakeContext(lambda g, c: c), 0, GRD, np.zeros((5, 2)), REC * 3)
    table = json.load(open(path))
    assert len(table) == 2
    assert Tuner(path=path, shipped=None).lookup(GRD, 5)["ctas_per_sm"] == 2


def test_tuner_refuses_schedule_dependent_results():
    t = Tuner(path="", candidates={"round_gate": (1.0, 2.0), "ctas_per_sm": (4,)}, repeats=1, shipped=None)
    ctx = FakeContext(lambda g, c: 1.0, picks_for=lambda p: [np.arange(3.0) * p["round_gate"]])
    with pytest.raises(RuntimeError, match="schedule independent"):
        t.tune(ctx, 0, GRD, CS, REC)


@pytest.mark.gpu
def test_tuner_on_the_gpu(tmp_path):
    from eikonalsolvers import Context
    w = CF.cfg3(scale=0.25, nsrc=4, nrec_side=5)
    ctx, ref = Context(0), Context(0)
    try:
        mid, mref = ctx.upload(w.vel, w.grd), ref.upload(w.vel, w.grd)
        t = Tuner(path=str(tmp_path / "t.json"), repeats=1, shipped=None)
        e = ctx.autotune(mid, w.grd, w.coordsrc, w.coordrec, tuner=t)
        assert len(e["timings"]) == 9 and e["ms"] == min(x[2] for x in e["timings"])
        got = ctx.traveltime(mid, w.grd, w.coordsrc, w.coordrec)
        want = ref.traveltime(mref, w.grd, w.coordsrc, w.coordrec)
        assert all(np.array_equal(a, b) for a, b in zip(got, want))
    finally:
        ctx.close()
        ref.close()


def test_shipped_table_covers_the_standard_workloads():
    """The table shipped with the package (measured on a B200 by Tuner.tune) has entries for
    the 256^3 x 32-source 3D workload and the 1024 x 640 x 64-source 2D workload, each one of
    the timed candidates, and the caller's own table takes precedence over it."""
    t = Tuner(path="")
    for w, n in ((CF.cfg3(scale=1.0, nsrc=1, nrec_side=2), 32), (CF.cfg2(scale=1.0, nsrc=1), 64)):
        e = t.lookup(w.grd, n, ExtraParams())
        assert e is not None
        assert [e["round_gate"], e["ctas_per_sm"], e["ms"]] in e["timings"]
        ctx = FakeContext(lambda g, c: 1.0)
        assert t.apply_known(ctx, w.grd, n, ExtraParams()) == e
        assert ctx.params == {"round_gate": e["round_gate"], "ctas_per_sm": float(e["ctas_per_sm"])}
    own = Tuner(path="")
    own.table[workload_key(CF.cfg2(scale=1.0, nsrc=1).grd, 64)] = {"round_gate": 9.0, "ctas_per_sm": 1}
    assert own.lookup(CF.cfg2(scale=1.0, nsrc=1).grd, 64)["round_gate"] == 9.0
