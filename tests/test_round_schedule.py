"""The forward round solver's schedule, emulated on the host (round_schedule_harness.cpp: the
node visit of node.cuh restated around the product's order rule, stencil.cuh compiled for the
host), reaches the oracle's heap-FMM traveltimes bit for bit whatever the order of the visits
within a round and whatever the round width: visits one after the other in list or random
order, visits interleaved at the extreme concurrent visits allow (all of a round's reads, then
all its writes, then all its relist filters), visits that read a neighbour changed earlier in
the round at its old or its new state (its traveltime, code and key level each from its own
moment, as unordered loads may see them, or tied together), and nodes waiting above the front
parked by front (exactly, or in buckets by front) instead of listed again every round. Seeds 21
and 37 of the independent-read mode are the orders in which 3Dconst2 and 3Dconst3 reached NaN
traveltimes and a wrong fixed point before node_key ignored a special key beside an unreached
traveltime. The kernels run the
same visit with concurrent visits inside a round; these runs pin, on all 16 reference cases and
three seeded workloads and without a GPU, that the fixed point does not depend on the order."""
import os
import shutil
import struct
import subprocess

import numpy as np
import pytest

import eikoracle as O
import refcases as RC
from eikonalsolvers import ExtraParams
from eikonalsolvers import configs as CF

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "eikonalsolvers.jl_b200", "csrc")


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    if not shutil.which("g++"):
        pytest.skip("g++ not available")
    d = tmp_path_factory.mktemp("rounds")
    exe = str(d / "harness")
    cmd = ["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-I", CSRC,
           os.path.join(HERE, "round_schedule_harness.cpp"), "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    return exe, d


def _emulate(harness, vel, grd, src, gate, mode, seed):
    """Runs the emulated round solver for one source (no refined start-up) and returns
    (its traveltimes, the oracle's, the run's counters)."""
    exe, d = harness
    dbg = O.forward_debug(vel, grd, np.asarray(src, dtype=np.float64), extraparams=ExtraParams(refinearoundsrc=False))
    tt = dbg["tt"].ravel(order="F")
    seeds = np.ascontiguousarray(dbg["srcpts"], dtype=np.int64)
    slow = 1.0 / np.asarray(vel, dtype=np.float64).ravel(order="F")  # as the product's slowness kernel
    n = list(grd.grsize) + [1] * (3 - grd.ndim)
    fin, fout = str(d / "in.bin"), str(d / "out.bin")
    with open(fin, "wb") as f:
        f.write(struct.pack("<4i2diQq", grd.ndim, *n, grd.hgrid, gate, mode, seed, seeds.size))
        f.write(slow.tobytes())
        f.write(seeds.tobytes())
        f.write(np.ascontiguousarray(tt[seeds]).tobytes())
    subprocess.run([exe, fin, fout], check=True)
    out = np.fromfile(fout, dtype=np.float64, count=tt.size)
    st = np.fromfile(fout, dtype=np.int64, offset=8 * tt.size)
    stats = dict(rounds=int(st[0]), entries=int(st[1]), evals=int(st[2]), visits=[int(x) for x in st[3:10]],
                 unparked=int(st[10]), unsettled=int(st[11]), special_unreached=int(st[12]))
    return out, tt, stats


def _check(out, tt, stats):
    ndiff = int((out != tt).sum())
    assert ndiff == 0, f"{ndiff} nodes differ from the oracle"
    assert stats["rounds"] < 1 << 20 and stats["unsettled"] == 0
    # every special key sits beside a reached traveltime (what lets node_key ignore the others)
    assert stats["special_unreached"] == 0
    assert sum(stats["visits"]) == stats["entries"]
    assert sum(stats["visits"][4:7]) == stats["evals"]


@pytest.mark.parametrize("case", RC.all_forward_cases(), ids=lambda c: c["name"])
def test_reference_cases_any_order_any_width(harness, case):
    src = np.atleast_2d(case["coordsrc"])[0]
    for gate, mode, seed in [(1.0, 0, 0), (0.5, 1, 1), (2.0, 1, 2), (8.0, 1, 3), (1.0, 2, 4), (1.0, 5, 5),
                             (1.0, 7, 6), (4.0, 7, 7), (2.0, 8, 11), (2.0, 8, 21), (2.0, 8, 37), (2.0, 9, 8),
                             (2.0, 10, 9), (2.0, 11, 10)]:
        _check(*_emulate(harness, case["vel"], case["grd"], src, gate, mode, seed))


_WORKLOADS = {
    "cfg1_300x220": lambda: CF.cfg1(),
    "cfg3_32cubed": lambda: CF.cfg3(scale=0.125, nsrc=2, nrec_side=3),
    "cfg2_128x80_random_field": lambda: CF.cfg2(scale=0.125, nsrc=2),
}


@pytest.mark.parametrize("which", sorted(_WORKLOADS))
def test_seeded_workloads_any_order(harness, which):
    w = _WORKLOADS[which]()
    for s, src in enumerate(w.coordsrc[:2]):
        for gate, mode, seed in [(1.0, 1, 10 + s), (4.0, 1, 20 + s), (1.0, 2, 30 + s), (1.0, 3, 40 + s),
                                 (1.0, 7, 50 + s), (2.0, 8, 60 + s)]:
            _check(*_emulate(harness, w.vel, w.grd, src, gate, mode, seed))


def test_parking_waiting_nodes_saves_list_entries(harness):
    """Waiting nodes are most of the list entries at narrow round widths: parking them by
    front leaves the result unchanged and takes about a third fewer entries (300x220 at round
    width 1); buckets of 1/16 round width by front keep most of that."""
    w = CF.cfg1()
    src = w.coordsrc[0]
    out1, tt, listed = _emulate(harness, w.vel, w.grd, src, 1.0, 1, 5)
    out2, _, parked = _emulate(harness, w.vel, w.grd, src, 1.0, 2, 5)
    out3, _, bucketed = _emulate(harness, w.vel, w.grd, src, 1.0, 5, 5)
    for o, st in ((out1, listed), (out2, parked), (out3, bucketed)):
        _check(o, tt, st)
    assert parked["unparked"] > 0 and bucketed["unparked"] > 0
    assert parked["entries"] < 0.8 * listed["entries"], (parked["entries"], listed["entries"])
    assert bucketed["entries"] < 0.8 * listed["entries"], (bucketed["entries"], listed["entries"])
