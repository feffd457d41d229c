"""Autotuner of the forward solve's launch parameters.

The forward solve's result is the unique fixed point of the FMM order rule, so its launch
parameters change only how much work it takes to get there: the round width
(``round_gate``, in units of smallest spacing x smallest slowness: wider rounds mean fewer
grid barriers but more nodes evaluated before their inputs are final) and the number of
resident CTAs per SM of the persistent launch (``ctas_per_sm``: more CTAs hide more memory
latency, fewer leave each thread more registers and less barrier traffic). The best pair
depends on the grid size, the number of sources in flight and the GPU.

``Tuner.tune`` times every candidate pair on the caller's own workload (a traveltime call,
the forward being most of a gradient call too), checks that every candidate returned the
same picks bit for bit (a live check of the schedule independence the solver relies on:
a difference raises), sets the fastest pair on the context and remembers it under a key of
the workload's shape class (dimension, node count and source count rounded up to powers of
two, refined start-up or not). Later calls with a workload of the same class reuse the
entry without timing. The table can be kept in a JSON file (``path``, or the
``EIK_TUNE_CACHE`` environment variable) so that a serving process or a sampler starts
tuned. Below the caller's table sits the table shipped with the package
(``tuned_b200.json``: entries measured by ``Tuner.tune`` on a B200 for the standard
workloads), consulted when the caller's table has no entry for a class.
"""
from __future__ import annotations

import json
import math
import os
import threading
from typing import Dict, Iterable, Optional, Sequence

import numpy as np

DEFAULT_CANDIDATES: Dict[str, Sequence[float]] = {"round_gate": (1.0, 2.0, 3.0), "ctas_per_sm": (2, 3, 4)}
SHIPPED_TABLE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuned_b200.json")


def _pow2(n: int) -> int:
    return 1 << max(0, int(math.ceil(math.log2(max(1, int(n))))))


def workload_key(grd, nsrc: int, extraparams=None) -> str:
    refine = True if extraparams is None else bool(extraparams.refinearoundsrc)
    npts = int(np.prod(grd.grsize))
    return f"{type(grd).__name__}:n{_pow2(npts)}:s{_pow2(nsrc)}:r{int(refine)}"


class Tuner:
    """Table of tuned launch parameters per workload class, optionally kept in a JSON file."""

    def __init__(self, path: Optional[str] = None, candidates: Optional[Dict[str, Iterable[float]]] = None,
                 repeats: int = 2, shipped: Optional[str] = SHIPPED_TABLE):
        self.path = path if path is not None else os.environ.get("EIK_TUNE_CACHE")
        self.candidates = {k: tuple(v) for k, v in (candidates or DEFAULT_CANDIDATES).items()}
        self.repeats = max(1, int(repeats))
        self.table: Dict[str, dict] = {}
        self.base: Dict[str, dict] = {}
        self._lock = threading.Lock()
        if shipped and os.path.exists(shipped):
            with open(shipped) as f:
                self.base = json.load(f)
        if self.path and os.path.exists(self.path):
            with open(self.path) as f:
                self.table = json.load(f)

    def _save(self):
        if not self.path:
            return
        tmp = self.path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(self.table, f, indent=1, sort_keys=True)
        os.replace(tmp, self.path)

    @staticmethod
    def apply(ctx, entry: dict):
        ctx.set_param("round_gate", float(entry["round_gate"]))
        ctx.set_param("ctas_per_sm", float(entry["ctas_per_sm"]))

    def _get(self, key: str) -> Optional[dict]:
        with self._lock:
            e = self.table.get(key)
        return e if e is not None else self.base.get(key)

    def lookup(self, grd, nsrc: int, extraparams=None) -> Optional[dict]:
        return self._get(workload_key(grd, nsrc, extraparams))

    def apply_known(self, ctx, grd, nsrc: int, extraparams=None) -> Optional[dict]:
        """Applies the table's entry for this workload class, if any (no timing)."""
        e = self.lookup(grd, nsrc, extraparams)
        if e is not None:
            self.apply(ctx, e)
        return e

    def tune(self, ctx, model: int, grd, coordsrc, coordrec, extraparams=None, force: bool = False) -> dict:
        """Sets the fastest (round_gate, ctas_per_sm) for this workload on ``ctx`` and returns
        the table entry: {"round_gate", "ctas_per_sm", "ms", "timings"}."""
        nsrc = int(np.atleast_2d(coordsrc).shape[0])
        key = workload_key(grd, nsrc, extraparams)
        entry = self._get(key)
        if entry is not None and not force:
            self.apply(ctx, entry)
            return entry
        ref = None
        timings = []
        best = None
        for gate in self.candidates["round_gate"]:
            for ctas in self.candidates["ctas_per_sm"]:
                ctx.set_param("round_gate", float(gate))
                ctx.set_param("ctas_per_sm", float(ctas))
                ms = math.inf
                for _ in range(self.repeats):
                    picks = ctx.traveltime(model, grd, coordsrc, coordrec, extraparams=extraparams)
                    ms = min(ms, float(ctx.last_stats.device_ms))
                if ref is None:
                    ref = picks
                elif any(not np.array_equal(a, b) for a, b in zip(ref, picks)):
                    raise RuntimeError(f"forward picks changed with round_gate={gate}, ctas_per_sm={ctas}: "
                                       "the solve is not schedule independent on this workload")
                timings.append([float(gate), int(ctas), ms])
                if best is None or ms < best[2]:
                    best = timings[-1]
        entry = {"round_gate": best[0], "ctas_per_sm": best[1], "ms": best[2], "timings": timings}
        self.apply(ctx, entry)
        with self._lock:
            self.table[key] = entry
            self._save()
        return entry


_default_tuner: Optional[Tuner] = None


def default_tuner() -> Tuner:
    global _default_tuner
    if _default_tuner is None:
        _default_tuner = Tuner()
    return _default_tuner
