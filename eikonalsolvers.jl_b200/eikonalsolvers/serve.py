"""Continuous-batching request loop for many-model traveltime / gradient evaluations.

The reference has no server: its callers (an HMC sampler evaluating `eikttimemisfit` and
`eikgradient` for model after model, `HMCtraveltimes.jl`) call the solvers one at a time.
This loop serves such callers from many threads or processes on one GPU:

* velocity models are registered once and kept resident on the device (uploaded lazily to
  each worker slot and reused by every request that names them);
* every worker slot owns a libeikcuda context (its own CUDA stream, scratch memory under
  its own HBM budget, a share of the SMs for the persistent solve kernels), so requests
  taken by different slots run on the GPU at the same time;
* a slot that becomes free takes the oldest waiting request, together with every other
  waiting traveltime request on the same model and parameters (up to a source cap): they
  run as one batched call and the picks are split back per request;
* admission by device memory: with a server-wide ``hbm_budget`` every batch's device
  footprint is estimated (``request_bytes``: the per-node-source state of the forward solve,
  and of the adjoint for gradients, times grid nodes and sources, plus the refined windows),
  and a slot that took a batch waits until the batch fits beside the batches in flight; a
  batch that could not fit even alone fails with an error and the server goes on;
* a request that does not fit a slot's own HBM budget fails alone (EIK_ERR_OUT_OF_BUDGET);
* latency (submission to completion) is recorded per request; `stats()` gives p50/p99 and
  source-solves/s;
* each call runs with the launch parameters the autotuner's table holds for its workload
  class (the library's choice by size otherwise).

Results do not depend on the mix: the forward traveltimes are the unique fixed point of
the order rule whatever the batch, and gradient requests are never merged (their
source-point carry-over would couple them), so each result is identical to the same
request served alone.
"""
from __future__ import annotations

import threading
import time
from collections import deque
from concurrent.futures import Future
from dataclasses import dataclass, field
from typing import Any, Dict, List, Optional

import numpy as np

from .api import Context
from .structs import ExtraParams
from .tune import default_tuner


@dataclass
class Request:
    """One evaluation: `kind` is "traveltime" or "gradient" (then `whichgrad`)."""
    model: Any
    kind: str
    coordsrc: np.ndarray
    coordrec: List[np.ndarray]
    pickobs: Optional[List[np.ndarray]] = None
    stdobs: Optional[List[np.ndarray]] = None
    whichgrad: str = "gradvel"
    extraparams: Optional[ExtraParams] = None
    t_submit: float = 0.0
    t_start: float = 0.0
    t_done: float = 0.0
    future: Future = field(default_factory=Future)

    @property
    def nsrc(self) -> int:
        return int(np.atleast_2d(self.coordsrc).shape[0])


def request_bytes(grd, nsrc: int, kind: str, extraparams: Optional[ExtraParams] = None) -> int:
    """Estimated device memory of one batched call: per node and source the forward's fields
    (traveltime, codes, keys: 18 B) and round-solver state (stamp, cached front, dirty flag,
    two worklist entries: 29 B), for gradients also the adjoint's (λ, right-hand side and
    2·(D t) per axis: 16 + 8·ndim B); plus the refined windows ((2r+1)·ds+1 nodes per axis)."""
    ep = extraparams or ExtraParams()
    n = int(np.prod(grd.grsize))
    per = 47 + ((16 + 8 * grd.ndim) if kind == "gradient" else 0)
    fine = 0
    if ep.refinearoundsrc:
        side = (2 * ep.grdrefpars.noderadius + 1) * ep.grdrefpars.downscalefactor + 1
        fine = side ** grd.ndim * 48
    return int(nsrc) * (n * per + fine)


def _ep_key(ep: Optional[ExtraParams]):
    if ep is None:
        return None
    return (ep.refinearoundsrc, ep.grdrefpars.downscalefactor, ep.grdrefpars.noderadius,
            ep.radiussmoothgradsrc, ep.smoothgradkern, ep.parallelkind)


class Server:
    """Serves `Request`s on one GPU with `slots` concurrent worker contexts."""

    def __init__(self, device: int = 0, slots: int = 2, hbm_budget_per_slot: int = 0,
                 max_batch_sources: int = 64, context_factory=None, tuner=None, hbm_budget: int = 0):
        self.slots = max(1, int(slots))
        self.hbm_budget = int(hbm_budget)  # device bytes the batches in flight may take together (0 = no limit)
        self._inflight = 0
        self.max_inflight_seen = 0
        self._mem_cv = threading.Condition()  # admission waits here, apart from the request queue
        # launch parameters per workload class (autotuner table; results do not depend on them)
        self.tuner = tuner if tuner is not None else default_tuner()
        self.max_batch_sources = int(max_batch_sources)
        make = context_factory or (lambda: Context(device, hbm_budget_per_slot))
        self._ctx = []
        for _ in range(self.slots):
            c = make()
            c.set_param("sm_fraction", 1.0 / self.slots)
            self._ctx.append(c)
        self._models: Dict[Any, tuple] = {}
        self._resident: List[Dict[Any, int]] = [dict() for _ in range(self.slots)]
        self._queue: deque = deque()
        self._cv = threading.Condition()
        self._closing = False
        self._done: List[Request] = []
        self._busy_s = 0.0
        self._threads = [threading.Thread(target=self._worker, args=(i,), daemon=True) for i in range(self.slots)]
        for t in self._threads:
            t.start()

    # ---------------------------------------------------------------- models --
    def register_model(self, key, vel: np.ndarray, grd):
        """Makes a velocity model available under `key` (uploaded on first use per slot)."""
        with self._cv:
            self._models[key] = (np.asarray(vel, dtype=np.float64), grd)

    def _model_id(self, slot: int, key) -> int:
        res = self._resident[slot]
        if key not in res:
            vel, grd = self._models[key]
            res[key] = self._ctx[slot].upload(vel, grd)
        return res[key]

    # ---------------------------------------------------------------- requests --
    def submit(self, req: Request) -> Future:
        if req.model not in self._models:
            raise KeyError(f"model {req.model!r} is not registered")
        if req.kind not in ("traveltime", "gradient"):
            raise ValueError("kind must be 'traveltime' or 'gradient'")
        req.t_submit = time.perf_counter()
        with self._cv:
            if self._closing:
                raise RuntimeError("server is closed")
            self._queue.append(req)
            self._cv.notify()
        return req.future

    def _take(self) -> Optional[List[Request]]:
        """Oldest request plus the waiting traveltime requests it can be batched with."""
        with self._cv:
            while not self._queue and not self._closing:
                self._cv.wait()
            if not self._queue:
                return None
            head = self._queue.popleft()
            batch = [head]
            if head.kind == "traveltime":
                n = head.nsrc
                key = (head.model, _ep_key(head.extraparams))
                grd = self._models[head.model][1]
                keep = deque()
                while self._queue:
                    r = self._queue.popleft()
                    # with a device-memory budget, a merged batch must still fit it: requests
                    # that fit alone are not refused only because they were batched together
                    fits = (self.hbm_budget <= 0 or
                            request_bytes(grd, n + r.nsrc, "traveltime", head.extraparams) <= self.hbm_budget)
                    if (r.kind == "traveltime" and (r.model, _ep_key(r.extraparams)) == key
                            and n + r.nsrc <= self.max_batch_sources and fits):
                        batch.append(r)
                        n += r.nsrc
                    else:
                        keep.append(r)
                self._queue = keep
            return batch

    def _admit(self, need: int) -> bool:
        """Waits until `need` bytes fit beside the batches in flight; False if they never can."""
        if self.hbm_budget <= 0:
            return True
        if need > self.hbm_budget:
            return False
        with self._mem_cv:
            while self._inflight + need > self.hbm_budget:
                self._mem_cv.wait()
            self._inflight += need
            self.max_inflight_seen = max(self.max_inflight_seen, self._inflight)
        return True

    def _release(self, need: int):
        if self.hbm_budget <= 0:
            return
        with self._mem_cv:
            self._inflight -= need
            self._mem_cv.notify_all()

    def _worker(self, slot: int):
        ctx = self._ctx[slot]
        while True:
            batch = self._take()
            if batch is None:
                return
            grd0 = self._models[batch[0].model][1]
            need = request_bytes(grd0, sum(r.nsrc for r in batch), batch[0].kind, batch[0].extraparams)
            if not self._admit(need):
                err = MemoryError(f"request needs ~{need} bytes of device memory, the server's budget is "
                                  f"{self.hbm_budget}")
                t1 = time.perf_counter()
                with self._cv:
                    for r in batch:
                        r.t_start = r.t_done = t1
                        self._done.append(r)
                for r in batch:
                    r.future.set_exception(err)
                continue
            t0 = time.perf_counter()
            for r in batch:
                r.t_start = t0
            try:
                grd = self._models[batch[0].model][1]
                mid = self._model_id(slot, batch[0].model)
                nsrc = sum(r.nsrc for r in batch)
                if not self.tuner.apply_known(ctx, grd, nsrc, batch[0].extraparams):
                    ctx.set_param("round_gate", 0.0)  # the library's choice by size
                    ctx.set_param("ctas_per_sm", 0)
                if batch[0].kind == "traveltime":
                    cs = np.vstack([np.atleast_2d(r.coordsrc) for r in batch])
                    recs = [rr for r in batch for rr in r.coordrec]
                    picks = ctx.traveltime(mid, grd, cs, recs, extraparams=batch[0].extraparams)
                    k = 0
                    results = []
                    for r in batch:
                        results.append(picks[k:k + r.nsrc])
                        k += r.nsrc
                else:
                    r = batch[0]
                    results = [ctx.gradient(mid, grd, r.coordsrc, r.coordrec, r.pickobs, r.stdobs, r.whichgrad,
                                            extraparams=r.extraparams)]
                err = None
            except Exception as e:  # the request fails, the server goes on
                err = e
            self._release(need)
            t1 = time.perf_counter()
            with self._cv:
                self._busy_s += t1 - t0
                for i, r in enumerate(batch):
                    r.t_done = t1
                    self._done.append(r)
            for i, r in enumerate(batch):
                if err is None:
                    r.future.set_result(results[i])
                else:
                    r.future.set_exception(err)

    # ------------------------------------------------------------------- stats --
    def stats(self) -> dict:
        with self._cv:
            done = list(self._done)
        if not done:
            return {"requests": 0}
        lat = np.array([r.t_done - r.t_submit for r in done])
        t0 = min(r.t_submit for r in done)
        t1 = max(r.t_done for r in done)
        nsrc = sum(r.nsrc for r in done)
        return {"requests": len(done), "p50_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_ms": float(np.percentile(lat, 99) * 1e3), "mean_ms": float(lat.mean() * 1e3),
                "source_solves_per_s": nsrc / (t1 - t0) if t1 > t0 else None,
                "requests_per_s": len(done) / (t1 - t0) if t1 > t0 else None}

    def close(self):
        with self._cv:
            self._closing = True
            self._cv.notify_all()
        for t in self._threads:
            t.join()
        for s, c in enumerate(self._ctx):
            for mid in self._resident[s].values():
                try:
                    c.release(mid)
                except Exception:
                    pass
            c.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
