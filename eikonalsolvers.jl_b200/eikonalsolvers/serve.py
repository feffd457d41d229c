"""Continuous-batching request loop for many-model traveltime / gradient evaluations.

The reference has no server: its callers (an HMC sampler evaluating `eikttimemisfit` and
`eikgradient` for model after model, `HMCtraveltimes.jl`) call the solvers one at a time.
This loop serves such callers from many threads or processes on one GPU:

* velocity models are registered once and kept resident on the device (uploaded lazily to
  each worker slot and reused by every request that names them);
* every worker slot owns a libeikcuda context (its own CUDA stream, scratch memory under
  its own HBM budget, a share of the SMs for the persistent solve kernels), so requests
  taken by different slots run on the GPU at the same time;
* a slot that becomes free takes the oldest waiting request, together with the waiting
  requests it can share a call with (up to a source cap): traveltime requests on any models
  of the same dimension and parameters (one eik_traveltime_multi pipeline, grids of
  different sizes side by side), or gradient requests on the same model with the same
  `whichgrad` and parameters (one eik_gradient_groups pipeline, each request a source group
  with its own buffer and outputs); the results are split back per request;
* admission by device memory: with a server-wide ``hbm_budget`` every batch's device
  footprint is estimated (``request_bytes``: the per-node-source state of the forward solve,
  and of the adjoint for gradients, times grid nodes and sources, plus the refined windows),
  and a slot that took a batch waits until the batch fits beside the batches in flight; a
  batch that could not fit even alone fails with an error and the server goes on;
* a request that does not fit a slot's own HBM budget fails alone (EIK_ERR_OUT_OF_BUDGET);
* cancellation: a request whose future was cancelled (``Future.cancel()``) before a slot
  took it is dropped from the queue and never reaches the GPU;
* load shedding: with ``max_queue`` > 0 a request that arrives while that many wait is
  refused at once (its future raises ServerOverloaded) instead of queueing without bound;
  `stats()` counts the refusals;
* latency (submission to completion) is recorded per request; `stats()` gives p50/p99 and
  source-solves/s;
* each call runs with the launch parameters the autotuner's table holds for its workload
  class (the library's choice by size otherwise).

Results do not depend on the mix: the forward traveltimes are the unique fixed point of
the order rule whatever the batch, and merged gradient requests keep their own source-point
carry-over and sums (per-group outputs), so each result is identical to the same request
served alone.
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


class ServerOverloaded(RuntimeError):
    """The request queue was full when the request arrived (Server(max_queue=...))."""


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


def batch_bytes(batch, models) -> int:
    """Estimated device memory of one merged call: request_bytes at the largest grid of the
    batch (the per-source arrays of a multi-model call share that stride) for all its sources."""
    grds = [models[r.model][1] for r in batch]
    big = max(grds, key=lambda g: int(np.prod(g.grsize)))
    return request_bytes(big, sum(r.nsrc for r in batch), batch[0].kind, batch[0].extraparams)


def _ep_key(ep: Optional[ExtraParams]):
    if ep is None:
        return None
    return (ep.refinearoundsrc, ep.grdrefpars.downscalefactor, ep.grdrefpars.noderadius,
            ep.radiussmoothgradsrc, ep.smoothgradkern, ep.parallelkind)


class Server:
    """Serves `Request`s on one GPU with `slots` concurrent worker contexts."""

    def __init__(self, device: int = 0, slots: int = 2, hbm_budget_per_slot: int = 0,
                 max_batch_sources: int = 64, context_factory=None, tuner=None, hbm_budget: int = 0,
                 max_queue: int = 0):
        self.slots = max(1, int(slots))
        self.hbm_budget = int(hbm_budget)  # device bytes the batches in flight may take together (0 = no limit)
        self._inflight = 0
        self.max_inflight_seen = 0
        self._mem_cv = threading.Condition()  # admission waits here, apart from the request queue
        # launch parameters per workload class (autotuner table; results do not depend on them)
        self.tuner = tuner if tuner is not None else default_tuner()
        self.max_batch_sources = int(max_batch_sources)
        self.max_queue = int(max_queue)  # waiting requests beyond which arrivals are refused (0 = no limit)
        self._refused = 0
        self._cancelled = 0
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
            if self.max_queue > 0 and len(self._queue) >= self.max_queue:
                self._refused += 1
                req.future.set_exception(ServerOverloaded(f"{len(self._queue)} requests are waiting"))
                return req.future
            self._queue.append(req)
            self._cv.notify()
        return req.future

    def _batch_key(self, r: Request):
        """Requests with equal keys can share one call."""
        if r.kind == "traveltime":
            return ("traveltime", self._models[r.model][1].ndim, _ep_key(r.extraparams))
        return ("gradient", r.model, r.whichgrad, _ep_key(r.extraparams))

    def _take(self) -> Optional[List[Request]]:
        """Oldest request plus the waiting requests it can share a call with."""
        with self._cv:
            while True:
                while not self._queue and not self._closing:
                    self._cv.wait()
                if not self._queue:
                    return None
                head = self._queue.popleft()
                if head.future.set_running_or_notify_cancel():
                    break
                self._cancelled += 1  # cancelled while waiting: dropped
            batch = [head]
            key = self._batch_key(head)
            n = head.nsrc
            keep = deque()
            while self._queue:
                r = self._queue.popleft()
                # with a device-memory budget, a merged batch must still fit it: requests
                # that fit alone are not refused only because they were batched together
                ok = self._batch_key(r) == key and n + r.nsrc <= self.max_batch_sources
                if ok and self.hbm_budget > 0:
                    ok = batch_bytes(batch + [r], self._models) <= self.hbm_budget
                if r.future.cancelled():
                    self._cancelled += 1
                elif ok and r.future.set_running_or_notify_cancel():
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
            need = batch_bytes(batch, self._models)
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
                results = [(True, x) for x in self._run(slot, ctx, batch)]
            except Exception as e:  # the request fails, the server goes on
                if len(batch) == 1:
                    results = [(False, e)]
                else:
                    # a merged call failed: each request again on its own, so that a failure
                    # stays with the request that caused it
                    results = []
                    for r in batch:
                        try:
                            results.append((True, self._run(slot, ctx, [r])[0]))
                        except Exception as e1:
                            results.append((False, e1))
            self._release(need)
            t1 = time.perf_counter()
            with self._cv:
                self._busy_s += t1 - t0
                for i, r in enumerate(batch):
                    r.t_done = t1
                    self._done.append(r)
            for (ok, x), r in zip(results, batch):
                if ok:
                    r.future.set_result(x)
                else:
                    r.future.set_exception(x)

    def _run(self, slot: int, ctx, batch: List[Request]) -> list:
        """One call for the batch; one result per request, in batch order."""
        head = batch[0]
        nsrc = sum(r.nsrc for r in batch)
        grds = [self._models[r.model][1] for r in batch]
        big = max(grds, key=lambda g: int(np.prod(g.grsize)))
        if not self.tuner.apply_known(ctx, big, nsrc, head.extraparams):
            ctx.set_param("round_gate", 0.0)  # the library's choice by size
            ctx.set_param("ctas_per_sm", 0)
        if head.kind == "gradient":
            grd = grds[0]
            mid = self._model_id(slot, head.model)
            if len(batch) == 1:
                return [ctx.gradient(mid, grd, head.coordsrc, head.coordrec, head.pickobs, head.stdobs,
                                     head.whichgrad, extraparams=head.extraparams)]
            return ctx.gradient_groups(mid, grd, [(r.coordsrc, r.coordrec, r.pickobs, r.stdobs) for r in batch],
                                       head.whichgrad, extraparams=head.extraparams)
        # traveltime: the requests of each model together, models in order of first appearance
        order = []
        for r in batch:
            if r.model not in order:
                order.append(r.model)
        if len(order) == 1:
            mid = self._model_id(slot, head.model)
            cs = np.vstack([np.atleast_2d(r.coordsrc) for r in batch])
            recs = [rr for r in batch for rr in r.coordrec]
            picks = ctx.traveltime(mid, grds[0], cs, recs, extraparams=head.extraparams)
        else:
            reqs = []
            for key in order:
                rs = [r for r in batch if r.model == key]
                reqs.append((self._model_id(slot, key), self._models[key][1],
                             np.vstack([np.atleast_2d(r.coordsrc) for r in rs]), [rr for r in rs for rr in r.coordrec]))
            per_model = ctx.traveltime_multi(reqs, extraparams=head.extraparams)
            by_model = dict(zip(order, per_model))
            picks = []
            taken = {k: 0 for k in order}
            for r in batch:
                k0 = taken[r.model]
                picks.extend(by_model[r.model][k0:k0 + r.nsrc])
                taken[r.model] = k0 + r.nsrc
        results, k = [], 0
        for r in batch:
            results.append(picks[k:k + r.nsrc])
            k += r.nsrc
        return results

    # ------------------------------------------------------------------- stats --
    def stats(self) -> dict:
        with self._cv:
            done = list(self._done)
            refused = self._refused
            cancelled = self._cancelled
        if not done:
            return {"requests": 0, "refused": refused, "cancelled": cancelled}
        lat = np.array([r.t_done - r.t_submit for r in done])
        t0 = min(r.t_submit for r in done)
        t1 = max(r.t_done for r in done)
        nsrc = sum(r.nsrc for r in done)
        return {"requests": len(done), "p50_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_ms": float(np.percentile(lat, 99) * 1e3), "mean_ms": float(lat.mean() * 1e3),
                "source_solves_per_s": nsrc / (t1 - t0) if t1 > t0 else None,
                "requests_per_s": len(done) / (t1 - t0) if t1 > t0 else None, "refused": refused,
                "cancelled": cancelled}

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
