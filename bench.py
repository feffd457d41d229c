#!/usr/bin/env python
"""Benchmark of the forward + discrete-adjoint path: gradient source-solves/s.

Workload (default): 3D Cartesian eikgradient :gradvelandsrcloc on 256^3 nodes, hgrid 0.1,
4-layer velocity (3.0/4.2/5.5/6.8) with seeded sinusoidal interfaces plus 2% white
perturbation, 32 sources in the lower half, 400 receivers on a 20x20 surface grid,
observations from a 5%-perturbed model plus N(0, 0.01^2) noise, default ExtraParams
(refined start-up ds=5 r=3, source smoothing radius 3). All inputs are seeded synthetic.

One step = one batched gradient call over the rank's sources (forward FMM fixed point,
adjoint dataflow solve, gradient assembly). Every per-source field is 134 MB and the
working set is tens of GB, far above the 126 MB L2, so no flush is needed between steps.

Lines printed by rank 0 (one JSON object):
  value     source-solves/s of the whole job, inputs resident on the device (C-ABI
            eik_gradient_device), timed with CUDA events on the library's stream
  e2e       the same through eik_gradient with pinned host buffers, host<->device copies
            inside the timed region
  plain     the same workload one source per call (the unbatched path)
  roofline  HBM roofline of the dominant kernel (algorithmic bytes / measured duration)
  cpu_baseline  the oracle (C++ restatement of the reference algorithm) on the host cores, on
            the 256^3 workload itself (one source per thread), with the earlier 128^3
            sub-block sample beside it
  serve     the serving leg: Poisson arrivals of a mixed traveltime/gradient workload
  rays      the ray-tracing leg (tracerays on 128^3 grids): GPU rays/s beside the oracle's
  hmc       HMC-style evaluations: eik_gradient per new velocity vs a replayed CUDA-graph plan
  parity    the timed configuration against the oracle: forward fields of 4 of the batched
            call's sources bit for bit, the gradient of the CPU leg's sources (rel. L2)
  configs   the other benchmark configurations (2D 300x220 traveltime, 2D 1024x640 and
            Grid3DSphere 200x180x180 gradients) end to end beside the oracle, and the batched
            call over one source per call at 64^3, 128^3 and 512x320

--impl reference: times the oracle on the host cores instead (rank 0 only).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "eikonalsolvers.jl_b200"))

import numpy as np  # noqa: E402

METRIC = "gradient source-solves/s @256^3 batched vs plain GPU; p50/p99 serve latency"
UNIT = "source-solves/s"
L2_BYTES = 126 * 1024 * 1024


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--scale", type=float, default=1.0, help="grid scale (1.0 = 256^3)")
    ap.add_argument("--nsrc", type=int, default=32, help="sources per rank")
    ap.add_argument("--plain-sources", type=int, default=2,
                    help="sources timed one per call for the plain path (0 = skip)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--no-parity", action="store_true", help="skip the parity check against the oracle")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the other benchmark configurations and the batched/plain sizes")
    ap.add_argument("--e2e-steps", type=int, default=1)
    ap.add_argument("--serve-requests", type=int, default=30,
                    help="requests of the serving leg (Poisson arrivals; 0 = skip)")
    ap.add_argument("--serve-rate", type=float, default=2.0, help="arrival rate of the serving leg, req/s")
    ap.add_argument("--serve-slots", type=int, default=2)
    ap.add_argument("--ray-sources", type=int, default=8, help="sources of the ray-tracing leg (0 = skip)")
    ap.add_argument("--hmc-evals", type=int, default=20, help="evaluations of the HMC-style leg (0 = skip)")
    ap.add_argument("--ray-cpu-rays", type=int, default=24, help="rays the oracle traces for the CPU figure")
    ap.add_argument("--serve-scale", type=float, default=1.0, help="grid scale of the serving mix")
    ap.add_argument("--serve-sweep", type=str, default="",
                    help="comma-separated arrival rates (req/s): run only the serving sweep, each rate for "
                         "min(2000, 60 s x rate) requests, and print one JSON line")
    ap.add_argument("--serve-max-queue", type=int, default=64,
                    help="waiting requests beyond which the sweep's server refuses arrivals")
    ap.add_argument("--serve-batch-sources", type=int, default=128, help="source cap of a merged call")
    return ap.parse_args()


# ------------------------------------------------------------------------ helpers --
def log(msg):
    sys.stderr.write(f"[bench] {msg}\n")
    sys.stderr.flush()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def measured_peaks():
    p = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(name):
    """DRAM bytes per node-solve of a kernel from a committed ncu summary, if one exists:
    a line `traffic_bytes_per_node_solve: <float>` in profiles/<name>.md (captured on a
    smaller case; traffic grows with the node-solves of a launch)."""
    p = os.path.join(REPO, "profiles", name + ".md")
    if not os.path.exists(p):
        return None
    m = re.search(r"traffic_bytes_per_node_solve:\s*([0-9.eE+]+)", open(p).read())
    return float(m.group(1)) if m else None


class Clocks:
    """nvidia-smi samples (200 ms) during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = []
        for line in open(self.f.name):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 9 and parts[1].replace(".", "").isdigit():
                rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in rows]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": float(rows[0][2]), "reasons": reasons,
                "samples": len(rows), "power_w_max": max(float(r[3]) for r in rows if r[3].replace(".", "").isdigit())}


def host_cores(cap=32, gb_per_thread=1.5):
    """Host threads for the CPU leg: all cores this process may use, at most `cap` and at
    most one per `gb_per_thread` GB of available RAM (the oracle holds ~1 GB per 128^3
    gradient, ~10 GB per 256^3 gradient)."""
    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        n = os.cpu_count() or 1
    try:
        avail = os.sysconf("SC_AVPHYS_PAGES") * os.sysconf("SC_PAGE_SIZE")
        n = min(n, max(1, int(avail / (gb_per_thread * 1e9))))
    except (ValueError, OSError):
        pass
    return max(1, min(n, cap))


# ------------------------------------------------------------------- workloads --
def make_workload(scale, nsrc_total, forward=None):
    from eikonalsolvers import configs as CF
    return CF.cfg3(scale=scale, nsrc=nsrc_total, forward=forward, nrec_side=20)


def flat_inputs(w, s0, s1):
    cs = np.ascontiguousarray(w.coordsrc[s0:s1], dtype=np.float64)
    recs = w.coordrec[s0:s1]
    off = np.zeros(len(recs) + 1, dtype=np.int64)
    for i, r in enumerate(recs):
        off[i + 1] = off[i] + r.shape[0]
    rec = np.ascontiguousarray(np.concatenate(recs), dtype=np.float64)
    po = np.ascontiguousarray(np.concatenate(w.pickobs[s0:s1]), dtype=np.float64)
    so = np.ascontiguousarray(np.concatenate(w.stdobs[s0:s1]), dtype=np.float64)
    return cs, off, rec, po, so


# ----------------------------------------------------------------- CPU leg (oracle) --
def cpu_sample(w, nthreads, nsrc):
    """Bounded CPU sample of the workload for the oracle: a 128^3 sub-block of the model
    (x, y nodes 64..191, z nodes 128..255: the lower half where the sources are) with the
    workload's sources mapped into it and a 20x20 receiver grid on its top face."""
    from eikonalsolvers import Grid3DCart
    n = w.grd.grsize[0]
    b = n // 2
    lo = np.array([n // 4, n // 4, n // 2])
    vel = np.ascontiguousarray(w.vel[lo[0]:lo[0] + b, lo[1]:lo[1] + b, lo[2]:lo[2] + b])
    h = w.grd.hgrid
    grd = Grid3DCart(hgrid=h, cooinit=(0.0, 0.0, 0.0), grsize=(b, b, b))
    ext = float(grd.x[-1])  # the grid's own last coordinate (Julia range arithmetic)
    src = []
    for s in range(nsrc):
        x, y, z = w.coordsrc[s % len(w.coordsrc)]
        full = (n - 1) * h
        src.append([0.05 * ext + 0.9 * ext * x / full, 0.05 * ext + 0.9 * ext * y / full,
                    min(max(z - lo[2] * h, 0.05 * ext), 0.95 * ext)])
    xr = np.linspace(0.0, ext, 20)
    rec = np.array([[a, c, 0.0] for c in xr for a in xr])
    return vel, grd, np.array(src), [rec.copy() for _ in range(nsrc)], (b / n) ** 3


def run_cpu_leg(w, steps, warmup, nthreads):
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import eikoracle as O
    from eikonalsolvers import ExtraParams
    nsrc = nthreads
    vel, grd, cs, rec, frac = cpu_sample(w, nthreads, nsrc)
    ep = ExtraParams(parallelkind="sharedmem")
    picks = O.eiktraveltime(vel * 1.02, grd, cs, rec, extraparams=ep, nthreads=nthreads)
    std = [0.01 * np.ones(p.shape) for p in picks]
    times = []
    for it in range(warmup + steps):
        t0 = time.perf_counter()
        O.eikgradient(vel, grd, cs, rec, picks, std, "gradvelandsrcloc", extraparams=ep, nthreads=nthreads)
        dt = time.perf_counter() - t0
        if it >= warmup:
            times.append(dt)
    t = sum(times) / len(times)
    value = nsrc / t * frac
    sample = (f"{nsrc} sources (one per thread) of the workload on a {grd.grsize[0]}^3 sub-block of its "
              f"model, gradvelandsrcloc, {t:.2f} s per call; source-solves/s scaled to 256^3 by node count "
              f"(x{frac:.4g})")
    return value, sample, t


def run_cpu_full(w, nthreads, ep):
    """The oracle on the benchmark workload itself (256^3): `nthreads` of its sources, one per
    thread (:sharedmem, one source per group), :gradvelandsrcloc, timed once. Returns the
    source-solves/s, a description, and the oracle's result with its inputs (the parity check
    runs the GPU on the same inputs)."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import eikoracle as O
    k = max(1, min(nthreads, len(w.coordsrc)))
    idx = list(range(k))
    cs = w.coordsrc[idx]
    rec = [w.coordrec[i] for i in idx]
    po = [w.pickobs[i] for i in idx]
    so = [w.stdobs[i] for i in idx]
    t0 = time.perf_counter()
    res = O.eikgradient(w.vel, w.grd, cs, rec, po, so, "gradvelandsrcloc", extraparams=ep, nthreads=k)
    t = time.perf_counter() - t0
    sample = (f"{k} sources of the {w.grd.grsize[0]}^3 workload itself, one per thread (:sharedmem), "
              f":gradvelandsrcloc, {t:.1f} s for the call")
    return k / t, sample, (cs, rec, po, so, k, res)


def rel_l2(a, b):
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))


def run_parity(ctx, mid, w, ep, full, sel=(0, 7, 15, 31)):
    """Parity of the benchmarked configuration against the oracle: the traveltime fields of
    sources `sel` of one batched call over all the workload's sources (the timed call's
    forward) bit for bit, and the gradient of the CPU leg's sources (same inputs, same
    :sharedmem groups) within the gradient tolerance."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import eikoracle as O
    from eikonalsolvers.tune import default_tuner
    sel = [s for s in sel if s < len(w.coordsrc)]
    default_tuner().apply_known(ctx, w.grd, len(w.coordsrc), ep)
    _, tt = ctx.traveltime(mid, w.grd, w.coordsrc, w.coordrec, returntt=True, extraparams=ep)
    _, ott = O.eiktraveltime(w.vel, w.grd, w.coordsrc[sel], [w.coordrec[i] for i in sel], returntt=True,
                             extraparams=ep, nthreads=len(sel))
    ndiff = [int((tt[s] != ott[k]).sum()) for k, s in enumerate(sel)]
    del tt, ott
    out = {"forward_sources_checked": sel, "forward_nodes_differing": ndiff,
           "forward_bitexact": all(n == 0 for n in ndiff)}
    if full is not None:
        cs, rec, po, so, k, ores = full
        from eikonalsolvers import ExtraParams
        epg = ExtraParams(parallelkind="sharedmem")
        default_tuner().apply_known(ctx, w.grd, k, epg)
        gv, gs, m = ctx.gradient(mid, w.grd, cs, rec, po, so, "gradvelandsrcloc", extraparams=epg, nthreads=k)
        out.update({"grad_sources": k, "gradvel_rel_l2": rel_l2(gv, ores[0]), "gradsrc_rel_l2": rel_l2(gs, ores[1]),
                    "misfit_rel": abs(m - ores[2]) / abs(ores[2]), "grad_tolerance": 1e-4})
    return out


# ----------------------------------------------------------------------- GPU arm --
def main_b200(args):
    import torch
    import torch.distributed as dist
    from eikonalsolvers import Context, ExtraParams
    from eikonalsolvers import _lib

    ws, rank, local = dist_env()
    if args.gpus > 1 and ws == 1:
        print(json.dumps({"error": "run --gpus N>1 under torch.distributed.run"}))
        return 2
    torch.cuda.set_device(local)
    if ws > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    dev = torch.device("cuda", local)
    if args.serve_sweep:
        if rank == 0:
            print(json.dumps(run_serve_sweep(args, local)), flush=True)
        return 0
    ctx = Context(local)
    L = ctx.L

    # ---- workload: every rank takes its own contiguous block of sources
    nsrc = args.nsrc
    w = make_workload(args.scale, nsrc * ws)
    s0, s1 = rank * nsrc, (rank + 1) * nsrc
    ep = ExtraParams()
    mid_obs = ctx.upload(w.vel_obs, w.grd)
    picks = ctx.traveltime(mid_obs, w.grd, w.coordsrc[s0:s1], w.coordrec[s0:s1], extraparams=ep)
    ctx.release(mid_obs)
    rng = np.random.default_rng(12 + rank)
    w.pickobs = [None] * (nsrc * ws)
    w.stdobs = [None] * (nsrc * ws)
    for i, p in enumerate(picks):
        w.pickobs[s0 + i] = p + rng.normal(0.0, 0.01, p.shape)
        w.stdobs[s0 + i] = 0.01 * np.ones(p.shape)
    mid = ctx.upload(w.vel, w.grd)
    # launch parameters of this workload class from the autotuner's table (no timing here)
    from eikonalsolvers.tune import default_tuner
    tuned = default_tuner().apply_known(ctx, w.grd, nsrc, ep)
    launch_params = ({"round_gate": tuned["round_gate"], "ctas_per_sm": tuned["ctas_per_sm"],
                      "source": "autotuner table shipped with the package"} if tuned else
                     {"round_gate": "by size", "ctas_per_sm": 0, "source": "library defaults"})
    N = int(np.prod(w.grd.grsize))
    nd = w.grd.ndim
    cs, off, rec, po, so = flat_inputs(w, s0, s1)
    d_cs = torch.from_numpy(cs).to(dev)
    d_rec = torch.from_numpy(rec).to(dev)
    d_po = torch.from_numpy(po).to(dev)
    d_so = torch.from_numpy(so).to(dev)
    d_gv = torch.empty(N, dtype=torch.float64, device=dev)
    d_gs = torch.empty(nsrc * nd, dtype=torch.float64, device=dev)
    d_m = torch.empty(1, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()
    epc = _lib.extra_struct(ep)
    stream = torch.cuda.ExternalStream(L.eik_ctx_stream(ctx.h), device=dev)
    P = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731

    def step(st):
        rc = L.eik_gradient_device(ctx.h, C.c_int64(mid), nsrc, P(d_cs), _lib.ptr(off), P(d_rec), P(d_po),
                                   P(d_so), 3, C.byref(epc), P(d_gv), P(d_gs), P(d_m), C.byref(st))
        _lib.check(rc, ctx.h)
        if ws > 1:  # the gradient of the whole job is the sum over the ranks' sources
            with torch.cuda.stream(stream):
                dist.all_reduce(d_gv)
                dist.all_reduce(d_m)

    st = _lib.eik_stats()
    for i in range(args.warmup):
        t0 = time.perf_counter()
        step(st)
        log(f"warmup step {i}: {time.perf_counter() - t0:.2f} s (fine {st.fine_ms:.0f} ms, solve {st.solve_ms:.0f} ms, "
            f"adjoint {st.adj_ms:.0f} ms, device {st.device_ms:.0f} ms)")
    # ---- timed region (device-resident inputs)
    fine_ms = solve_ms = adj_ms = 0.0
    launches = 0
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with Clocks(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            step(st)
            fine_ms += st.fine_ms
            solve_ms += st.solve_ms
            adj_ms += st.adj_ms
            launches += st.launches
        e1.record(stream)
        torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    t = torch.tensor([ms], dtype=torch.float64, device=dev)
    if ws > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = nsrc * ws * args.steps / (ms_max / 1000.0)
    clocks = clk.summary()

    # ---- end to end through the host C-ABI entry point, pinned host buffers
    h_cs, h_off, h_rec, h_po, h_so = (torch.from_numpy(a).pin_memory() for a in (cs, off, rec, po, so))
    h_gv = torch.empty(N, dtype=torch.float64).pin_memory()
    h_gs = torch.empty(nsrc * nd, dtype=torch.float64).pin_memory()
    h_m = C.c_double()
    st2 = _lib.eik_stats()
    Ph = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    if ws > 1:
        dist.barrier()
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(args.e2e_steps):
        rc = L.eik_gradient(ctx.h, C.c_int64(mid), nsrc, Ph(h_cs), Ph(h_off), Ph(h_rec), Ph(h_po), Ph(h_so), 3,
                            C.byref(epc), Ph(h_gv), Ph(h_gs), C.byref(h_m), C.byref(st2))
        _lib.check(rc, ctx.h)
    f1.record(stream)
    torch.cuda.synchronize()
    t = torch.tensor([f0.elapsed_time(f1)], dtype=torch.float64, device=dev)
    if ws > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e = nsrc * ws * args.e2e_steps / (float(t.item()) / 1000.0)
    h2d = cs.nbytes + off.nbytes + rec.nbytes + po.nbytes + so.nbytes
    d2h = N * 8 + nsrc * nd * 8 + 8

    # ---- plain path: one source per call
    plain = None
    if args.plain_sources > 0:
        npl = min(args.plain_sources, nsrc)
        if not default_tuner().apply_known(ctx, w.grd, 1, ep):
            ctx.set_param("round_gate", 0.0)  # the library's choice by size
            ctx.set_param("ctas_per_sm", 0)
        stp = _lib.eik_stats()
        offs = [np.array([0, off[i + 1] - off[i]], dtype=np.int64) for i in range(npl)]
        if ws > 1:
            dist.barrier()
        torch.cuda.synchronize()
        g0 = torch.cuda.Event(enable_timing=True)
        g1 = torch.cuda.Event(enable_timing=True)
        g0.record(stream)
        for i in range(npl):
            r0 = int(off[i])
            rc = L.eik_gradient_device(ctx.h, C.c_int64(mid), 1, C.c_void_p(d_cs.data_ptr() + 8 * nd * i),
                                       _lib.ptr(offs[i]), C.c_void_p(d_rec.data_ptr() + 8 * nd * r0),
                                       C.c_void_p(d_po.data_ptr() + 8 * r0), C.c_void_p(d_so.data_ptr() + 8 * r0),
                                       3, C.byref(epc), P(d_gv), C.c_void_p(d_gs.data_ptr() + 8 * nd * i), P(d_m),
                                       C.byref(stp))
            _lib.check(rc, ctx.h)
        g1.record(stream)
        torch.cuda.synchronize()
        t = torch.tensor([g0.elapsed_time(g1)], dtype=torch.float64, device=dev)
        if ws > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        pv = npl * ws / (float(t.item()) / 1000.0)
        plain = {"value": pv, "unit": UNIT, "sources_timed_per_rank": npl, "batched_over_plain": value / pv}

    # ---- roofline of the dominant kernel (measured inside the timed region)
    peak, peak_kind = measured_peaks()
    kern = {"coarse_rounds_kernel": (solve_ms, 16), "adj_rounds_kernel": (adj_ms, 16),
            "fine_fmm_kernel": (fine_ms, 16)}
    top = max(kern, key=lambda k: kern[k][0])
    kms, bpn = kern[top]
    per_launch_ms = kms / args.steps
    alg_bytes = bpn * N * nsrc  # per launch: one launch serves all the rank's sources
    achieved = alg_bytes / (per_launch_ms / 1000.0) / 1e9
    traffic_ss = profile_traffic(top)
    roof = {"kernel": top, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "peak_kind": peak_kind,
            "traffic": (traffic_ss * N * nsrc if traffic_ss is not None else None),
            "traffic_note": "DRAM bytes per launch: the per-node-solve figure of profiles/<kernel>.md (ncu, "
                            "256^3 x 1 source, same launch parameters) times the node-solves of this launch",
            "algorithmic_bytes_per_launch": alg_bytes, "avg_launch_ms": per_launch_ms,
            "share_of_step": kms / ms,
            "kernel_ms_per_step": {k: v[0] / args.steps for k, v in kern.items()}}

    # ---- CPU baseline (rank 0, N=1 only): the workload itself, and the 128^3 sub-block sample
    cpu = None
    full = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cores = host_cores(cap=32, gb_per_thread=10.0 * (args.scale ** 3))
        try:
            vf, samplef, full = run_cpu_full(w, cores, ExtraParams(parallelkind="sharedmem"))
            cpu = {"value": vf, "unit": UNIT, "cores": full[4], "kind": "port", "sample": samplef}
        except Exception as e:  # the GPU line is still worth printing
            cpu = {"value": None, "unit": UNIT, "cores": cores, "kind": "port", "error": str(e)}
        try:
            cores_s = host_cores()
            v, sample, _ = run_cpu_leg(w, steps=1, warmup=0, nthreads=cores_s)
            cpu["subblock_sample"] = {"value": v, "cores": cores_s, "sample": sample}
        except Exception as e:
            cpu["subblock_sample"] = {"error": str(e)}
    parity = None
    if rank == 0 and ws == 1 and not args.no_parity:
        try:
            parity = run_parity(ctx, mid, w, ep, full)
        except Exception as e:
            parity = {"error": str(e)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": f"3D Cartesian eikgradient :gradvelandsrcloc, {w.grd.grsize[0]}^3, "
                                   f"hgrid {w.grd.hgrid}, 4-layer model, {nsrc} sources per GPU, 400 receivers, "
                                   "default ExtraParams (refined start-up ds=5 r=3, smoothing radius 3)",
                       "sources_per_gpu": nsrc, "nodes": N, "parallelism": f"sources sharded over {ws} GPU(s)",
                       "l2": "inputs and per-source fields far larger than L2 (no flush)",
                       "launch_params": launch_params},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                    "steps": args.e2e_steps},
            "plain": plain,
            "roofline": roof,
            "cpu_baseline": cpu,
            "parity": parity,
            "clocks": clocks,
            "gpu_launches": int(launches),
            "serve": None,
            "stats": {"tile_activations": int(st.tile_activations), "node_evals": int(st.node_evals),
                      "adj_rounds": int(st.adj_rounds), "fwd_rounds": int(st.fwd_rounds), "evals_per_node": st.node_evals / (N * nsrc)},
        }
    ctx.release(mid)
    ctx.close()
    if rank == 0:
        if ws == 1 and args.serve_requests > 0:
            try:
                line["serve"] = run_serve_leg(args, local)
            except Exception as e:
                line["serve"] = {"error": str(e)}
        if ws == 1 and args.hmc_evals > 0:
            try:
                line["hmc"] = run_hmc_leg(args, local)
            except Exception as e:
                line["hmc"] = {"error": str(e)}
        if ws == 1 and args.ray_sources > 0:
            try:
                line["rays"] = run_rays_leg(args, local)
            except Exception as e:
                line["rays"] = {"error": str(e)}
        if ws == 1 and not args.no_configs:
            try:
                line["configs"] = run_configs_leg(args, local)
            except Exception as e:
                line["configs"] = {"error": str(e)}
        print(json.dumps(line), flush=True)
    if ws > 1:
        dist.destroy_process_group()
    return 0


def run_rays_leg(args, device):
    """Ray tracing (tracerays) on the 3D layered workload at 128^3: every receiver of
    `ray_sources` sources, steplen 0.01 (the reference's default). GPU rays/s through
    eik_tracerays with the traveltime grids and the rays in host memory (copies timed), beside
    the oracle on the host cores for a sample of the same rays."""
    from eikonalsolvers import Context, ExtraParams, tracerays
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import eikoracle as O
    w = make_workload(0.5, args.ray_sources)
    ctx = Context(device)
    try:
        mid = ctx.upload(w.vel, w.grd)
        _, tt = ctx.traveltime(mid, w.grd, w.coordsrc, w.coordrec, returntt=True, extraparams=ExtraParams())
        ctx.release(mid)
        tracerays(w.grd, tt, w.coordsrc, w.coordrec, steplen=0.01, ctx=ctx)  # warm-up (scratch growth)
        ms = []
        for _ in range(3):
            rays = tracerays(w.grd, tt, w.coordsrc, w.coordrec, steplen=0.01, ctx=ctx)
            ms.append(float(ctx.last_stats.device_ms))
    finally:
        ctx.close()
    nray = sum(len(r) for r in rays)
    npts = sum(x.shape[0] for r in rays for x in r)
    gpu_ms = min(ms)
    # oracle: one source's spline and its first rays, single thread
    k = max(1, min(args.ray_cpu_rays, len(w.coordrec[0])))
    t0 = time.perf_counter()
    ora = O.tracerays(w.grd, tt[:1], w.coordsrc[:1], [w.coordrec[0][:k]], steplen=0.01)
    cpu_s = time.perf_counter() - t0
    cpu_pts = sum(x.shape[0] for x in ora[0])
    same = all(np.array_equal(a, b) for a, b in zip(ora[0], rays[0][:k]))
    return {"workload": f"3D layered 128^3, {args.ray_sources} sources x 400 receivers, steplen 0.01",
            "rays": nray, "points": npts, "gpu_ms": gpu_ms, "rays_per_s": nray / (gpu_ms / 1000.0),
            "points_per_s": npts / (gpu_ms / 1000.0),
            "gpu_timing": "eik_tracerays device time incl. the grids' upload and the paths' download, best of 3",
            "cpu_baseline": {"rays_per_s": k / cpu_s, "points_per_s": cpu_pts / cpu_s, "cores": 1, "kind": "port",
                             "sample": f"{k} rays of source 0 (spline of that source included)"},
            "bit_identical_to_oracle_on_sample": bool(same)}


def run_hmc_leg(args, device):
    """HMC-style evaluations (the pattern of HMCtraveltimes.jl: eikgradient model after model
    with the same sources and receivers) on the 2D Cartesian 300x220 grid of the reference's
    CPU example, 4 sources x 10 receivers, a new velocity every evaluation: eik_gradient
    (upload + call) against a captured plan replayed with the new velocity (eik_plan_run).
    Host clock per evaluation, results checked identical."""
    from eikonalsolvers import Context, Grid2DCart
    g = Grid2DCart(hgrid=0.5, cooinit=(0.0, 0.0), grsize=(300, 220))
    j = np.arange(1, 221)[None, :]
    base = np.ascontiguousarray(np.broadcast_to(2.5 + 0.034 * j, g.grsize), dtype=np.float64)
    cs = np.column_stack([0.5 * np.linspace(10, 290, 4), np.full(4, 100.0)])
    rec = [np.column_stack([0.5 * np.linspace(8, 294, 10), np.full(10, 10.0)])] * 4
    rng = np.random.default_rng(3)
    vels = [base * (1.0 + 0.01 * rng.standard_normal(g.grsize)) for _ in range(args.hmc_evals + 2)]
    ctx = Context(device)
    try:
        mid = ctx.upload(base, g)
        pobs = ctx.traveltime(mid, g, cs, rec)
        sobs = [0.01 * np.ones(p.shape) for p in pobs]
        # plain calls: upload the new model, one eik_gradient, release
        t_plain, ref = [], []
        for v in vels:
            t0 = time.perf_counter()
            m = ctx.upload(v, g)
            ref.append(ctx.gradient(m, g, cs, rec, pobs, sobs, "gradvel"))
            ctx.release(m)
            t_plain.append(time.perf_counter() - t0)
        plan = ctx.plan_gradient(mid, g, cs, rec, "gradvel")
        t_plan, same = [], True
        try:
            for v, want in zip(vels, ref):
                t0 = time.perf_counter()
                got = plan.run(pobs, sobs, vel=v)
                t_plan.append(time.perf_counter() - t0)
                same = same and np.array_equal(got[0], want[0]) and got[1] == want[1]
        finally:
            plan.close()
        ctx.release(mid)
    finally:
        ctx.close()
    med = lambda x: float(np.median(x[2:])) * 1e3  # noqa: E731  (first two evaluations are warm-up)
    return {"workload": "2D Cartesian 300x220, 4 sources x 10 receivers, :gradvel, new velocity per evaluation",
            "evaluations": args.hmc_evals, "eik_gradient_ms": med(t_plain), "plan_run_ms": med(t_plan),
            "plan_speedup": med(t_plain) / med(t_plan), "identical_results": bool(same),
            "timing": "host clock per evaluation (median), velocity upload included"}


def run_serve_leg(args, device, rate=None, n=None, max_queue=0):
    """Serving mix (2D/3D Cartesian models resident on the device, 70 % traveltime / 30 %
    gradient requests with 1-64 sources) arriving as a Poisson process; latency from
    submission to result, on the host clock. A server with max_queue > 0 refuses arrivals
    while that many requests wait (counted in `refused`)."""
    from eikonalsolvers import configs as CF
    from eikonalsolvers.serve import Request, Server
    rate = args.serve_rate if rate is None else rate
    n = args.serve_requests if n is None else n
    models, reqs = CF.serving_requests(n=n, rate=rate, seed=9, scale=args.serve_scale)
    # server-wide admission: merged calls in flight together within 150 GB of device memory
    with Server(device=device, slots=args.serve_slots, max_batch_sources=args.serve_batch_sources,
                hbm_budget=150 * 10 ** 9, hbm_budget_per_slot=int(160e9 / args.serve_slots),
                max_queue=max_queue) as srv:
        for k, (vel, grd, _) in models.items():
            srv.register_model(k, vel, grd)
        # warm each slot on every model (uploads, scratch growth) before the clock starts
        centre = lambda g: np.array([[0.5 * (g.grsize[d] - 1) * g.spacing[d] + 1e-3 for d in range(g.ndim)]])  # noqa: E731
        warm = [srv.submit(Request(model=k, kind="traveltime", coordsrc=centre(g), coordrec=[np.zeros((1, g.ndim))]))
                for k, (v, g, _) in models.items() for _ in range(args.serve_slots)]
        for f in warm:
            f.result()
        srv._done.clear()
        t0 = time.perf_counter()
        futs = []
        for r in reqs:
            delay = t0 + r["t"] - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            futs.append(srv.submit(Request(model=r["model"], kind=r["kind"], coordsrc=r["coordsrc"],
                                           coordrec=r["coordrec"], pickobs=r.get("pickobs"),
                                           stdobs=r.get("stdobs"))))
        t_arrivals = time.perf_counter() - t0
        failed = 0
        for f in futs:
            try:
                f.result()
            except Exception as e:
                if type(e).__name__ != "ServerOverloaded":
                    failed += 1
        st = srv.stats()
    st.update({"offered_rate_req_s": rate, "offered_requests": n, "arrival_window_s": t_arrivals,
               "failed": failed, "slots": args.serve_slots, "max_queue": max_queue,
               "max_batch_sources": args.serve_batch_sources,
               "mix": "seeded: 60% 2D side 128-1024, 40% 3D side 64-192 (x serve-scale), 1-64 sources, 70% "
                      "traveltime / 30% gradvel, 6 resident models"})
    return st


def run_serve_sweep(args, device):
    rates = [float(x) for x in args.serve_sweep.split(",") if x.strip()]
    out = []
    for rate in rates:
        n = int(min(2000, round(60.0 * rate)))
        st = run_serve_leg(args, device, rate=rate, n=n, max_queue=args.serve_max_queue)
        log(f"serve rate {rate}: {json.dumps(st)}")
        out.append(st)
    served = [(r["offered_rate_req_s"], r.get("requests_per_s") or 0.0) for r in out]
    # saturation: the first rate whose served rate falls below 90 % of the offered one
    sat = next((o for o, v in served if v < 0.9 * o), None)
    return {"serve_sweep": out, "saturation_offered_rate_req_s": sat,
            "served_rate_at_saturation_req_s": max(v for _, v in served) if served else None}


def _obs(ctx, w, vel, sigma, seed):
    mid = ctx.upload(vel, w.grd)
    try:
        picks = ctx.traveltime(mid, w.grd, w.coordsrc, w.coordrec)
    finally:
        ctx.release(mid)
    rng = np.random.default_rng(seed)
    return [p + rng.normal(0.0, sigma, p.shape) for p in picks], [sigma * np.ones(p.shape) for p in picks]


def _gpu_timed(fn, reps):
    fn()  # warm-up: scratch growth, first-call set-up
    ts = []
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        ts.append(time.perf_counter() - t0)
    return float(np.median(ts))


def run_configs_leg(args, device):
    """The other benchmark configurations, each end to end through the host C-ABI entry point
    (inputs and results in host memory, copies inside the host-clock timing) beside the oracle
    on the host cores, with the roofline of the dominant kernel of the call; and the batched
    call against one source per call at several grid sizes."""
    from eikonalsolvers import Context, ExtraParams
    from eikonalsolvers import configs as CF
    from eikonalsolvers.tune import default_tuner
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import eikoracle as O
    peak, peak_kind = measured_peaks()
    cores = host_cores()
    out = {}
    ctx = Context(device)
    try:
        def leg(name, w, kind, ncpu, cpu_ep, desc):
            nsrc = len(w.coordsrc)
            N = int(np.prod(w.grd.grsize))
            ep = ExtraParams()
            if not default_tuner().apply_known(ctx, w.grd, nsrc, ep):
                ctx.set_param("round_gate", 0.0)
                ctx.set_param("ctas_per_sm", 0)
            mid = ctx.upload(w.vel, w.grd)
            try:
                if kind == "traveltime":
                    call = lambda: ctx.traveltime(mid, w.grd, w.coordsrc, w.coordrec, returntt=True, extraparams=ep)  # noqa: E731
                else:
                    call = lambda: ctx.gradient(mid, w.grd, w.coordsrc, w.coordrec, w.pickobs, w.stdobs, "gradvel",  # noqa: E731
                                                extraparams=ep)
                t = _gpu_timed(call, reps=3)
                st = ctx.last_stats
            finally:
                ctx.release(mid)
            k = max(1, min(ncpu, nsrc))
            t0 = time.perf_counter()
            if kind == "traveltime":
                O.eiktraveltime(w.vel, w.grd, w.coordsrc[:k], w.coordrec[:k], returntt=True, extraparams=cpu_ep,
                                nthreads=min(k, cores))
            else:
                O.eikgradient(w.vel, w.grd, w.coordsrc[:k], w.coordrec[:k], w.pickobs[:k], w.stdobs[:k], "gradvel",
                              extraparams=cpu_ep, nthreads=min(k, cores))
            tc = time.perf_counter() - t0
            kern = {"coarse_rounds_kernel": float(st.solve_ms), "adj_rounds_kernel": float(st.adj_ms)}
            top = max(kern, key=kern.get)
            alg = 16 * N * nsrc
            achieved = alg / (kern[top] / 1000.0) / 1e9 if kern[top] > 0 else None
            out[name] = {"workload": desc, "gpu_e2e": {"value": nsrc / t, "unit": UNIT, "ms_per_call": t * 1e3,
                                                       "device_ms": float(st.device_ms)},
                         "cpu_baseline": {"value": k / tc, "unit": UNIT, "cores": min(k, cores), "kind": "port",
                                          "sample": f"{k} of the sources, one per thread"},
                         "gpu_over_cpu": (nsrc / t) / (k / tc),
                         "roofline": {"kernel": top, "bound": "hbm", "achieved": achieved, "peak": peak,
                                      "unit": "GB/s", "frac": achieved / peak if achieved else None,
                                      "peak_kind": peak_kind, "algorithmic_bytes_per_launch": alg,
                                      "avg_launch_ms": kern[top]},
                         "fwd_rounds": int(st.fwd_rounds)}
            log(f"config {name}: GPU {nsrc / t:.1f} src/s, CPU {k / tc:.2f} src/s")

        w1 = CF.cfg1()
        leg("cfg1", w1, "traveltime", 4, ExtraParams(parallelkind="sharedmem"),
            "2D Cartesian 300x220 h=0.5, v=2.5+0.034j, 4 sources x 10 receivers, eiktraveltime + returntt")
        w2 = CF.cfg2()
        w2.pickobs, w2.stdobs = _obs(ctx, w2, w2.vel_obs, 0.01, 11)
        leg("cfg2", w2, "gradient", cores, ExtraParams(parallelkind="sharedmem"),
            "2D Cartesian 1024x640 h=0.25, correlated random field 2-5, 64 sources x 200 receivers, :gradvel")
        w4 = CF.cfg4()
        w4.pickobs, w4.stdobs = _obs(ctx, w4, w4.vel, 0.05, 13)
        leg("cfg4", w4, "gradient", cores, ExtraParams(parallelkind="sharedmem"),
            "Grid3DSphere 200x180x180, r 5771-6371 km, 20x20 deg, 1D profile + 3% correlated, 48 sources x 500 "
            "receivers, :gradvel")
        # batched vs one source per call at several sizes (device-resident work, host clock)
        bp = {}
        for name, w, which, kplain in (("3D 64^3 x32", CF.cfg3(scale=0.25, nsrc=32), "gradvelandsrcloc", 4),
                                       ("3D 128^3 x16", CF.cfg3(scale=0.5, nsrc=16), "gradvelandsrcloc", 2),
                                       ("2D 512x320 x64", CF.cfg2(scale=0.5, nsrc=64), "gradvel", 4)):
            nsrc = len(w.coordsrc)
            w.pickobs, w.stdobs = _obs(ctx, w, w.vel * 1.03, 0.01, 5)
            ep = ExtraParams()
            mid = ctx.upload(w.vel, w.grd)
            try:
                def batched():
                    if not default_tuner().apply_known(ctx, w.grd, nsrc, ep):
                        ctx.set_param("round_gate", 0.0)
                        ctx.set_param("ctas_per_sm", 0)
                    ctx.gradient(mid, w.grd, w.coordsrc, w.coordrec, w.pickobs, w.stdobs, which, extraparams=ep)

                def plain():
                    if not default_tuner().apply_known(ctx, w.grd, 1, ep):
                        ctx.set_param("round_gate", 0.0)
                        ctx.set_param("ctas_per_sm", 0)
                    for s in range(kplain):
                        ctx.gradient(mid, w.grd, w.coordsrc[s:s + 1], w.coordrec[s:s + 1], w.pickobs[s:s + 1],
                                     w.stdobs[s:s + 1], which, extraparams=ep)
                tb = _gpu_timed(batched, reps=2)
                tp = _gpu_timed(plain, reps=1)
            finally:
                ctx.release(mid)
            bp[name] = {"batched": nsrc / tb, "plain": kplain / tp, "batched_over_plain": (nsrc / tb) / (kplain / tp),
                        "unit": UNIT}
            log(f"batched/plain {name}: {bp[name]['batched_over_plain']:.2f}")
        out["batched_over_plain_by_size"] = bp
    finally:
        ctx.close()
    return out


def main_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    cores = host_cores()
    w = make_workload(args.scale, args.nsrc)
    v, sample, t_step = run_cpu_leg(w, steps=args.steps, warmup=args.warmup, nthreads=cores)
    # beside the bounded per-step sample: one call on the workload itself (one source per
    # thread), with observations from straight rays at the model's mean velocity (the cost of
    # the gradient does not depend on the observed values)
    full = None
    if not args.no_cpu:
        from eikonalsolvers import ExtraParams
        try:
            vm = float(np.mean(w.vel))
            w.pickobs = [np.linalg.norm(r - c[None, :], axis=1) / vm for c, r in zip(w.coordsrc, w.coordrec)]
            w.stdobs = [0.01 * np.ones(p.shape) for p in w.pickobs]
            fv, fsample, res = run_cpu_full(w, host_cores(cap=32, gb_per_thread=10.0 * (args.scale ** 3)),
                                            ExtraParams(parallelkind="sharedmem"))
            full = {"value": fv, "unit": UNIT, "cores": res[4], "kind": "port", "sample": fsample}
        except Exception as e:
            full = {"error": str(e)}
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": f"3D Cartesian eikgradient :gradvelandsrcloc, {w.grd.grsize[0]}^3, "
                                   f"hgrid {w.grd.hgrid}, 4-layer model, {args.nsrc} sources per GPU, 400 receivers, "
                                   "default ExtraParams (refined start-up ds=5 r=3, smoothing radius 3)",
                       "sources_per_gpu": args.nsrc, "nodes": int(np.prod(w.grd.grsize)),
                       "implementation": "oracle (C++ restatement of the reference FMM + CSR adjoint), "
                                         "threaded by source groups as :sharedmem; each step a bounded sample "
                                         "of the workload (see cpu_baseline.sample)"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample,
                             "full_workload": full},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    a = parse()
    sys.exit(main_reference(a) if a.impl == "reference" else main_b200(a))
