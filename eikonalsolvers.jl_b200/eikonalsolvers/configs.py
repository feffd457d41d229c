"""Seeded synthetic workloads with the shapes, sizes and value distributions of the
five benchmark configurations (no public dataset exists for this path; every input is
generated here from fixed seeds).

* cfg1: Grid2DCart h=0.5, 300x220, v = 2.5 + 0.034*j, 4 sources, 10 receivers each,
  eiktraveltime with returntt.
* cfg2: Grid2DCart h=0.25, 1024x640, Gaussian-correlated random field (correlation
  length 20 cells) mapped to (2, 5); 64 sources at depth cells 100-150; 200 receivers on
  the top row; observed picks from a +-5% perturbed model plus N(0, 0.01^2) noise.
* cfg3: Grid3DCart h=0.1, 256^3, 4 layers (3.0/4.2/5.5/6.8) with seeded sinusoidal
  interfaces of amplitude 8 cells plus 2% white perturbation; 32 sources in the lower half;
  400 receivers on a 20x20 surface grid; observations as in cfg2.
* cfg4: Grid3DSphere 200x180x180, r in [5771, 6371] km, theta/phi in [80, 100] deg;
  v(r) = 5.8 + 2.2*(6371-r)/600 times (1 + 0.03*g), g correlated over 15 km; 48 sources at
  10-400 km depth; 500 random surface receivers; observation noise N(0, 0.05^2).
* cfg5: serving mix (see ``serving_requests``).

``scale`` shrinks a configuration's grid (and source count) for tests; the benchmark
always uses scale=1.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from .structs import ExtraParams, Grid2DCart, Grid3DCart, Grid3DSphere


@dataclass
class Workload:
    name: str
    grd: object
    vel: np.ndarray
    coordsrc: np.ndarray
    coordrec: List[np.ndarray]
    extraparams: ExtraParams
    pickobs: Optional[List[np.ndarray]] = None
    stdobs: Optional[List[np.ndarray]] = None
    vel_obs: Optional[np.ndarray] = None      # model the observations were generated from
    meta: dict = field(default_factory=dict)


def _linrange(a, b, n):
    return np.array([(1 - i / (n - 1)) * a + (i / (n - 1)) * b for i in range(n)])


def gaussian_random_field(shape, corr_cells, seed):
    """White noise (seeded) filtered by a Gaussian of sigma=corr_cells (FFT, periodic),
    standardised to zero mean and unit variance."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal(shape)
    F = np.fft.fftn(w)
    kern = np.ones(shape)
    for d, n in enumerate(shape):
        sig = corr_cells[d] if np.ndim(corr_cells) else corr_cells
        k = np.fft.fftfreq(n)
        g = np.exp(-2.0 * (math.pi * sig * k) ** 2)
        sh = [1] * len(shape)
        sh[d] = n
        kern = kern * g.reshape(sh)
    f = np.real(np.fft.ifftn(F * kern))
    f = (f - f.mean()) / f.std()
    return f


def _normal_cdf(z):
    from scipy.special import ndtr
    return ndtr(z)


def cfg1() -> Workload:
    n1, n2 = 300, 220
    grd = Grid2DCart(hgrid=0.5, cooinit=(0.0, 0.0), grsize=(n1, n2))
    j = np.arange(1, n2 + 1)
    vel = np.broadcast_to(2.5 + 0.034 * j, (n1, n2)).copy()
    xs = 0.5 * _linrange(10, 290, 4)
    coordsrc = np.column_stack([xs, 100.0 * np.ones(4)])
    xr = 0.5 * _linrange(8, 294, 10)
    rec = np.column_stack([xr, 10.0 * np.ones(10)])
    return Workload("cfg1", grd, vel, coordsrc, [rec.copy() for _ in range(4)], ExtraParams(),
                    meta=dict(returntt=True))


def _observations(vel_true, grd, coordsrc, coordrec, extraparams, sigma, seed, forward):
    picks = forward(vel_true, grd, coordsrc, coordrec, extraparams)
    rng = np.random.default_rng(seed)
    pickobs = [p + rng.normal(0.0, sigma, p.shape) for p in picks]
    stdobs = [sigma * np.ones(p.shape) for p in picks]
    return pickobs, stdobs


def _avoid_node_and_half(x, h, rng_u):
    """Nudge a coordinate away from a node or a half-spacing (within 1e-6*h)."""
    r = math.fmod(x, h)
    for bad in (0.0, 0.5 * h, h):
        if abs(r - bad) <= 1e-6 * h:
            x += 3e-6 * h
    return x


def cfg2(scale: float = 1.0, nsrc: int = 64, forward=None) -> Workload:
    n1, n2 = int(1024 * scale), int(640 * scale)
    h = 0.25
    grd = Grid2DCart(hgrid=h, cooinit=(0.0, 0.0), grsize=(n1, n2))
    f = gaussian_random_field((n1, n2), 20.0 * scale if scale < 1 else 20.0, seed=2)
    vel = 2.0 + 3.0 * _normal_cdf(f)
    rng = np.random.default_rng(3)
    x0, x1 = grd.x[0], grd.x[-1]
    zlo, zhi = 100 * scale * h, 150 * scale * h
    cs = []
    for s in range(nsrc):
        x = rng.uniform(x0 + 5 * h, x1 - 5 * h)
        z = rng.uniform(zlo, zhi)
        cs.append([_avoid_node_and_half(x, h, rng), _avoid_node_and_half(z, h, rng)])
    coordsrc = np.array(cs)
    nrec = 200
    rec = np.column_stack([_linrange(x0, x1, nrec), np.zeros(nrec)])
    coordrec = [rec.copy() for _ in range(nsrc)]
    g = gaussian_random_field((n1, n2), 20.0 * scale if scale < 1 else 20.0, seed=4)
    g = g / np.abs(g).max()
    vel_obs = vel * (1.0 + 0.05 * g)
    w = Workload("cfg2", grd, vel, coordsrc, coordrec, ExtraParams(), vel_obs=vel_obs)
    if forward is not None:
        w.pickobs, w.stdobs = _observations(vel_obs, grd, coordsrc, coordrec, w.extraparams, 0.01, 11, forward)
    return w


def layered_3d(n, seed=5):
    """4 layers separated by sinusoidal interfaces (amplitude 8 cells) plus 2% white noise."""
    rng = np.random.default_rng(seed)
    n1, n2, n3 = n
    X = np.arange(n1)[:, None]
    Y = np.arange(n2)[None, :]
    L = float(max(n1, n2))
    amp = 8.0 * n3 / 256.0
    depths = [n3 * 64 / 256, n3 * 128 / 256, n3 * 192 / 256]
    surfs = []
    for d in depths:
        a, b = rng.integers(1, 4, size=2)
        p1, p2 = rng.uniform(0, 2 * math.pi, size=2)
        surfs.append(d + amp * np.sin(2 * math.pi * a * X / L + p1) * np.sin(2 * math.pi * b * Y / L + p2))
    Z = np.arange(n3)[None, None, :]
    vlay = np.array([3.0, 4.2, 5.5, 6.8])
    idx = np.zeros(n, dtype=np.int64)
    for s in surfs:
        idx += (Z >= s[:, :, None]).astype(np.int64)
    vel = vlay[idx]
    vel = vel * (1.0 + 0.02 * rng.standard_normal(n))
    return vel


def cfg3(scale: float = 1.0, nsrc: int = 32, forward=None, nrec_side: int = 20) -> Workload:
    n = int(256 * scale)
    h = 0.1
    grd = Grid3DCart(hgrid=h, cooinit=(0.0, 0.0, 0.0), grsize=(n, n, n))
    vel = layered_3d((n, n, n), seed=5)
    rng = np.random.default_rng(6)
    x0, x1 = grd.x[0], grd.x[-1]
    cs = []
    for s in range(nsrc):
        x = rng.uniform(x0 + 5 * h, x1 - 5 * h)
        y = rng.uniform(x0 + 5 * h, x1 - 5 * h)
        z = rng.uniform(0.5 * x1, x1 - 5 * h)
        cs.append([_avoid_node_and_half(v, h, rng) for v in (x, y, z)])
    coordsrc = np.array(cs)
    xr = _linrange(x0, x1, nrec_side)
    rec = np.array([[xr[i], xr[j], 0.0] for j in range(nrec_side) for i in range(nrec_side)])
    coordrec = [rec.copy() for _ in range(nsrc)]
    rng2 = np.random.default_rng(7)
    g = 0.05 * np.clip(rng2.standard_normal((n, n, n)), -1, 1)
    vel_obs = vel * (1.0 + g)
    w = Workload("cfg3", grd, vel, coordsrc, coordrec, ExtraParams(), vel_obs=vel_obs)
    if forward is not None:
        w.pickobs, w.stdobs = _observations(vel_obs, grd, coordsrc, coordrec, w.extraparams, 0.01, 12, forward)
    return w


def cfg4(scale: float = 1.0, nsrc: int = 48, forward=None) -> Workload:
    nr, nt, npf = int(200 * scale), int(180 * scale), int(180 * scale)
    r0, r1 = 5771.0, 6371.0
    dr = (r1 - r0) / (nr - 1)
    dth = 20.0 / (nt - 1)
    dph = 20.0 / (npf - 1)
    grd = Grid3DSphere(Δr=dr, Δθ=dth, Δφ=dph, cooinit=(r0, 80.0, 80.0), grsize=(nr, nt, npf))
    r = np.array(grd.r)[:, None, None]
    v1d = 5.8 + 2.2 * (6371.0 - r) / 600.0
    arc = 6371.0 * math.radians(dth)
    g = gaussian_random_field((nr, nt, npf), (15.0 / dr, 15.0 / arc, 15.0 / arc), seed=7)
    vel = np.broadcast_to(v1d, (nr, nt, npf)) * (1.0 + 0.03 * g)
    rng = np.random.default_rng(8)
    cs = []
    for s in range(nsrc):
        depth = rng.uniform(10.0, min(400.0, r1 - r0 - 5 * dr))
        cs.append([r1 - depth, rng.uniform(80.0 + 5 * dth, 100.0 - 5 * dth),
                   rng.uniform(80.0 + 5 * dph, 100.0 - 5 * dph)])
    coordsrc = np.array(cs)
    nrec = 500
    rec = np.column_stack([np.full(nrec, r1), rng.uniform(80.0, 100.0, nrec), rng.uniform(80.0, 100.0, nrec)])
    coordrec = [rec.copy() for _ in range(nsrc)]
    w = Workload("cfg4", grd, np.ascontiguousarray(vel), coordsrc, coordrec, ExtraParams())
    if forward is not None:
        w.pickobs, w.stdobs = _observations(vel, grd, coordsrc, coordrec, w.extraparams, 0.05, 13, forward)
    return w


def serving_requests(n: int, rate: float, seed: int = 9, scale: float = 1.0, nmodels: int = 6,
                     max_sources: int = 64):
    """The serving mix: `n` requests with Poisson arrivals at `rate` per second over a pool
    of `nmodels` resident models. 60 % 2D Cartesian (side U[128, 1024] nodes), 40 % 3D
    Cartesian (side U[64, 192]); velocity a linear gradient (cfg1 style) or a correlated
    random field (cfg2 style), half each; nsrc ~ U{1..max_sources}; 70 % eiktraveltime, 30 %
    eikgradient :gradvel with observations from a 3 %-faster model plus N(0, 0.01^2).
    `scale` shrinks the sides (tests). Returns (models, requests): models maps a key to
    (vel, grd, vel_obs); every request is a dict with its arrival offset in seconds."""
    rng = np.random.default_rng(seed)
    models = {}
    for m in range(nmodels):
        three_d = rng.uniform() < 0.4
        if three_d:
            side = max(8, int(rng.integers(64, 193) * scale))
            shape = (side, side, side)
            h = 0.1
            grd = Grid3DCart(hgrid=h, cooinit=(0.0, 0.0, 0.0), grsize=shape)
        else:
            side = max(8, int(rng.integers(128, 1025) * scale))
            shape = (side, max(8, (side * 5) // 8))
            h = 0.25
            grd = Grid2DCart(hgrid=h, cooinit=(0.0, 0.0), grsize=shape)
        if rng.uniform() < 0.5:
            depth = np.arange(1, shape[-1] + 1, dtype=np.float64)
            vel = np.broadcast_to(2.5 + 2.5 * depth / shape[-1], shape).copy()
        else:
            f = gaussian_random_field(shape, 4.0 if scale < 1 else 20.0, seed=int(rng.integers(1 << 30)))
            vel = 2.0 + 3.0 * _normal_cdf(f)
        models[f"m{m}"] = (np.ascontiguousarray(vel), grd, np.ascontiguousarray(vel * 1.03))
    keys = list(models)
    t = 0.0
    reqs = []
    for i in range(n):
        t += rng.exponential(1.0 / rate)
        key = keys[int(rng.integers(len(keys)))]
        vel, grd, _ = models[key]
        nd = grd.ndim
        ns = int(rng.integers(1, max_sources + 1))
        ext = [float(grd.cooinit[d] + (grd.grsize[d] - 1) * grd.spacing[d]) for d in range(nd)]
        cs = np.array([[_avoid_node_and_half(rng.uniform(0.1 * e, 0.9 * e), grd.spacing[d], rng)
                        for d, e in enumerate(ext)] for _ in range(ns)])
        nr = 10
        rec = np.column_stack([np.linspace(0.0, ext[0], nr)] + [np.full(nr, 0.5 * ext[d]) for d in range(1, nd - 1)]
                              + [np.zeros(nr)])
        kind = "traveltime" if rng.uniform() < 0.7 else "gradient"
        r = dict(t=t, model=key, kind=kind, coordsrc=cs, coordrec=[rec.copy() for _ in range(ns)])
        if kind == "gradient":  # straight-ray times at the mean velocity, plus noise
            vm = float(np.mean(vel))
            r["pickobs"] = [np.linalg.norm(rec - cs[k], axis=1) / vm + rng.normal(0.0, 0.01, nr) for k in range(ns)]
            r["stdobs"] = [np.full(nr, 0.01) for _ in range(ns)]
        reqs.append(r)
    return models, reqs
