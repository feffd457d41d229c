"""Sources sharded over ranks (one process per GPU, torch.distributed for the exchange).

The reference parallelises by source only (`:sharedmem` threads, `:distribmem` workers),
with the contiguous groups of `distribsrcs` (src/EikSolv/eikutils.jl:171-190). Here rank
r takes group r of `distribsrcs(nsrc, world)`, solves it on its own GPU, and the group
results are combined as the reference combines its groups (eikmaingrad.jl:137-150): the
velocity gradients and the misfits are summed, the per-source results gathered in source
order. Because a group's gradient buffer carry-over (source points inheriting the previous
source's value) stays inside the group, the result equals the reference's `:sharedmem`
gradient with `world` threads.

The only exchange is one all-reduce of the summed gradient (N values) and the misfit, and
an all-gather of picks / source gradients: the path has no other communication.

Failure detection: before any result is exchanged every rank reports whether its shard
succeeded (one all-gather of a status word, the same collective steps on every rank); when a
shard failed, every rank raises ShardFailed naming the failed ranks, instead of waiting for a
result that will not come. A rank that dies outright is detected by the process group's
timeout (or the backend's broken connection) at that first exchange.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Tuple

import numpy as np


class ShardFailed(RuntimeError):
    """A rank's shard of the sources failed; raised on every rank."""


def distribsrcs(nsrc: int, nw: int) -> List[Tuple[int, int]]:
    """Contiguous source groups [first, last] (0-based, inclusive), as eikutils.jl:171-190."""
    if nsrc >= nw:
        dis, resto = divmod(nsrc, nw)
        sizes = [dis + (1 if i < resto else 0) for i in range(nw)]
    else:
        sizes = [1] * nsrc
    out, c = [], 0
    for s in sizes:
        out.append((c, c + s - 1))
        c += s
    return out


def shard(nsrc: int, world: int, rank: int) -> Optional[Tuple[int, int]]:
    """Half-open source range [s0, s1) of this rank, or None when it has no source."""
    g = distribsrcs(nsrc, world)
    if rank >= len(g):
        return None
    return g[rank][0], g[rank][1] + 1


def eikgradient_sharded(vel, grd, coordsrc, coordrec, pickobs, stdobs, whichgrad, extraparams=None,
                        local: Optional[Callable] = None, group=None):
    """eikgradient over all ranks of `group` (torch.distributed, initialised by the caller).

    `local(vel, grd, coordsrc, coordrec, pickobs, stdobs, whichgrad, extraparams)` solves one
    shard and returns what `eikgradient` returns; by default the GPU path of this rank's
    device. Every rank returns the full result."""
    import torch
    import torch.distributed as dist
    if local is None:
        from .api import eikgradient as local  # noqa: N813
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    nsrc = int(np.atleast_2d(coordsrc).shape[0])
    nd = grd.ndim
    rng = shard(nsrc, world, rank)
    wg = whichgrad.lstrip(":")
    N = int(np.prod(grd.grsize))
    gv = np.zeros(N, dtype=np.float64)
    gs = np.zeros((nsrc, nd), dtype=np.float64)
    misf = 0.0
    err = None
    if rng is not None:
        s0, s1 = rng
        try:
            res = local(vel, grd, np.asarray(coordsrc)[s0:s1], coordrec[s0:s1], pickobs[s0:s1], stdobs[s0:s1], wg,
                        extraparams)
            if wg == "gradvel":
                gv = np.asarray(res[0], dtype=np.float64).ravel(order="F")
            elif wg == "gradsrcloc":
                gs[s0:s1] = res[0]
            else:
                gv = np.asarray(res[0], dtype=np.float64).ravel(order="F")
                gs[s0:s1] = res[1]
            misf = float(res[-1])
        except Exception as e:  # reported to every rank below
            err = e
    dev = torch.device("cuda", torch.cuda.current_device()) if dist.get_backend(group) == "nccl" else "cpu"
    status = [torch.zeros(1, dtype=torch.float64, device=dev) for _ in range(world)]
    dist.all_gather(status, torch.tensor([1.0 if err is not None else 0.0], dtype=torch.float64, device=dev),
                    group=group)
    failed = [r for r, f in enumerate(status) if float(f.item()) != 0.0]
    if failed:
        raise ShardFailed(f"the source shard of rank(s) {failed} failed" + (f": {err}" if err is not None else "")) \
            from err
    # group sums in group order: g0 + g1 + ... (a sum of two terms is order independent)
    parts = [torch.zeros(N + 1, dtype=torch.float64, device=dev) for _ in range(world)]
    mine = torch.from_numpy(np.concatenate([gv, [misf]])).to(dev)
    dist.all_gather(parts, mine, group=group)
    tot = parts[0].clone()
    for p in parts[1:]:
        tot = tot + p
    tot = tot.cpu().numpy()
    gsrc = torch.from_numpy(gs.ravel()).to(dev)
    dist.all_reduce(gsrc, group=group)  # disjoint rows: the sum is exact
    gvel = tot[:N].reshape(grd.grsize, order="F")
    gsrc = gsrc.cpu().numpy().reshape(nsrc, nd)
    if wg == "gradvel":
        return gvel, float(tot[N])
    if wg == "gradsrcloc":
        return gsrc, float(tot[N])
    return gvel, gsrc, float(tot[N])
