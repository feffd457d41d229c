"""Two ranks on CPU (gloo): the sharded gradient equals the reference's :sharedmem gradient
with two threads (each rank solves one distribsrcs group, here with the oracle as the local
solver), and the shard ranges are distribsrcs' groups. Failure detection: a rank whose shard
raises makes every rank raise ShardFailed; a rank that dies before the exchange makes the
other's collective end with an error within the process group's timeout, not hang."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from eikonalsolvers.parallel import distribsrcs, shard


def test_distribsrcs_groups():
    assert distribsrcs(7, 3) == [(0, 2), (3, 4), (5, 6)]
    assert distribsrcs(2, 4) == [(0, 0), (1, 1)]
    assert shard(7, 3, 1) == (3, 5) and shard(2, 4, 3) is None


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, case, out):
    import torch.distributed as dist
    import eikoracle as O
    from eikonalsolvers.parallel import eikgradient_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    vel, grd, cs, rec, po, so, ep = case

    def local(v, g, c, r, p, s, wg, e):
        return O.eikgradient(v, g, c, r, p, s, wg, extraparams=e)
    res = eikgradient_sharded(vel, grd, cs, rec, po, so, "gradvelandsrcloc", ep, local=local)
    out[rank] = res
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_gradient_equals_sharedmem_groups():
    import eikoracle as O
    from eikonalsolvers import ExtraParams
    from eikonalsolvers import configs as CF
    w = CF.cfg2(scale=0.125, nsrc=2)
    h = w.grd.hgrid
    x0 = w.coordsrc[0][0]
    cs = np.array([[x0 + 0.37 * h * k, (60 - 6.3 * k) * h + 0.011] for k in range(5)])  # stacked: carry-over matters
    rec = [w.coordrec[0]] * 5
    ep = ExtraParams(radiussmoothgradsrc=0)
    po = O.eiktraveltime(w.vel * 1.02, w.grd, cs, rec, extraparams=ep)
    so = [0.01 * np.ones(p.shape) for p in po]
    case = (w.vel, w.grd, cs, rec, po, so, ep)
    ctx = mp.get_context("spawn")
    with ctx.Manager() as man:
        out = man.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, case, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=300)
        assert all(p.exitcode == 0 for p in procs)
        res = dict(out)
    eps = ExtraParams(radiussmoothgradsrc=0, parallelkind="sharedmem")
    gv, gs, m = O.eikgradient(w.vel, w.grd, cs, rec, po, so, "gradvelandsrcloc", extraparams=eps, nthreads=2)
    gv1, gs1, m1 = O.eikgradient(w.vel, w.grd, cs, rec, po, so, "gradvelandsrcloc", extraparams=ep)
    assert np.linalg.norm(gv - gv1) > 1e-6 * np.linalg.norm(gv)  # the grouping is visible
    for r in range(2):
        g, s, mm = res[r]
        assert np.array_equal(g, gv)
        assert np.array_equal(s, gs)
        assert mm == m


def _failing_rank(rank, world, port, mode, out):
    import torch.distributed as dist
    from eikonalsolvers import configs as CF
    from eikonalsolvers.parallel import eikgradient_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=10))
    w = CF.cfg2(scale=0.125, nsrc=2)
    if mode == "dies" and rank == 1:
        os._exit(3)  # leaves between steps, with nothing in flight

    def local(v, g, c, r, p, s, wg, e):
        if rank == 1:
            raise ValueError("bad shard")
        N = int(np.prod(g.grsize))
        return np.zeros(N), 0.0
    po = [np.zeros(r.shape[0]) for r in w.coordrec]
    try:
        eikgradient_sharded(w.vel, w.grd, w.coordsrc, w.coordrec, po, po, "gradvel", None, local=local)
        out[rank] = "returned"
    except Exception as e:
        out[rank] = f"{type(e).__name__}: {e}"
    os._exit(0)


@pytest.mark.parametrize("mode", ["raises", "dies"])
def test_a_failed_shard_is_reported_on_every_rank(mode):
    import time
    ctx = mp.get_context("spawn")
    with ctx.Manager() as man:
        out = man.dict()
        port = _free_port()
        procs = [ctx.Process(target=_failing_rank, args=(r, 2, port, mode, out)) for r in range(2)]
        t0 = time.time()
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
        assert all(p.exitcode is not None for p in procs), "a rank hung"
        res = dict(out)
    assert time.time() - t0 < 120
    if mode == "raises":
        assert res[0].startswith("ShardFailed") and "rank(s) [1]" in res[0], res
        assert res[1].startswith("ShardFailed") and "bad shard" in res[1], res
    else:
        assert procs[1].exitcode == 3
        assert res[0] != "returned" and 0 in res, res  # the collective ended with an error
