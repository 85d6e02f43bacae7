"""Replica layout of bench.py's multi-GPU run, on two gloo ranks (CPU):
each rank traverses its own seeded source set (the CPU oracle stands in for
the GPU here), and the job's GTEPS is all ranks' work over the slowest
rank's time."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

import xbtrav
from oracle import oracle as O
from xbtrav import replicas


def _free_port() -> int:
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import datetime
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    for p in (os.path.dirname(here), os.path.join(os.path.dirname(here), "xblossom-sigmetrics27-ae_b200")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import torch.distributed as dist

    from oracle import oracle as O2
    import xbtrav as X
    from xbtrav import replicas as R

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ro, ci = X.HostCSR.rmat(10, 8, seed=9).arrays()
    src = X.select_sources_csr(ro, R.rank_seed(100, rank), 32)
    _, _, edges, _ = O2.msbfs(ro, ci, src)
    ms = 10.0 * (rank + 1)  # a fixed per-rank time, so the result is checkable
    gteps, job_ms = R.whole_job_gteps(dist, edges, ms)
    out[rank] = (list(map(int, src)), int(edges), gteps, job_ms)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_aggregate_like_the_bench():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    (s0, e0, g0, t0), (s1, e1, g1, t1) = res[0], res[1]
    assert s0 != s1  # each rank its own sources
    ro, ci = xbtrav.HostCSR.rmat(10, 8, seed=9).arrays()
    for r, (s, e) in enumerate(((s0, e0), (s1, e1))):
        assert s == list(xbtrav.select_sources_csr(ro, replicas.rank_seed(100, r), 32))
        assert e == O.msbfs(ro, ci, np.array(s, np.int32))[2]
    assert t0 == t1 == 20.0  # the slowest rank
    want = (e0 + e1) / 0.020 / 1e9
    assert abs(g0 - want) < 1e-9 * want and abs(g1 - want) < 1e-9 * want


def test_single_process_needs_no_collective():
    assert replicas.whole_job_gteps(None, 2e9, 1000.0) == (2.0, 1000.0)
    assert replicas.rank_seed(5, 0) == 5
