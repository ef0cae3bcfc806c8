"""The multi-GPU path of bench.py on CPU: world size 2 over gloo.  Every rank
steps its own scene (seed = rank, no collective on the data path); the
slowest rank's time is taken with an all-reduce MAX and the whole-job
throughput is aggregated on rank 0."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import time
    import numpy as np
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        import bench
        import oracle
        from iwf_mfree_gpu_3d_b200 import scenes
        sc = scenes.orthogonal_cutting(10, 6, 5, seed=rank)
        o = oracle.Oracle(sc, prec=64, threads=1)
        t0 = time.perf_counter()
        for _ in range(2):
            o.step()
        t = time.perf_counter() + (0.05 if rank == 1 else 0.0) - t0
        tmax = bench.reduce_max(dist, t, "cpu")
        first = float(sc.pos[0, 0])
        firsts = [None] * world
        dist.all_gather_object(firsts, first)
        if rank == 0:
            q.put((t, tmax, firsts, bench.aggregate(sc.n, 2, world, tmax)))
        else:
            q.put((t, tmax, firsts, None))
    finally:
        dist.destroy_process_group()


def test_two_rank_weak_scaling_aggregation():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    times = [r[0] for r in res]
    assert all(r[1] == pytest.approx(max(times)) for r in res)
    firsts = res[0][2]
    assert firsts[0] != firsts[1]  # independent scenes (seed = rank)
    agg = [r[3] for r in res if r[3] is not None][0]
    assert agg == pytest.approx(10 * 6 * 5 * 2 * 2 / max(times))
