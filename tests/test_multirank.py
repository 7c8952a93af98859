"""The multi-GPU bench path's host logic on CPU ranks (gloo, world size 2): every rank runs its
own batch (seed = rank), and the timed region is the maximum over ranks."""

import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world))
    from datetime import timedelta

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench
    from scatrs_b200 import workloads as W

    w = W.batched_spheres(seed=rank, scale=0.01)
    ms = bench.max_over_ranks(10.0 + rank, device="cpu")
    nodes = bench.total_nodes(world, w.n_nodes_total)
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, ms, nodes, float(w.m[0, 0].real)))


def test_two_ranks_weak_scaling_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [11.0, 11.0]  # the slowest rank's time on every rank
    assert res[0][2] == res[1][2] == 2 * res[0][2] // 2
    assert res[0][3] != res[1][3]  # each rank its own seeded batch
