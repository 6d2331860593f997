"""Host logic of batched ensembles (no GPU): the longest-processing-time
placement of members on GPUs, and the one-process-per-GPU split checked
across world_size-2 gloo ranks."""
from __future__ import annotations

import os

import numpy as np
import pytest


def test_partition_lpt():
    from powerllel_channel_sycl_b200 import partition
    costs = [7.0, 5.0, 4.0, 3.0, 3.0, 2.0]
    g = partition(costs, 2)
    loads = [sum(c for c, k in zip(costs, g) if k == r) for r in range(2)]
    assert sorted(loads) == [12.0, 12.0]
    assert partition(costs, 1) == [0] * 6
    assert sorted(set(partition(costs, 8))) == list(range(6))  # one member per GPU, 2 idle
    assert partition([], 4) == []


def test_partition_balance_random():
    from powerllel_channel_sycl_b200 import partition
    rng = np.random.default_rng(4)
    for _ in range(20):
        n, w = int(rng.integers(1, 40)), int(rng.integers(1, 9))
        costs = rng.uniform(1, 100, n)
        g = partition(list(costs), w)
        loads = np.bincount(g, weights=costs, minlength=w)
        # LPT bound: max load <= (4/3 - 1/(3w)) * optimum <= (4/3) * max(mean, max cost)
        assert loads.max() <= (4 / 3) * max(costs.sum() / w, costs.max()) + 1e-9


def _rank_main(rank, world, port, costs, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from powerllel_channel_sycl_b200.ensemble import members_of_rank
    mine = members_of_rank(costs, rank, world)
    got = [None] * world
    dist.all_gather_object(got, mine)
    if rank == 0:
        out.put(got)
    dist.barrier()
    dist.destroy_process_group()


def test_ranks_split_members_gloo():
    import multiprocessing as mp
    import socket
    ctx = mp.get_context("spawn")
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    # config 3 shape: 16 channels between 64x48x48 and 256x192x128
    rng = np.random.default_rng(0)
    dims = [(int(rng.choice([64, 96, 128, 192, 256])), int(rng.choice([48, 64, 96, 128, 192])),
             int(rng.choice([48, 64, 96, 128]))) for _ in range(16)]
    costs = [float(a * b * c) for a, b, c in dims]
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, costs, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    flat = sorted(got[0] + got[1])
    assert flat == list(range(16))
    loads = [sum(costs[i] for i in g) for g in got]
    assert max(loads) / min(loads) < 1.2
