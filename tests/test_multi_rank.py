"""The multi-GPU path's host logic with two gloo ranks on the CPU: the scene partition every rank computes
is identical, disjoint and complete, and the timing / count reductions see both ranks."""
import os
import socket

import numpy as np
import pytest


def test_partition_is_complete_disjoint_and_balanced():
    from rainbow_b200.sharding import partition_scenes
    rng = np.random.default_rng(3)
    costs = np.round(np.exp(rng.uniform(np.log(8), np.log(256), 1024)))
    for n in (1, 2, 3, 4, 8):
        parts = partition_scenes(costs, n)
        allidx = np.concatenate(parts)
        assert len(allidx) == len(costs) and len(np.unique(allidx)) == len(costs)
        loads = np.array([costs[p].sum() for p in parts])
        assert loads.max() - loads.min() <= costs.max()      # LPT bound: within one scene of each other


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from rainbow_b200.sharding import max_over_ranks, partition_scenes, sum_over_ranks
    costs = np.arange(1, 101, dtype=np.float64)[::-1]
    mine = partition_scenes(costs, world)[rank]
    t_max = max_over_ranks(10.0 + rank)               # each rank's own "device time"
    n_sum = sum_over_ranks(len(mine))
    out.put((rank, mine.tolist(), t_max, n_sum))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_share_scenes_and_reduce_timings():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, m0, t0, n0), (r1, m1, t1, n1) = res
    assert sorted(m0 + m1) == list(range(100)) and not set(m0) & set(m1)
    assert t0 == t1 == 11.0                             # max over ranks
    assert n0 == n1 == 100.0                            # sum over ranks
