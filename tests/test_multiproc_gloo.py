"""N>1 path of bench.py on CPU with gloo, world_size 2: the weak-scaling box set (256 boxes per
rank) is placed on the ranks by the library's mdpd_place, each rank computing the same placement
and taking its share (no data-path collective); only the timing/throughput reduction crosses
ranks (max of time, sum of particle-steps)."""
import os
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench
    cfg = bench.rank_boxes(rank, world)
    ntot = sum(c["n"] for c in cfg)
    # which boxes this rank took (seeds are unique per box): every rank sees every share
    import torch
    mine = torch.tensor(sorted(c["seed"] for c in cfg) + [-1] * (512 - len(cfg)), dtype=torch.int64)
    shares = [torch.zeros_like(mine) for _ in range(world)]
    dist.all_gather(shares, mine)
    out["shares"] = [[int(x) for x in t if x >= 0] for t in shares]
    secs = 1.0 + rank  # rank 1 is the slow one
    value, tmax = bench.aggregate(ntot * 10, secs, world, device="cpu")
    out[rank] = (ntot, value, tmax)
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_weak_scaling_reduction():
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = 29500 + os.getpid() % 1000
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    (n0, v0, t0), (n1, v1, t1) = out[0], out[1]
    import bench
    every = sorted(c["seed"] for c in bench.batched_boxes(seed=1) + bench.batched_boxes(seed=2))
    a, b = out["shares"]
    assert not set(a) & set(b) and sorted(a + b) == every  # each box on exactly one rank
    assert abs(n0 - n1) / (n0 + n1) < 0.01  # particles balanced between the ranks
    assert t0 == t1 == 2.0  # time is the max over ranks
    assert v0 == v1 == pytest.approx((n0 + n1) * 10 / 2.0)


def test_box_sets_are_seeded_and_uneven():
    import bench
    a, b = bench.batched_boxes(seed=1), bench.batched_boxes(seed=1)
    assert a == b and len(a) == 256
    ns = [c["n"] for c in a]
    assert min(ns) >= 2000 and max(ns) <= 200000 and max(ns) / min(ns) > 20
