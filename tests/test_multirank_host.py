"""The multi-rank host logic of the benchmark on CPU with a world-size-2 gloo
group: ranks split the independent batch problems round robin with no data
exchange, and the only collectives are the max over ranks of the device times
and the sum of the work counts, called once by every rank in the same order."""
import os
import pathlib
import sys

import pytest
import torch.multiprocessing as mp

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _worker(rank, world, port, out):
    sys.path[:0] = [str(ROOT), str(ROOT / "twophaseamr.jl_b200")]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime
    import torch.distributed as dist
    import bench
    from tpagmg import workloads as W

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        problems = bench.rank_share(W.batch_problems(16), rank, world)
        mine = [p["index"] for p in problems]
        # per-rank "times" and work counts
        mx, sm = bench.combine_over_ranks([1.0 + rank, 10.0 * (rank + 1)], [len(mine), sum(mine)], world)
        out.put((rank, mine, mx, sm))
    finally:
        dist.destroy_process_group()


def test_two_ranks_split_problems_and_reduce_timings():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = 29000 + os.getpid() % 1000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, m0, mx0, sm0), (r1, m1, mx1, sm1) = res
    assert sorted(m0 + m1) == list(range(16)) and not set(m0) & set(m1)
    assert mx0 == mx1 == [2.0, 20.0]
    assert sm0 == sm1 == [16.0, float(sum(range(16)))]


def test_single_rank_needs_no_process_group():
    sys.path[:0] = [str(ROOT), str(ROOT / "twophaseamr.jl_b200")]
    import bench
    assert bench.rank_share(range(5), 0, 1) == [0, 1, 2, 3, 4]
    assert bench.combine_over_ranks([3.0], [4.0], 1) == ([3.0], [4.0])
