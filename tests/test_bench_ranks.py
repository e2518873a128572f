"""Multi-rank logic of bench.py on CPU: two gloo ranks, each with its own
events, combine their timings as the max over ranks, and the whole-job rate
counts every rank's events against the slowest rank."""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    sys.path.insert(0, str(ROOT))
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    # rank r took (r + 1) * 10 ms for FP32 and 5 ms flat for FP64
    got = bench.max_over_ranks(dist, [10.0 * (rank + 1), 5.0], "cpu")
    out[rank] = (got, bench.rank_seed_base(rank))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max_and_shard_events():
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
    for r in range(world):
        assert res[r][0] == [20.0, 5.0]  # every rank sees the slowest rank
    seeds = [res[r][1] for r in range(world)]
    assert len(set(seeds)) == world and min(abs(a - b) for a in seeds for b in seeds if a != b) >= 1000


def test_whole_job_rate_counts_all_ranks():
    sys.path.insert(0, str(ROOT))
    import bench
    # 2 ranks x 5 events in a slowest-rank time of 100 ms -> 100 events/s
    assert bench.whole_job_rate(2, 5, 100.0) == pytest.approx(100.0)
    assert bench.max_over_ranks(None, [3.0, 4.0], "cpu") == [3.0, 4.0]
