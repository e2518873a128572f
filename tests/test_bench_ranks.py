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


def test_lpt_assignment_balances_uneven_events():
    """The bench's longest-processing-time-first assignment (cost N^2 x
    steps): every event on exactly one rank, deterministic, and the largest
    rank load within one event's cost of the smallest."""
    sys.path.insert(0, str(ROOT))
    import bench
    for world in (1, 2, 3, 4, 8):
        evs = bench.job_events(bench.HEADLINE, world)
        costs = [e["cost"] for e in evs]
        a = bench.lpt_assign(costs, world)
        assert a == bench.lpt_assign(costs, world)
        flat = sorted(i for r in a for i in r)
        assert flat == list(range(len(evs)))
        loads = [sum(costs[i] for i in r) for r in a]
        assert max(loads) - min(loads) <= max(costs)
        # weak scaling: every rank carries one workload's worth of sites
        per_gpu = sum(c["count"] * c["N"] ** 2 * bench.steps_of(bench.HEADLINE, c)
                      for c in bench.HEADLINE["classes"])
        assert all(abs(l - per_gpu) <= max(costs) for l in loads)


def _lpt_rank(rank, world, port, out):
    sys.path.insert(0, str(ROOT))
    import torch
    import torch.distributed as dist
    import bench
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    evs = bench.job_events(bench.LARGE, world)
    mine = bench.lpt_assign([e["cost"] for e in evs], world)[rank]
    # every rank computes the same assignment on its own: gather and compare
    got = [None] * world
    dist.all_gather_object(got, mine)
    out[rank] = (mine, got, bench.site_updates(bench.LARGE, [evs[i] for i in mine]))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_the_lpt_shards():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        procs = [ctx.Process(target=_lpt_rank, args=(r, world, port, out))
                 for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        res = dict(out)
    for r in range(world):
        assert res[r][1] == [res[q][0] for q in range(world)]
    assert sorted(res[0][0] + res[1][0]) == list(range(16))
    assert res[0][2] == res[1][2]  # 8 equal 1024^2 events per rank
