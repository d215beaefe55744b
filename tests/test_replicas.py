"""Multi-GPU form of the benchmark: N independent replicas, one process per GPU.

The path has no cross-GPU exchange, so the only multi-rank logic is how the
whole-job figures are formed: units are summed over ranks and the time is the
slowest rank's.  These tests run that logic as two `gloo` ranks on the CPU
(rendezvous on 127.0.0.1), with ranks that processed different amounts of
work in different times, and check the reference arm's rank handling.
"""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import datetime
    import torch
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        cpu = torch.device("cpu")
        units = bench.sum_over_ranks(1000 + 7 * rank, cpu, world)   # ints stay ints
        ms = bench.max_over_ranks(2.5 + rank, cpu, world)
        value = units / (ms / 1e3)
        # second round in the same order: deletes
        units2 = bench.sum_over_ranks(10 * (rank + 1), cpu, world)
        ms2 = bench.max_over_ranks(1.0 / (rank + 1), cpu, world)
        q.put((rank, units, ms, value, units2, ms2, type(units).__name__))
    finally:
        torch.distributed.destroy_process_group()


def test_whole_job_figures_over_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    got = sorted(q.get(timeout=10) for _ in range(2))
    for rank, units, ms, value, units2, ms2, tname in got:
        assert units == 1000 + 1007 and tname == "int"
        assert ms == 3.5                     # the slower rank's time
        assert value == pytest.approx(2007 / 3.5e-3)
        assert units2 == 30 and ms2 == 1.0


def test_single_rank_is_identity():
    import bench
    assert bench.sum_over_ranks(5, None, 1) == 5
    assert bench.max_over_ranks(1.25, None, 1) == 1.25


def test_reference_arm_runs_on_rank_zero_only():
    import argparse
    import bench
    args = argparse.Namespace(steps=1, warmup=3)
    assert bench.run_reference_arm(args, rank=1, world=2) is None
