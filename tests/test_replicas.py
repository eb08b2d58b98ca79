"""The multi-GPU path of bench.py on CPU: two gloo ranks on 127.0.0.1.

The P3BCA path does not shard (one GPU holds the whole cell grid), so N GPUs run N independent
replicas; the only collectives are the barrier and the reductions of the timed region: the job's
triplets are the sum over ranks and its time is the slowest rank.  The reference arm's other
ranks exit without work.
"""
import os
import socket
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=30))
    try:
        import bench
        trips = [48272380 * 3, 48272380 * 3][rank]
        ms = [2.1, 2.4][rank]
        t, m = bench.aggregate(trips, ms, world)
        bench.barrier(world)
        out[rank] = (t, m, bench.allreduce_max(float(rank), world), bench.allreduce_sum(1.0, world))
    finally:
        dist.destroy_process_group()


def test_replica_aggregation_two_gloo_ranks():
    world = 2
    port = _free_port()
    with mp.get_context("spawn").Manager() as mgr:  # no fork of this multi-threaded process
        out = mgr.dict()
        mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    for rank in range(world):
        trips, ms, rmax, rsum = res[rank]
        assert trips == 2 * 48272380 * 3  # whole-job triplets: the sum over replicas
        assert ms == pytest.approx(2.4)  # the job's time: the slowest replica
        assert rmax == 1.0 and rsum == 2.0


def test_reference_arm_other_ranks_do_nothing(capsys):
    sys.path.insert(0, str(ROOT))
    import bench

    class Args:
        workload = "c3"
        steps = 1
        warmup = 3

    bench.run_reference(Args(), world=2, rank=1)
    assert capsys.readouterr().out == ""
