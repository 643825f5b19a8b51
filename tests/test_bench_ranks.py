"""The multi-GPU form of bench.py is N independent replicas, one per rank: the
job time is the largest rank's time and the job value sums the replicas' work.
Checked here with two gloo ranks on the CPU (the reduction bench.py runs over
NCCL on GPUs)."""
import os
import socket
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, times, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        t = bench.max_over_ranks(times[rank], world, "cpu")
        out[rank] = (t, bench.job_value(1030301, 25, 10, world, t))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_replicas_take_the_slowest_rank():
    world, port = 2, _free_port()
    times = [0.25, 0.40]
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, times, out), nprocs=world, join=True)
        got = dict(out)
    for rank in range(world):
        t, value = got[rank]
        assert t == max(times)
        assert abs(value - 2 * 1030301 * 25 * 10 / 0.40 / 1e6) < 1e-6


def test_single_rank_is_its_own_time():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(0.123, 1, "cpu") == 0.123
    assert abs(bench.job_value(100, 2, 5, 1, 1.0) - 1000 / 1e6) < 1e-12
