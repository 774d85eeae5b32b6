"""Multi-rank timing of bench.py on CPU (gloo, world size 2): every rank
reports the slowest rank's step time, and the job's throughput is the number
of replicas over that time (one independent replica per GPU, no collective on
the data path)."""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank(rank, world, port, out):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ms = 10.0 + 5.0 * rank  # the second replica is slower
        out[rank] = bench.max_over_ranks(ms, device="cpu")
    finally:
        dist.destroy_process_group()


def test_step_time_is_the_max_over_ranks():
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        assert dict(out) == {0: 15.0, 1: 15.0}
    sys.path.insert(0, ROOT)
    import bench
    # one replica at the slowest replica's pace: simulated seconds per wall second times dt
    one = bench.sim_years_per_day(15.0, 1800.0)
    assert one == pytest.approx(86400.0 / 0.015 * 1800.0 / bench.SECONDS_PER_YEAR, rel=1e-12)


def test_single_process_passes_the_value_through():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, device="cpu") == 3.5
