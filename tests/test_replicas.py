"""The multi-GPU path of bench.py runs independent replicas (one simulation
per rank, no data-path collective): the only cross-rank steps are a barrier
and the max-over-ranks reduction of the timed region.  Checked here with
two gloo ranks on the CPU."""
import os
import socket
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import bench
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        local_ms = 100.0 * (rank + 1)  # rank 1 is the slower replica
        dist.barrier()
        m = bench.max_over_ranks(local_ms, dist, "cpu")
        out[rank] = (m, bench.whole_job_rate(20, world, m))
    finally:
        dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank():
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_rank, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
        res = dict(out)
    assert res[0] == res[1]
    max_ms, rate = res[0]
    assert max_ms == 200.0
    assert rate == pytest.approx(2 * 20 / 0.2)


def test_single_rank_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(5.0, None, "cpu") == 5.0
    assert bench.whole_job_rate(10, 1, 500.0) == pytest.approx(20.0)
