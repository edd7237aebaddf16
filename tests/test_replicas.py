"""Multi-GPU runs are independent replicas (no data-path collective): the
only cross-rank step is the max of the timed totals.  Checked with two gloo
ranks on the CPU (the same reduction bench.py runs over NCCL)."""
import os
import socket
import sys

import pytest

torch = pytest.importorskip("torch")
import torch.multiprocessing as mp  # noqa: E402

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    torch.distributed.init_process_group("gloo", rank=rank, world_size=world,
                                         timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        total = 1.0 + 0.5 * rank                      # rank 1 is the slow one
        m = bench.reduce_max(total, torch, "cpu")
        out[rank] = (m, bench.replica_value(world, 10, m))
    finally:
        torch.distributed.destroy_process_group()


def test_two_rank_max_and_replica_value():
    world, port = 2, _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1] == (1.5, 2 * 10 / 1.5)


def test_single_process_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.reduce_max(3.25, torch, "cpu") == 3.25
    assert bench.replica_value(1, 4, 2.0) == 2.0
