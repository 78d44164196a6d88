"""The N-rank path of bench.py on CPU: gloo process group of two ranks (replicas, no data-path
collective; the only exchange is the max-over-ranks of the device time)."""
import os
import socket

import pytest

torch = pytest.importorskip("torch")
import torch.distributed as dist  # noqa: E402
import torch.multiprocessing as mp  # noqa: E402


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import datetime
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    ms = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")
    out[rank] = ms
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_gloo():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
    assert out[0] == out[1] == 15.0


def test_value_is_whole_job_aggregate():
    """value = all ranks' cell-updates / slowest rank's time (weak scaling, one replica per GPU)."""
    cells, species, steps, world, ms = 1000, 2, 10, 4, 50.0
    value = cells * species * 2 * steps * world / (ms / 1e3)
    assert value == pytest.approx(3.2e6)
