"""The multi-rank plumbing of bench.py on CPU: two gloo ranks (one process
each, as torchrun starts one per GPU) with independent intervals and no
data-path collective; the job time is the max over ranks and the throughput
counts every rank's intervals (weak scaling). The solver itself needs no
collective: intervals are independent."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    import bench
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    w, r, local = bench._dist_setup()
    assert (w, r, local) == (world, rank, rank)
    bench._barrier(w)
    t_local = 1.0 + rank  # rank 1 is the slow one
    t_max, value = bench.weak_scaling_value(t_local, 10, w, None)
    out[rank] = (t_max, value)
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_weak_scaling():
    world = 2
    port = _free_port()
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank_main, args=(world, port, out), nprocs=world, join=True)
    for rank in range(world):
        t_max, value = out[rank]
        assert t_max == 2.0
        assert value == pytest.approx(2.0 / (10 * world))


def test_single_rank_is_local_time():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.weak_scaling_value(3.0, 6, 1, None) == (3.0, 0.5)
