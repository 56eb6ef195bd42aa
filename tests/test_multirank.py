"""Multi-GPU runs of bench.py are independent replicas: the only exchange is
the max over ranks of the device time. Checked here with two gloo ranks on
CPU (no GPU involved)."""

import os
import socket
import sys
from pathlib import Path

import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench

    t = bench.max_over_ranks(10.0 + 5.0 * rank, dist, device="cpu")
    out[rank] = (t, bench.replica_rate(world, t / 4))
    dist.barrier()
    dist.destroy_process_group()


def test_two_replicas_report_the_slowest_rank():
    world, port = 2, _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert res[0] == res[1]
    t, rate = res[0]
    assert t == 15.0  # the slower rank's time
    assert abs(rate - 2 * 1e3 / (15.0 / 4)) < 1e-9
