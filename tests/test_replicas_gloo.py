"""The N-replica aggregation of bench.py on world_size 2 with gloo (CPU): the
job's time is the max over ranks, its particle-steps the sum."""
import os
import socket
import sys
from pathlib import Path

import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, str(ROOT))
    import bench
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms, ps, v = bench.aggregate(100.0 + 50.0 * rank, 1e9 * (rank + 1), world)
    out[rank] = (ms, ps, v)
    bench.barrier(world)
    dist.destroy_process_group()


def test_replica_aggregation_gloo():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    for r in range(world):
        ms, ps, v = out[r]
        assert ms == 150.0 and ps == 3e9
        assert abs(v - 3e9 / 0.15) < 1e-3 * v
