"""bench.py's multi-GPU form is replicas only: every rank runs its own
seeded sources on its own copy of the graph, with no collective on the data
path.  This checks, with two gloo ranks on the CPU, the host logic around
it: distinct per-rank sources, the whole-job value (entries of all ranks over
the slowest rank's time), and that the reference arm runs on rank 0 only."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import sys
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    import datetime

    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    rp = np.concatenate([[0], np.cumsum(np.arange(1000) % 7)]).astype(np.int64)
    srcs = bench.pick_sources(rp, 8, 7, salt=rank)
    edges = 1000 * (rank + 1)
    ms = 10.0 * (rank + 1)
    value, total, mx = bench.replica_gteps(world, edges, ms)
    bench.barrier_sync(world)
    # The reference arm does its work on rank 0 only; other ranks return
    # nothing (and exit 0).
    import argparse
    ref = bench.run_reference(argparse.Namespace(scale=8, edge_factor=4, seed=7, sources=4, warmup=1, steps=1),
                              world, rank) if rank != 0 else "skipped"
    out[rank] = (srcs, value, total, mx, ref)
    dist.destroy_process_group()


def test_two_gloo_ranks_replica_accounting():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    s0, s1 = res[0][0], res[1][0]
    assert len(s0) == 8 and len(s1) == 8 and s0 != s1
    for r in range(world):
        _, value, total, mx, _ = res[r]
        assert total == 3000.0 and mx == 20.0
        assert abs(value - 3000.0 / 0.020 / 1e9) < 1e-12
    assert res[1][4] is None
