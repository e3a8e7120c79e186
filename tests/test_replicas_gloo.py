"""Multi-GPU replica logic of bench.py, run as two gloo ranks on the CPU.

The path does not shard across GPUs: every rank solves its own seeded
instance with no collective on the data path.  The only cross-rank work is
the aggregation of the timing (slowest rank's time, all ranks' iterations),
which must be the same collectives in the same order on every rank.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        elapsed = [120.0, 95.0][rank]          # ms of this rank's timed trajectories
        iters = [4724, 4800][rank]             # CG iterations this rank ran
        t, it = bench.reduce_over_ranks(dist, elapsed, iters, "cpu")
        k, _ = bench.make_field(8, 1 + rank)   # per-rank seeded instance
        out[rank] = (t, it, float(np.sum(k)))
    finally:
        dist.destroy_process_group()


def test_replica_aggregation_two_ranks():
    port = _free_port()
    with mp.get_context("spawn").Manager() as m:
        out = m.dict()
        mp.spawn(_rank_main, args=(2, port, out), nprocs=2, join=True)
        res = dict(out)
    assert res[0][:2] == res[1][:2] == (120.0, 9524.0)    # max time, summed iterations
    assert res[0][2] != res[1][2]                          # ranks solve different seeded instances


def test_single_process_aggregation_is_identity():
    import bench

    assert bench.reduce_over_ranks(None, 12.5, 7, "cpu") == (12.5, 7.0)


if __name__ == "__main__":
    pytest.main([__file__, "-q"])
