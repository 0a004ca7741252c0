"""The multi-GPU layout of bench.py, run as two gloo ranks on the CPU.

Each rank searches its own seeded query batch against the same full database
(weak scaling, no collective on the data path); only the timings are reduced:
the job's throughput is all ranks' cells over the slowest rank's time.  These
tests check that layout (same database, disjoint query batches of the same
length distribution) and the reductions, without a GPU.
"""
import hashlib
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out):
    import argparse
    import datetime

    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    args = argparse.Namespace(scale=0.002, workload="sw_batched", queries=None)
    w = bench.rank_workload(args, rank)
    db_digest = hashlib.sha256(np.asarray(w.db_flat).tobytes() + np.asarray(w.db_offsets).tobytes()).hexdigest()
    cells = sum(len(q) for q in w.queries) * int(w.db_offsets[-1])
    seconds = 1.0 + rank                      # rank 1 is the slow one
    bench.barrier(dist)
    got_max = bench.reduce_max(dist, seconds)
    got_sum = bench.reduce_sum(dist, float(cells))
    gcups = bench.job_throughput(dist, cells, 3, seconds)
    dist.destroy_process_group()
    out.put((rank, db_digest, [len(q) for q in w.queries], w.queries[0], cells, got_max, got_sum, gcups))


def test_two_ranks_shard_queries_and_reduce_timings():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, db0, lens0, first0, cells0, max0, sum0, g0), (r1, db1, lens1, first1, cells1, max1, sum1, g1) = res
    assert db0 == db1                              # the same full database on every rank
    assert first0 != first1                        # different query batches
    assert len(lens0) == len(lens1)
    assert max0 == max1 == 2.0                     # the slowest rank's time
    assert sum0 == sum1 == float(cells0 + cells1)
    assert g0 == g1 == pytest.approx((cells0 + cells1) * 3 / 2.0 / 1e9)
