"""The multi-rank path of bench.py on CPU (two gloo ranks over 127.0.0.1):
timings reduce to the maximum over ranks, the whole-job rate counts every
rank's replica, and replicas of the same seeded job give the same graph."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, out):
    import sys
    from datetime import timedelta

    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench
    from indexgen_b200 import workloads as W
    from oracle import oracle as O

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        t = bench.max_over_ranks(10.0 + 5.0 * rank, dist, "cpu")
        # every rank builds the same seeded replica; the graphs must agree
        w = W.uniform_words(1500, 10, 77)
        rp, cols = O.conflict_upper(w, 10, 4, threads=1)
        digest = torch.tensor([int(rp[-1]), int(np.bitwise_xor.reduce(cols.astype(np.int64) * 2654435761 % (1 << 31)))],
                              dtype=torch.int64)
        got = [torch.zeros(2, dtype=torch.int64) for _ in range(world)]
        dist.all_gather(got, digest)
        out[rank] = (t, [g.tolist() for g in got])
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world = 2
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, join=True, start_method="spawn")
    assert sorted(out.keys()) == [0, 1]
    for r in range(world):
        t, digests = out[r]
        assert t == 15.0  # the max over ranks, seen by every rank
        assert digests[0] == digests[1] and digests[0][0] > 0


def test_replica_rate():
    import sys

    sys.path.insert(0, ROOT)
    import bench

    assert bench.replica_rate(1, 10**9, 1, 1.0) == 1.0
    assert bench.replica_rate(4, 10**9, 3, 2.0) == 6.0
    assert bench.max_over_ranks(3.5, None, "cpu") == 3.5


def test_alu_op_counts():
    """The roofline's ALU-pipe op counts per pair test, per lane form, as
    derived from the recurrences in ig_myers.cuh (11 ALU ops per character
    step; 5 fewer in the last step; flushes and threshold)."""
    import sys

    sys.path.insert(0, ROOT)
    import bench

    assert bench.alu_ops_per_pair(12, 4) == (11 * 12 - 5 + 3 * 2 + 4) / 8 == 17.125
    assert bench.alu_ops_per_pair(7, 3) == (11 * 7 - 5 + 3 * 1 + 4) / 8
    assert bench.alu_ops_per_pair(16, 5) == (11 * 16 - 3) / 4 == 43.25
    assert bench.alu_ops_per_pair(12, 9) == 4 * 12 and bench.alu_ops_per_pair(16, 9) == 8 * 16
