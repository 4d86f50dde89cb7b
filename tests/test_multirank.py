"""Multi-GPU plumbing of bench.py, run as two gloo ranks on the CPU: every
rank is a full replica that answers its own queries, the only exchange is the
max over ranks of the timed region, and the reference arm runs on rank 0 only."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import types

    import torch.distributed as dist
    import bench
    args = types.SimpleNamespace(impl="reference")
    r, w, _ = bench.dist_setup(args, backend="gloo")
    ms = bench.max_over_ranks(10.0 * (r + 1), w)
    bench.barrier(w)
    ran = bench.run_reference(args, r, w, r) if r != 0 else "rank0"
    out.put((r, w, ms, bench.rank_offset(r), ran))
    dist.destroy_process_group()


def test_two_gloo_ranks_take_the_max_time_and_split_queries():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(out.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [2, 2]
    assert [r[2] for r in res] == [20.0, 20.0]  # both ranks report the slowest rank's time
    assert res[0][3] != res[1][3]               # distinct query seeds per replica
    assert res[1][4] is None                    # reference arm: rank 1 does no work


def test_replica_queries_differ(hg):
    import bench
    X = hg.generate_walks(1184, 2000, 64)
    s = bench.sigma2_for(8)
    a = hg.generate_queries(bench.QUERY_SEED + bench.rank_offset(0), X, s)
    b = hg.generate_queries(bench.QUERY_SEED + bench.rank_offset(1), X, s)
    assert not np.array_equal(a, b)
