"""Sharded exact k-NN (hercules_b200/shard.py) on the CPU: per-shard answers
(the oracle's scan of each shard) merged into the answers of the whole
collection, directly and through two gloo ranks."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def bits(x):
    return np.asarray(x, np.float32).view(np.uint32)


def test_shard_ranges_cover_the_rows_once():
    from hercules_b200.shard import shard_range
    for n in (0, 1, 7, 1000, 1001):
        for w in (1, 2, 3, 8):
            got = [shard_range(n, w, r) for r in range(w)]
            assert sum(c for _, c in got) == n
            assert all(got[r][0] + got[r][1] == got[r + 1][0] for r in range(w - 1))
            assert max(c for _, c in got) - min(c for _, c in got) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def shard_answers(oracle_mod, X, q, k, world):
    from hercules_b200.shard import shard_range
    ds, ids = [], []
    for r in range(world):
        s, c = shard_range(X.shape[0], world, r)
        d, i = oracle_mod.pscan(X[s:s + c], q, k)
        ds.append(d)
        ids.append(np.where(i >= 0, i + s, -1))
    return np.concatenate(ds)[None], np.concatenate(ids)[None]


@pytest.mark.parametrize("world", [2, 3, 5])
def test_merged_shards_equal_the_whole_collection(oracle_mod, hg, world):
    from hercules_b200.shard import merge_topk
    X = hg.generate_walks(1184, 3000, 64)
    X[2500] = X[17]  # an exact duplicate in another shard: one distance, lowest id
    X[1900] = X[17]
    Q = np.concatenate([hg.generate_queries(14784, X, np.array([0.01, 0.1, 1.0] * 3)), X[17:18]])
    for k in (1, 10, 40):
        for q in Q:
            want_d, want_i = oracle_mod.pscan(X, q, k)
            d, i = shard_answers(oracle_mod, X, q, k, world)
            md, mi = merge_topk(d, i, k)
            assert np.array_equal(bits(md[0]), bits(want_d)) and np.array_equal(mi[0], want_i)


def test_torch_merge_equals_host_merge():
    import torch
    from hercules_b200.shard import merge_topk, merge_topk_torch
    rng = np.random.default_rng(3)
    d = rng.integers(0, 40, size=(50, 24)).astype(np.float32)  # many equal distances
    i = rng.permutation(50 * 24).reshape(50, 24).astype(np.int64)
    i[rng.random((50, 24)) < 0.1] = -1
    d[i < 0] = np.inf
    for k in (1, 7, 24):
        hd, hi = merge_topk(d, i, k)
        td, ti = merge_topk_torch(torch.from_numpy(d), torch.from_numpy(i), k)
        assert np.array_equal(bits(hd), bits(td.numpy())) and np.array_equal(hi, ti.numpy())


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import datetime

    import torch
    import torch.distributed as dist
    import hercules_b200 as H
    from hercules_b200.shard import allgather_knn, shard_range
    from oracle import oracle as O
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    X = H.generate_walks(1184, 2000, 64)
    Q = H.generate_queries(14784, X, np.array([0.01, 0.1, 1.0] * 2))
    k = 10
    s, c = shard_range(X.shape[0], world, rank)
    D = np.zeros((len(Q), k), np.float32)
    I = np.zeros((len(Q), k), np.int64)
    for j, q in enumerate(Q):
        D[j], I[j] = O.pscan(X[s:s + c], q, k)
    I = np.where(I >= 0, I + s, -1)
    md, mi = allgather_knn(torch.from_numpy(D), torch.from_numpy(I), k)
    out.put((rank, md.numpy(), mi.numpy()))
    dist.destroy_process_group()


def test_two_gloo_ranks_allgather_and_merge(oracle_mod, hg):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted((out.get(timeout=120) for _ in procs), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    X = hg.generate_walks(1184, 2000, 64)
    Q = hg.generate_queries(14784, X, np.array([0.01, 0.1, 1.0] * 2))
    for _, md, mi in res:  # every rank holds the merged answers
        for j, q in enumerate(Q):
            wd, wi = oracle_mod.pscan(X, q, 10)
            assert np.array_equal(bits(md[j]), bits(wd)) and np.array_equal(mi[j], wi)


def _rank_batch(rank, world, port, out):
    """bench.py's sharded step on the host: shard answers with per-query k
    (local ids, entries past k empty), then sharded_batch_answers."""
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import datetime

    import torch
    import torch.distributed as dist
    import hercules_b200 as H
    from hercules_b200.shard import shard_range, sharded_batch_answers
    from oracle import oracle as O
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    X = H.generate_walks(1184, 2500, 64)
    Q = H.generate_queries(14784, X, np.array([0.01, 0.1, 1.0] * 3))
    ks = np.array([1, 10, 25] * 3, np.uint32)
    kmax = int(ks.max())
    s, c = shard_range(X.shape[0], world, rank)
    D = np.full((len(Q), kmax), np.inf, np.float32)
    I = np.full((len(Q), kmax), -1, np.int64)
    for j, q in enumerate(Q):
        k = int(ks[j])
        D[j, :k], I[j, :k] = O.pscan(X[s:s + c], q, k)  # shard-local ids
    md, mi = sharded_batch_answers(torch.from_numpy(D), torch.from_numpy(I), s, ks, kmax)
    out.put((rank, md.numpy(), mi.numpy()))
    dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_sharded_batch_equals_one_index(oracle_mod, hg, world):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_batch, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted((out.get(timeout=120) for _ in procs), key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    X = hg.generate_walks(1184, 2500, 64)
    Q = hg.generate_queries(14784, X, np.array([0.01, 0.1, 1.0] * 3))
    ks = [1, 10, 25] * 3
    for _, md, mi in res:
        for j, q in enumerate(Q):
            k = ks[j]
            wd, wi = oracle_mod.pscan(X, q, k)
            assert np.array_equal(bits(md[j, :k]), bits(wd)) and np.array_equal(mi[j, :k], wi)
            assert np.all(np.isinf(md[j, k:])) and np.all(mi[j, k:] == -1)
