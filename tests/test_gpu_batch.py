"""GPU parity of the batched path (BF16 tensor-core filter with a certified
error bound + exact FP32 re-rank): its answers must be bit-identical to the
plain path's (itself pinned to the oracle and the reference), for mixed k,
through the filter (most queries verified) and through the fallback."""
import json

import numpy as np
import pytest

from conftest import golden_path

pytestmark = pytest.mark.gpu


def bits(x):
    return np.asarray(x, np.float32).view(np.uint32)


def same_as_plain(ix, Q, ks, d, ids):
    for kk in sorted(set(int(k) for k in ks)):
        sel = np.nonzero(ks == kk)[0]
        pd, pi = ix.knn(Q[sel], kk, use_lb_sax=True)
        assert np.array_equal(bits(d[sel, :kk]), bits(pd)), kk
        assert np.array_equal(ids[sel, :kk], pi), kk
        assert np.all(np.isinf(d[sel, kk:])) and np.all(ids[sel, kk:] == -1)


@pytest.fixture(scope="module")
def mid(hg, gpu_available):
    """200k x 256 walks, leaf 10000: queries at three noise levels plus fresh walks."""
    X = hg.generate_walks(1184, 200_000, 256)
    sig = np.array([0.01, 0.1, 1.0] * 60)
    Q = hg.generate_queries(14784, X, sig)
    fresh = hg.generate_walks(777, 20, 256)
    Q = np.concatenate([Q, fresh])
    ix = hg.HerculesIndex.build(X, 10_000)
    return X, Q, ix


@pytest.mark.parametrize("k", [1, 10, 100])
def test_batch_matches_plain_uniform_k(mid, k):
    X, Q, ix = mid
    d, ids, st = ix.knn_batch(Q, k, stats=True)
    same_as_plain(ix, Q, np.full(len(Q), k), d, ids)
    # the filter, not the fallback, answered nearly every query
    assert st["fallback_queries"] <= len(Q) // 20, st
    # LB_EAPCA keeps only part of the (query, leaf) pairs for the filter
    assert st["survivors"] > 0 and 0 < st["bf16_pairs"] <= len(Q) * X.shape[0]
    # the certified bound the filter used: positive, and at L = 256 on
    # z-normalised walks well below the plain 2u|q||x| bound (4.0)
    assert 0 < st["err_mean"] <= st["err_max"] < 4.0, st
    assert st["err_over_bound"] > 0, st


def test_pruned_filter_equals_dense_filter(mid):
    """Filtering only the leaves whose LB_EAPCA is within a query's bound
    gives the same answers as filtering every row, with fewer pairs."""
    X, Q, ix = mid
    ks = np.array([1, 10, 100, 5] * (len(Q) // 4) + [10] * (len(Q) % 4), np.uint32)
    d1, i1, s1 = ix.knn_batch(Q, ks, stats=True)
    d2, i2, s2 = ix.knn_batch(Q, ks, stats=True, dense_filter=True)
    assert np.array_equal(bits(d1), bits(d2)) and np.array_equal(i1, i2)
    assert s2["bf16_pairs"] >= len(Q) * X.shape[0]
    assert s1["bf16_pairs"] < s2["bf16_pairs"], (s1["bf16_pairs"], s2["bf16_pairs"])
    same_as_plain(ix, Q, ks, d1, i1)


def test_batch_mixed_k(mid):
    X, Q, ix = mid
    rng = np.random.default_rng(5)
    ks = rng.choice(np.array([1, 10, 100], np.uint32), size=len(Q))
    d, ids, st = ix.knn_batch(Q, ks, stats=True)
    assert d.shape == (len(Q), 100)
    same_as_plain(ix, Q, ks, d, ids)


def test_batch_matches_oracle(mid, oracle_mod):
    X, Q, ix = mid
    d, ids = ix.knn_batch(Q[:6], 10)
    for j in range(6):
        od, oid = oracle_mod.pscan(X, Q[j], 10)
        assert np.array_equal(bits(d[j]), bits(od))
        assert np.array_equal(ids[j], oid)


def test_batch_fallback_when_buckets_overflow(mid):
    """A one-entry bucket overflows for every query: all take the plain path."""
    X, Q, ix = mid
    d, ids, st = ix.knn_batch(Q[:12], 10, stats=True, bucket_cap=1)
    assert st["fallback_queries"] == 12
    same_as_plain(ix, Q[:12], np.full(12, 10), d, ids)


def test_batch_retry_with_tighter_bound(mid):
    """Small buckets overflow; the first survivors lower the bound and the
    filter runs again for those queries only; answers stay identical."""
    X, Q, ix = mid
    ks = np.array([10, 100] * 20, np.uint32)
    d, ids, st = ix.knn_batch(Q[-40:], ks, stats=True, bucket_cap=150)
    assert st["retried_queries"] > 0, st
    same_as_plain(ix, Q[-40:], ks, d, ids)


def test_batch_via_hg_knn_mode(mid, hg):
    X, Q, ix = mid
    d, ids = ix.knn(Q[:40], 10, mode=hg.MODE_BATCH)
    pd, pi = ix.knn(Q[:40], 10)
    assert np.array_equal(bits(d), bits(pd)) and np.array_equal(ids, pi)


def test_batch_device_entry(mid):
    import torch
    X, Q, ix = mid
    q = torch.from_numpy(Q[:32]).cuda()
    ks = np.array([1, 10, 100, 7] * 8, np.uint32)
    dd = torch.empty((32, 100), dtype=torch.float32, device="cuda")
    di = torch.empty((32, 100), dtype=torch.int64, device="cuda")
    ix.knn_batch_device(q.data_ptr(), 32, ks, 100, dd.data_ptr(), di.data_ptr())
    torch.cuda.synchronize()
    same_as_plain(ix, Q[:32], ks, dd.cpu().numpy(), di.cpu().numpy())


@pytest.mark.parametrize("name", ["n20000_L64_leaf500", "n30000_L96_leaf700", "n100000_L256_leaf2000"])
def test_batch_reference_configs(hg, gpu_available, name):
    """The golden configurations (L = 64 and 96 pad the 64-wide K step)."""
    g = json.load(open(golden_path(f"ref_{name}.json")))
    X = hg.generate_walks(g["data_seed"], g["n"], g["L"])
    Q = hg.generate_queries(g["query_seed"], X, np.array(g["sigma2"]))
    ix = hg.HerculesIndex.build(X, g["leaf"])
    for k in (1, 10, 100):
        d, ids = ix.knn_batch(Q, k)
        same_as_plain(ix, Q, np.full(len(Q), k), d, ids)


@pytest.mark.parametrize("L,n,leaf", [(16, 3000, 100), (1024, 6000, 500), (4096, 3000, 300), (16384, 1000, 100)])
def test_batch_other_lengths(hg, gpu_available, L, n, leaf):
    X = hg.generate_walks(51, n, L)
    Q = hg.generate_queries(52, X, np.array([0.01, 0.1, 1.0] * 4))
    ix = hg.HerculesIndex.build(X, leaf)
    d, ids = ix.knn_batch(Q, 10)
    same_as_plain(ix, Q, np.full(len(Q), 10), d, ids)


def test_batch_edge_cases(hg, gpu_available):
    # one leaf smaller than k, duplicates: the bound pass cannot find k rows
    X = hg.generate_walks(41, 45, 32)
    X[40] = X[3]
    X[41] = X[3]
    ix = hg.HerculesIndex.build(X, 100)
    d, ids, st = ix.knn_batch(X[3:5], 50, stats=True)
    pd, pi = ix.knn(X[3:5], 50)
    assert np.array_equal(bits(d), bits(pd)) and np.array_equal(ids, pi)
    # empty batch
    d, ids = ix.knn_batch(np.zeros((0, 32), np.float32), 5)
    assert d.shape == (0, 5)


def test_autotune_keeps_answers(mid):
    """The autotuner picks launch parameters from its candidates; answers of
    both paths are unchanged afterwards."""
    import torch
    X, Q, ix = mid
    before = ix.knn_batch(Q[:64], 10)
    q = torch.from_numpy(Q[:64]).cuda()
    t = ix.autotune_device(q.data_ptr(), 64, None, 10)
    assert t["filter_tiles_per_item"] in (16, 32, 64) and t["bound_tiles_per_item"] in (4, 8, 16)
    assert t["rerank_blocks_per_sm"] in (4, 8, 16) and t["approx_blocks_per_sm"] in (1, 2, 4)
    assert t["batch_ms"] > 0 and t["plain_ms"] > 0 and ix.tuning() == t
    after = ix.knn_batch(Q[:64], 10)
    assert np.array_equal(bits(before[0]), bits(after[0])) and np.array_equal(before[1], after[1])
    pd, pi = ix.knn(Q[:16], 10)
    same_as_plain(ix, Q[:16], np.full(16, 10), after[0][:16], after[1][:16])
    with pytest.raises(Exception):
        ix.set_tuning(filter_tiles_per_item=3)
    ix.set_tuning(filter_tiles_per_item=32, bound_tiles_per_item=8, rerank_blocks_per_sm=8, approx_blocks_per_sm=2)


def test_batch_unit_vectors(hg, gpu_available, oracle_mod):
    """Unit-normalised Gaussian vectors (norms 1, not sqrt(L)): the batched
    answers equal the plain path's and the oracle's."""
    X = hg.generate_unit_vectors(91, 60_000, 96)
    Q = hg.generate_unit_queries(92, X, np.full(40, 0.1))
    ix = hg.HerculesIndex.build(X, 5_000)
    ks = np.array([1, 10, 100, 10] * 10, np.uint32)
    d, ids, st = ix.knn_batch(Q, ks, stats=True)
    same_as_plain(ix, Q, ks, d, ids)
    assert st["fallback_queries"] <= 4, st
    od, oid = oracle_mod.pscan(X, Q[1], 10)
    assert np.array_equal(bits(d[1, :10]), bits(od)) and np.array_equal(ids[1, :10], oid)
