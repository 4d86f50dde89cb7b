"""Sizes past the single-pass capacities, against the oracle.

k above 224 (the per-warp candidate lists hold 256 entries) is answered in
rounds above the previous round's last distance; more than 1,024 candidate
leaves take the LSD radix branch of the candidate sort; more than 8,192
leaves put the sort's and the batched grouping's arrays in global memory.
The reference has none of these limits (queue_bounded_sorted_insert,
hercules_query_engine.c:4034-4082, takes any k; its tree has no leaf cap)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bits(x):
    return np.asarray(x, np.float32).view(np.uint32)


def check_against_oracle(oi, Q, k, d, ids):
    """Distances bit for bit and ids; the oracle marks missing entries with
    row -1 (distance FLT_MAX), the library with +inf / -1."""
    ids_map = oi.row_ids()
    for j, q in enumerate(Q):
        od, orow, _, _ = oi.knn(q, k, tie_lowest=True)
        ok = orow >= 0
        assert np.array_equal(bits(d[j][ok]), bits(od[ok])), (j, k)
        assert np.array_equal(ids[j][ok], ids_map[orow[ok]]), (j, k)
        assert np.all(np.isinf(d[j][~ok])) and np.all(ids[j][~ok] == -1), (j, k)


@pytest.fixture(scope="module")
def small(hg, oracle_mod, gpu_available):
    X = hg.generate_walks(1184, 40000, 64)
    Q = np.concatenate([hg.generate_queries(14784, X, np.array([0.01, 0.1, 1.0, 1.0])),
                        hg.generate_walks(99991, 2, 64)])
    ix = hg.HerculesIndex.build(X, 500)
    oi = oracle_mod.OracleIndex.build(X, 500)
    yield X, Q, ix, oi
    ix.close()


@pytest.mark.parametrize("k", [224, 225, 448, 500, 1000])
def test_large_k_plain_path_matches_oracle(small, k):
    X, Q, ix, oi = small
    for lbsax in (False, True):
        d, ids = ix.knn(Q, k, use_lb_sax=lbsax)
        check_against_oracle(oi, Q, k, d, ids)


def test_large_k_pscan_matches_oracle(small, oracle_mod):
    X, Q, ix, oi = small
    d, ids = ix.pscan(Q, 300)
    for j, q in enumerate(Q):
        od, oid = oracle_mod.pscan(X, q, 300)
        assert np.array_equal(bits(d[j]), bits(od)) and np.array_equal(ids[j], oid)


def test_large_kmax_batch_equals_plain_path(small):
    X, Q, ix, oi = small
    ks = np.array([1, 300, 10, 700, 224, 225], np.uint32)
    bd, bi = ix.knn_batch(Q, ks)
    assert bd.shape == (len(Q), 700)
    for j, k in enumerate(ks):
        d, ids = ix.knn(Q[j:j + 1], int(k))
        assert np.array_equal(bits(bd[j, :k]), bits(d[0])) and np.array_equal(bi[j, :k], ids[0])
        assert np.all(np.isinf(bd[j, k:])) and np.all(bi[j, k:] == -1)


def test_k_beyond_the_distinct_distances(hg, oracle_mod, gpu_available):
    """Fewer distinct distances than k: the rounds stop and the rest is
    +inf / -1 (duplicates collapse to their lowest id)."""
    X = hg.generate_walks(5, 600, 32)
    X[300:400] = X[0:100]  # 100 duplicated rows
    ix = hg.HerculesIndex.build(X, 64)
    oi = oracle_mod.OracleIndex.build(X, 64)
    Q = hg.generate_queries(6, X, np.array([0.1, 1.0]))
    d, ids = ix.knn(Q, 800)
    check_against_oracle(oi, Q, 800, d, ids)
    assert np.isinf(d[:, 500:]).all() and (ids[:, 500:] == -1).all()
    ix.close()


def test_many_candidate_leaves_radix_branch(hg, oracle_mod, gpu_available):
    """About 4,000 leaves of at most 100 rows: fresh random-walk queries keep
    well over 1,024 candidate leaves, so the candidate sort runs its LSD
    radix passes."""
    X = hg.generate_walks(1184, 300000, 64)
    ix = hg.HerculesIndex.build(X, 100)
    oi = oracle_mod.OracleIndex.build(X, 100)
    assert ix.info.num_leaves > 2048
    Q = np.concatenate([hg.generate_walks(99991, 4, 64), hg.generate_queries(14784, X, np.array([1.0, 1.0]))])
    for k in (1, 10):
        d, ids, st = ix.knn(Q, k, use_lb_sax=True, stats=True)
        check_against_oracle(oi, Q, k, d, ids)
        assert st["leaves_scanned"] / len(Q) > 1024, st["leaves_scanned"]
    bd, bi = ix.knn_batch(Q, 10)
    d, ids = ix.knn(Q, 10)
    assert np.array_equal(bits(bd), bits(d)) and np.array_equal(bi, ids)
    ix.close()


def test_more_than_8192_leaves(hg, oracle_mod, gpu_available):
    """About 15,000 leaves: the candidate sort and the batched grouping use
    global scratch; plain, batched and PSCAN answers equal the oracle's."""
    X = hg.generate_walks(1184, 600000, 16)
    ix = hg.HerculesIndex.build(X, 64)
    oi = oracle_mod.OracleIndex.build(X, 64)
    assert ix.info.num_leaves > 8192 and ix.info.num_leaves == oi.num_leaves()
    Q = np.concatenate([hg.generate_walks(99991, 3, 16), hg.generate_queries(14784, X, np.array([0.1, 1.0, 1.0]))])
    for k in (1, 10, 250):
        d, ids = ix.knn(Q, k, use_lb_sax=True)
        check_against_oracle(oi, Q, k, d, ids)
    bd, bi = ix.knn_batch(Q, np.array([1, 10, 100] * 2, np.uint32))
    for j, k in enumerate([1, 10, 100] * 2):
        d, ids = ix.knn(Q[j:j + 1], k)
        assert np.array_equal(bits(bd[j, :k]), bits(d[0])) and np.array_equal(bi[j, :k], ids[0])
    ix.close()


@pytest.mark.parametrize("L_max", [2, 8, 40])
def test_greedy_seeding_keeps_the_answers(small, L_max):
    """approx_leaves > 1 scans that many leaves best-first before filtering
    the rest against the tighter bound: the answers are those of the
    reference's serial search (the oracle) and of the unseeded path."""
    X, Q, ix, oi = small
    for k in (1, 10, 100):
        d0, i0 = ix.knn(Q, k, use_lb_sax=True)
        d, ids = ix.knn(Q, k, use_lb_sax=True, approx_leaves=L_max)
        check_against_oracle(oi, Q, k, d, ids)
        assert np.array_equal(bits(d), bits(d0)) and np.array_equal(ids, i0)
