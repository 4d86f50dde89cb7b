"""The oracle (CPU restatement) against the reference: golden fixtures
produced by the reference itself (tests/golden/make_golden.py), and the
reference compiled from source when its sources are present."""
import json
import os

import numpy as np
import pytest

from conftest import golden_path


def bits(x):
    return np.asarray(x, np.float32).view(np.uint32)


@pytest.fixture(scope="module")
def kat():
    return np.load(golden_path("kat_primitives.npz"))


@pytest.mark.parametrize("L", [64, 256])
def test_ed_matches_reference_kat(oracle_mod, kat, L):
    X, Q, bounds, want = kat[f"L{L}_X"], kat[f"L{L}_Q"], kat[f"L{L}_bounds"], kat[f"L{L}_ed"]
    got = np.array([[[oracle_mod.ed(q, x, b) for b in bounds] for x in X] for q in Q], np.float32)
    assert np.array_equal(bits(got), bits(want))


@pytest.mark.parametrize("L", [64, 256])
def test_mean_stdev_matches_reference_kat(oracle_mod, kat, L):
    Q, segs, want = kat[f"L{L}_Q"], kat[f"L{L}_segs"], kat[f"L{L}_ms"]
    got = np.array([[oracle_mod.mean_stdev(q, int(a), int(b)) for a, b in segs] for q in Q], np.float32)
    assert np.array_equal(bits(got), bits(want))


@pytest.mark.parametrize("L", [64, 256])
def test_paa_sax_lbsax_match_reference_kat(oracle_mod, kat, L):
    X, Q = kat[f"L{L}_X"], kat[f"L{L}_Q"]
    paa = np.array([oracle_mod.paa(q) for q in Q])
    assert np.array_equal(bits(paa), bits(kat[f"L{L}_paa"]))
    words = np.array([oracle_mod.sax(x) for x in X])
    assert np.array_equal(words, kat[f"L{L}_sax"])
    lb = np.array([[oracle_mod.lb_sax(p, w, L) for w in words] for p in paa], np.float32)
    assert np.array_equal(bits(lb), bits(kat[f"L{L}_lbsax"]))


@pytest.mark.parametrize("L", [64, 256])
def test_lb_eapca_matches_reference_kat(oracle_mod, kat, L):
    Q, P, S, want = kat[f"L{L}_Q"], kat[f"L{L}_eapca_points"], kat[f"L{L}_eapca_sk"], kat[f"L{L}_eapca_lb"]
    for t in range(P.shape[0]):
        nseg = int(np.argmax(P[t] == L)) + 1
        got = np.array([oracle_mod.lb_eapca(q, P[t][:nseg], S[t][:nseg]) for q in Q], np.float32)
        assert np.array_equal(bits(got), bits(want[t])), t


def test_topk_insert_matches_reference_kat(oracle_mod, kat):
    import ctypes
    seq = kat["topk_seq"]
    for k in (1, 3, 5):
        dist = np.full(k, np.finfo(np.float32).max, np.float32)
        ids = np.full(k, -1, np.int64)
        cur = ctypes.c_int(0)
        for i, d in enumerate(seq):
            if d < dist[k - 1]:
                oracle_mod.olib().or_topk_insert(oracle_mod._p(dist), oracle_mod._p(ids), None, ctypes.byref(cur), k,
                                                 float(d), i, 0, 0)
        assert np.array_equal(dist, kat[f"topk_k{k}_dist"])
        assert np.array_equal(ids, kat[f"topk_k{k}_ids"])


def test_breakpoints_fixture_is_the_standard_normal_quantiles(oracle_mod):
    import scipy.special as sp
    bp = oracle_mod.breakpoints()
    want = np.array([sp.ndtri((s + 1) / 256.0) for s in range(255)]).astype(np.float32)
    assert np.array_equal(bits(bp), bits(want))


REF_CONFIGS = ["n20000_L64_leaf500", "n30000_L96_leaf700", "n100000_L256_leaf2000"]


@pytest.mark.parametrize("name", REF_CONFIGS)
def test_oracle_index_and_answers_match_reference_golden(oracle_mod, hg, tmp_path, name):
    """Oracle build == reference build (leaf files byte for byte, root.idx
    field by field); oracle exact search == reference CLI answers, including
    the per-query loaded-leaf and loaded-row counters."""
    import hashlib
    import sys
    sys.path.insert(0, os.path.dirname(golden_path("")))
    from make_golden import root_fields_digest
    g = json.load(open(golden_path(f"ref_{name}.json")))
    X = hg.generate_walks(g["data_seed"], g["n"], g["L"])
    assert hashlib.sha256(X.tobytes()).hexdigest() == g["data_sha256"]
    oi = oracle_mod.OracleIndex.build(X, g["leaf"])
    d = str(tmp_path) + "/"
    oi.write(d, g["buffer_mb"])
    assert hashlib.sha256(open(d + "leaves_raw.idx", "rb").read()).hexdigest() == g["stock"]["leaves_raw_sha256"]
    assert hashlib.sha256(open(d + "leaves_sims.idx", "rb").read()).hexdigest() == g["stock"]["leaves_sims_sha256"]
    assert root_fields_digest(d + "root.idx") == g["stock"]["root_fields_sha256"]
    assert g["nofma"] == g["stock"]
    Q = hg.generate_queries(g["query_seed"], X, np.array(g["sigma2"]))
    assert hashlib.sha256(Q.tobytes()).hexdigest() == g["queries_sha256"]
    rd = oracle_mod.OracleIndex.read(d)
    for j in range(g["nq"]):
        dist, rows, fp, st = rd.knn(Q[j], g["k"], tie_lowest=False)
        assert ["%f" % np.sqrt(np.float32(v)) for v in dist] == g["answers"]["exact_distance"][j]
        assert [str(int(v)) for v in fp] == g["answers"]["exact_node_file_pos"][j]
        assert st["loaded_leaves"] == int(g["answers"]["loaded_nodes"][j])
        assert st["loaded_rows"] == int(g["answers"]["loaded_ts"][j])


def test_oracle_matches_reference_at_1M_walks_leaf_100000(oracle_mod, hg, tmp_path):
    """The plain method's CPU-runnable configuration (1M x 256 walks, leaf
    100,000, 100 fresh random-walk queries, k = 1 and 10): the oracle's index
    files are the reference's and its answers and load counters are the
    reference CLI's."""
    import hashlib
    import sys
    sys.path.insert(0, os.path.dirname(golden_path("")))
    from make_golden import root_fields_digest
    g = json.load(open(golden_path("ref_walks1M_L256_leaf100000.json")))
    X = hg.generate_walks(g["data_seed"], g["n"], g["L"])
    assert hashlib.sha256(X.tobytes()).hexdigest() == g["data_sha256"]
    Q = hg.generate_walks(g["query_seed"], g["nq"], g["L"])
    assert hashlib.sha256(Q.tobytes()).hexdigest() == g["queries_sha256"]
    oi = oracle_mod.OracleIndex.build(X, g["leaf"])
    d = str(tmp_path) + "/"
    oi.write(d, g["buffer_mb"])
    del oi
    assert hashlib.sha256(open(d + "leaves_raw.idx", "rb").read()).hexdigest() == g["stock"]["leaves_raw_sha256"]
    assert hashlib.sha256(open(d + "leaves_sims.idx", "rb").read()).hexdigest() == g["stock"]["leaves_sims_sha256"]
    assert root_fields_digest(d + "root.idx") == g["stock"]["root_fields_sha256"]
    rd = oracle_mod.OracleIndex.read(d)
    assert rd.num_leaves() == g["num_leaves"]
    for k in g["ks"]:
        want = g["answers"]["k%d" % k]
        for j in range(g["nq"]):
            dist, rows, fp, st = rd.knn(Q[j], k, tie_lowest=False)
            assert ["%f" % np.sqrt(np.float32(v)) for v in dist] == want["exact_distance"][j], (k, j)
            assert [str(int(v)) for v in fp] == want["exact_node_file_pos"][j], (k, j)
            assert st["loaded_leaves"] == int(want["loaded_nodes"][j]), (k, j)
            assert st["loaded_rows"] == int(want["loaded_ts"][j]), (k, j)


@pytest.mark.parametrize("L,unit", [(256, False), (96, True), (1024, False), (16, False)])
def test_generator_restatement_matches_library_generator(oracle_mod, hg, L, unit):
    """oracle_gen.c gives the bits of hercules_b200's generator (its host
    path; the device path equals the host path in the GPU tests)."""
    n = 2000
    want = hg.generate_unit_vectors(1184, n, L, first=77) if unit else hg.generate_walks(1184, n, L, first=77)
    got = oracle_mod.gen_rows(1184, n, L, first=77, unit=unit)
    assert np.array_equal(bits(got), bits(want))
    X = hg.generate_unit_vectors(1184, n, L) if unit else hg.generate_walks(1184, n, L)
    s2 = np.array([0.01, 0.1, 1.0, 0.3] * 6)
    qw = (hg.generate_unit_queries if unit else hg.generate_queries)(14784, X, s2)
    qg, base = oracle_mod.gen_queries(1184, 14784, n, L, s2, unit=unit)
    assert np.array_equal(bits(qg), bits(qw))
    assert base.max() < n


@pytest.mark.parametrize("name", REF_CONFIGS + ["walks1M_L256_leaf100000"])
def test_multithreaded_build_writes_the_reference_index(oracle_mod, tmp_path, name):
    """or_build_mt (the benchmark's CPU-side build) writes the reference's
    leaves_raw.idx / leaves_sims.idx byte for byte and its root.idx field by
    field, from data made by the oracle's own generator."""
    import hashlib
    import sys
    sys.path.insert(0, os.path.dirname(golden_path("")))
    from make_golden import root_fields_digest
    g = json.load(open(golden_path(f"ref_{name}.json")))
    X = oracle_mod.gen_rows(g["data_seed"], g["n"], g["L"])
    assert hashlib.sha256(X.tobytes()).hexdigest() == g["data_sha256"]
    for keep in (False, True):
        oi = oracle_mod.OracleIndex.build_mt(X, g["leaf"], threads=4, keep_rows=keep)
        d = str(tmp_path / ("k%d" % keep)) + "/"
        os.makedirs(d)
        oi.write(d, g["buffer_mb"])
        del oi
        sha = lambda p: hashlib.sha256(open(p, "rb").read()).hexdigest()
        assert sha(d + "leaves_raw.idx") == g["stock"]["leaves_raw_sha256"]
        assert sha(d + "leaves_sims.idx") == g["stock"]["leaves_sims_sha256"]
        assert root_fields_digest(d + "root.idx") == g["stock"]["root_fields_sha256"]


APPROX = {"eps0.5": (0.5, 0), "eps2": (2.0, 0), "np3": (0.0, 3), "np10": (0.0, 10)}


@pytest.mark.parametrize("name", REF_CONFIGS)
def test_oracle_approximate_searches_match_reference_golden(oracle_mod, hg, name):
    """The oracle's epsilon and nprobes searches print the reference CLI's
    answers (--epsilon 0.5 / 2, --nprobes 3 / 10) on the reference's index."""
    g = json.load(open(golden_path(f"ref_{name}.json")))
    X = hg.generate_walks(g["data_seed"], g["n"], g["L"])
    Q = hg.generate_queries(g["query_seed"], X, np.array(g["sigma2"]))
    oi = oracle_mod.OracleIndex.build(X, g["leaf"])
    differs = 0
    for mode, (eps, npr) in APPROX.items():
        want = g["approx"][mode]
        for j in range(g["nq"]):
            dist, rows, fp, st = oi.approx_knn(Q[j], g["k"], epsilon=eps, nprobes=npr, tie_lowest=False)
            assert ["%f" % np.sqrt(np.float32(v)) for v in dist] == want["exact_distance"][j], (mode, j)
            assert [str(int(v)) for v in fp] == want["exact_node_file_pos"][j], (mode, j)
            differs += want["exact_distance"][j] != g["answers"]["exact_distance"][j]
    # nprobes answers are approximate: some differ from the exact ones
    assert differs > 0


def test_tie_rule_lowest_id_on_duplicates(oracle_mod, hg):
    """Duplicate series: the reference keeps the first one met and drops
    equal distances; the lowest-id rule keeps the smallest id instead; the
    distances are the same."""
    X = hg.generate_walks(3, 3000, 64)
    X[2500] = X[10]
    X[2600] = X[10]
    oi = oracle_mod.OracleIndex.build(X, 200)
    ids = oi.row_ids()
    q = X[10] + np.float32(0.001)
    d1, r1, _, _ = oi.knn(q, 5, tie_lowest=True)
    d0, r0, _, _ = oi.knn(q, 5, tie_lowest=False)
    assert np.array_equal(d1, d0)
    assert ids[r1[0]] == 10
    assert len(set(d1.tolist())) == 5


def test_pscan_equals_exact(oracle_mod, hg):
    X = hg.generate_walks(11, 5000, 64)
    Q = hg.generate_queries(12, X, np.array([0.1] * 5))
    oi = oracle_mod.OracleIndex.build(X, 300)
    ids = oi.row_ids()
    for q in Q:
        d, i = oracle_mod.pscan(X, q, 7)
        d2, r2, _, _ = oi.knn(q, 7)
        assert np.array_equal(d, d2)
        assert np.array_equal(i, ids[r2])


def _ref_sources():
    from oracle import oracle as O
    return O.have_ref_sources()


@pytest.mark.skipif(not _ref_sources(), reason="reference sources absent (set HERCULES_REF)")
def test_oracle_primitives_against_reference_library(oracle_mod, hg):
    """Fresh random inputs against the reference's own functions."""
    oracle_mod.build(ref=True)
    r = oracle_mod.rlib()
    import ctypes
    for L in (16, 96, 1024):
        X = hg.generate_walks(101, 30, L)
        Q = hg.generate_walks(102, 10, L)
        for q in Q:
            for x in X:
                for b in (np.inf, 30.0):
                    assert bits(oracle_mod.ed(q, x, b)) == bits(r.shim_ed(oracle_mod._p(q), oracle_mod._p(x), L,
                                                                            np.float32(b)))
            for a, b in [(0, L), (1, L - 3), (L // 2, L), (2, 5)]:
                m, s = ctypes.c_float(), ctypes.c_float()
                r.shim_mean_stdev(oracle_mod._p(q), a, b, ctypes.byref(m), ctypes.byref(s))
                mo, so = oracle_mod.mean_stdev(q, a, b)
                assert bits(mo) == bits(m.value) and bits(so) == bits(s.value)
