"""GPU parity: the B200 path (through the C ABI) against the oracle and the
reference's golden outputs.  Bit-exact for distances (reference summation
order), identical answer ids (ties to the lowest dataset id), identical
index files."""
import hashlib
import json
import os
import sys

import numpy as np
import pytest

from conftest import golden_path

pytestmark = pytest.mark.gpu

REF_CONFIGS = ["n20000_L64_leaf500", "n30000_L96_leaf700", "n100000_L256_leaf2000"]


def bits(x):
    return np.asarray(x, np.float32).view(np.uint32)


def golden(name):
    return json.load(open(golden_path(f"ref_{name}.json")))


@pytest.fixture(scope="module")
def built(hg, oracle_mod, gpu_available):
    """Per config: data, queries, product index, oracle index."""
    out = {}
    for name in REF_CONFIGS:
        g = golden(name)
        X = hg.generate_walks(g["data_seed"], g["n"], g["L"])
        Q = hg.generate_queries(g["query_seed"], X, np.array(g["sigma2"]))
        ix = hg.HerculesIndex.build(X, g["leaf"])
        oi = oracle_mod.OracleIndex.build(X, g["leaf"])
        out[name] = (g, X, Q, ix, oi)
    return out


def test_device_generator_matches_host(hg, gpu_available):
    import torch
    n, L = 1000, 256
    t = torch.empty((n, L), dtype=torch.float32, device="cuda")
    hg.generate_walks_device(1184, n, L, t.data_ptr())
    torch.cuda.synchronize()
    host = hg.generate_walks(1184, n, L)
    assert np.array_equal(t.cpu().numpy().view(np.uint32), host.view(np.uint32))
    sig = np.array([0.01, 0.1, 1.0] * 10)
    qd = torch.empty((30, L), dtype=torch.float32, device="cuda")
    hg.generate_queries_device(7, t.data_ptr(), n, L, sig, qd.data_ptr())
    torch.cuda.synchronize()
    qh = hg.generate_queries(7, host, sig)
    assert np.array_equal(qd.cpu().numpy().view(np.uint32), qh.view(np.uint32))


@pytest.mark.parametrize("unit", [False, True])
def test_seeded_query_generator_matches_generator_over_the_collection(hg, gpu_available, unit):
    """hg_generate_queries_seeded (base rows regenerated from the data seed,
    for row-range shards) gives the bits of the generator given the whole
    collection, on the device and on the host."""
    import torch
    n, L = 4000, 96
    X = hg.generate_unit_vectors(1184, n, L) if unit else hg.generate_walks(1184, n, L)
    s2 = np.array([0.01, 0.1, 1.0] * 11)
    want = (hg.generate_unit_queries if unit else hg.generate_queries)(77, X, s2)
    t = torch.empty((len(s2), L), dtype=torch.float32, device="cuda")
    hg.generate_queries_seeded_device(1184, 77, n, L, s2, t.data_ptr(), unit=unit)
    torch.cuda.synchronize()
    assert np.array_equal(t.cpu().numpy().view(np.uint32), want.view(np.uint32))
    host = hg.generate_queries_seeded(1184, 77, n, L, s2, unit=unit)
    assert np.array_equal(host.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("name", REF_CONFIGS)
def test_build_reproduces_reference_index_files(built, tmp_path, name):
    sys.path.insert(0, os.path.dirname(golden_path("")))
    from make_golden import root_fields_digest
    g, X, Q, ix, oi = built[name]
    d = str(tmp_path) + "/"
    ix.write(d, g["buffer_mb"])
    sha = lambda p: hashlib.sha256(open(p, "rb").read()).hexdigest()
    assert sha(d + "leaves_raw.idx") == g["stock"]["leaves_raw_sha256"]
    assert sha(d + "leaves_sims.idx") == g["stock"]["leaves_sims_sha256"]
    assert root_fields_digest(d + "root.idx") == g["stock"]["root_fields_sha256"]
    assert ix.info.num_leaves == g["num_leaves"]


@pytest.mark.parametrize("name", REF_CONFIGS)
def test_leaves_envelopes_ids_match_oracle(built, name):
    g, X, Q, ix, oi = built[name]
    assert ix.leaves() == oi.leaves()
    for i in range(ix.info.num_leaves):
        p1, e1 = ix.leaf_envelope(i)
        p2, e2 = oi.leaf_envelope(i)
        assert np.array_equal(p1, p2)
        assert np.array_equal(bits(e1), bits(e2))
    assert np.array_equal(ix.row_ids(), oi.row_ids())
    rows, sax = ix.rows()
    assert np.array_equal(bits(rows), bits(oi.rows()))


@pytest.mark.parametrize("name", REF_CONFIGS)
def test_route_and_leaf_lower_bounds_match_oracle(built, name):
    g, X, Q, ix, oi = built[name]
    leaves = ix.route(Q)
    for j, q in enumerate(Q):
        _, _, _, st = oi.knn(q, 1)
        assert leaves[j] == st["approx_leaf"]
        assert np.array_equal(bits(ix.leaf_lower_bounds(q)), bits(oi.leaf_lbs(q)))


@pytest.mark.parametrize("name", REF_CONFIGS)
@pytest.mark.parametrize("k", [1, 10, 100])
@pytest.mark.parametrize("lbsax", [False, True])
def test_knn_matches_oracle(built, name, k, lbsax):
    g, X, Q, ix, oi = built[name]
    ids_map = oi.row_ids()
    d, ids, st = ix.knn(Q, k, use_lb_sax=lbsax, stats=True)
    for j, q in enumerate(Q):
        od, orow, _, _ = oi.knn(q, k, tie_lowest=True)
        assert np.array_equal(bits(d[j]), bits(od)), (j, d[j][:4], od[:4])
        assert np.array_equal(ids[j], ids_map[orow]), j
    assert st["rows_visited"] > 0


APPROX = {"eps0.5": (0.5, 0), "eps2": (2.0, 0), "np3": (0.0, 3), "np10": (0.0, 10)}


@pytest.mark.parametrize("name", REF_CONFIGS)
@pytest.mark.parametrize("mode", sorted(APPROX))
def test_approximate_searches_match_oracle_and_reference(built, name, mode):
    """epsilon-approximate and nprobes searches (host tree walk, leaf scans on
    the GPU): bit-identical to the oracle's, the reference CLI's printed
    answers (golden), and the same number of leaves scanned."""
    g, X, Q, ix, oi = built[name]
    eps, npr = APPROX[mode]
    ids_map = oi.row_ids()
    want = g["approx"][mode]
    for k in (1, g["k"], 50):
        d, ids, pos, st = ix.knn(Q, k, with_leaf_pos=True, stats=True, epsilon=eps, nprobes=npr)
        loaded = 0
        for j, q in enumerate(Q):
            od, orow, ofp, ost = oi.approx_knn(q, k, epsilon=eps, nprobes=npr, tie_lowest=True)
            assert np.array_equal(bits(d[j]), bits(od)), (mode, k, j)
            assert np.array_equal(ids[j], ids_map[orow]), (mode, k, j)
            loaded += ost["loaded_leaves"] - 1  # the oracle counts the approximate leaf
            if k == g["k"]:
                assert ["%f" % np.sqrt(v) for v in d[j]] == want["exact_distance"][j], (mode, j)
                assert [str(int(v)) for v in pos[j]] == want["exact_node_file_pos"][j], (mode, j)
        assert st["leaves_scanned"] == loaded, (mode, k)


def test_approximate_search_arguments(built):
    g, X, Q, ix, oi = built[REF_CONFIGS[0]]
    with pytest.raises(Exception):
        ix.knn(Q[:1], 5, epsilon=-1.0)
    # epsilon 0 and nprobes 0 are the exact search
    d0, i0 = ix.knn(Q[:4], 5)
    d1, i1 = ix.knn(Q[:4], 5, epsilon=0.0, nprobes=0)
    assert np.array_equal(bits(d0), bits(d1)) and np.array_equal(i0, i1)


@pytest.mark.parametrize("name", REF_CONFIGS)
def test_knn_matches_reference_cli(built, name):
    """Printed distances (sqrt, %f) and the answer leaf's file_pos of the
    reference CLI (golden), k and queries of the fixture."""
    g, X, Q, ix, oi = built[name]
    d, ids, pos = ix.knn(Q, g["k"], with_leaf_pos=True)
    for j in range(g["nq"]):
        assert ["%f" % np.sqrt(v) for v in d[j]] == g["answers"]["exact_distance"][j]
        assert [str(int(v)) for v in pos[j]] == g["answers"]["exact_node_file_pos"][j]


@pytest.mark.parametrize("name", REF_CONFIGS)
def test_pscan_matches_oracle(built, oracle_mod, name):
    g, X, Q, ix, oi = built[name]
    d, ids = ix.pscan(Q[:8], 10)
    for j in range(8):
        od, oid = oracle_mod.pscan(X, Q[j], 10)
        assert np.array_equal(bits(d[j]), bits(od))
        assert np.array_equal(ids[j], oid)


def test_fp64_error_bound(built, oracle_mod):
    g, X, Q, ix, oi = built["n100000_L256_leaf2000"]
    d, ids = ix.knn(Q, 10)
    bd, bi = oracle_mod.brute_force_fp64(X, Q, 10)
    rel = np.abs(d.astype(np.float64) - bd) / np.maximum(bd, 1e-30)
    assert rel.max() < 1e-5


def test_read_reference_format_and_query(hg, oracle_mod, tmp_path, gpu_available):
    """An index written in the reference's format (by the oracle, whose files
    are byte-identical to the reference's) loads and answers identically."""
    X = hg.generate_walks(21, 6000, 128)
    Q = hg.generate_queries(22, X, np.array([0.1, 1.0, 0.01, 0.1]))
    oi = oracle_mod.OracleIndex.build(X, 400)
    d = str(tmp_path) + "/"
    oi.write(d, 100.0)
    ix = hg.HerculesIndex.read(d)
    assert ix.info.has_ids == 0
    assert ix.leaves() == oi.leaves()
    dist, ids = ix.knn(Q, 5)
    for j, q in enumerate(Q):
        od, orow, _, _ = oi.knn(q, 5)
        assert np.array_equal(bits(dist[j]), bits(od))
        assert np.array_equal(ids[j], orow)  # without leaves_ids.idx an id is the leaf-ordered row


def test_write_read_roundtrip_keeps_ids(hg, tmp_path, gpu_available):
    X = hg.generate_walks(31, 4000, 64)
    Q = hg.generate_queries(32, X, np.array([0.1] * 4))
    ix = hg.HerculesIndex.build(X, 300)
    d = str(tmp_path) + "/"
    ix.write(d)
    ix2 = hg.HerculesIndex.read(d)
    assert ix2.info.has_ids == 1
    a = ix.knn(Q, 7)
    b = ix2.knn(Q, 7)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_edge_cases(hg, oracle_mod, gpu_available):
    # one leaf (n < leaf size), n not a multiple of 32, k > n, duplicates
    X = hg.generate_walks(41, 45, 32)
    X[40] = X[3]
    X[41] = X[3]
    ix = hg.HerculesIndex.build(X, 100)
    assert ix.info.num_leaves == 1
    d, ids = ix.knn(X[3:4], 50)
    ok = np.isfinite(d[0])
    assert ok.sum() == 43  # 45 rows, two duplicates of row 3 collapse into it
    assert ids[0][0] == 3 and d[0][0] == 0.0
    assert np.all(ids[0][~ok] == -1)
    od, orow, _, _ = oracle_mod.OracleIndex.build(X, 100).knn(X[3], 50)
    assert np.array_equal(bits(d[0][ok]), bits(od[:43]))


@pytest.mark.parametrize("L,n,leaf", [(16, 3000, 100), (1024, 3000, 250), (4096, 2000, 200), (16384, 800, 100)])
def test_other_lengths(hg, oracle_mod, gpu_available, L, n, leaf):
    """Short and long series (L >= 4096 runs the distance stream with 8-lane
    slots, each list spread over every warp)."""
    X = hg.generate_walks(51, n, L)
    Q = hg.generate_queries(52, X, np.array([0.01, 0.1, 1.0] * 3))
    ix = hg.HerculesIndex.build(X, leaf)
    oi = oracle_mod.OracleIndex.build(X, leaf)
    assert ix.leaves() == oi.leaves()
    ids_map = oi.row_ids()
    for k, lbsax in ((10, True), (1, False), (100, True)):
        d, ids = ix.knn(Q, k, use_lb_sax=lbsax)
        for j, q in enumerate(Q):
            od, orow, _, _ = oi.knn(q, k)
            assert np.array_equal(bits(d[j]), bits(od)), (k, j)
            assert np.array_equal(ids[j], ids_map[orow]), (k, j)


def test_cli_is_a_drop_in_for_the_reference_cli(hg, tmp_path, gpu_available):
    """bin/hercules with the reference's flags (build, then query) prints
    the same Query_exact_distance / Query_exact_node_file_pos lines as the
    reference CLI (golden)."""
    import subprocess
    from hercules_b200 import build as B
    g = golden("n20000_L64_leaf500")
    X = hg.generate_walks(g["data_seed"], g["n"], g["L"])
    Q = hg.generate_queries(g["query_seed"], X, np.array(g["sigma2"]))
    data, qf = str(tmp_path / "data.bin"), str(tmp_path / "q.bin")
    X.tofile(data)
    Q.tofile(qf)
    idx = str(tmp_path / "idx") + "/"
    cli = B.build_cli()
    r = subprocess.run([cli, "--mode", "0", "--serial", "1", "--sims", "--num-threads", "2", "--num-write-threads",
                        "1", "--initial-db-size", "120000", "--buffer-size", "500", "--leaf-size", str(g["leaf"]),
                        "--timeseries-size", str(g["L"]), "--dataset-size", str(g["n"]), "--dataset", data,
                        "--index-path", idx], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([cli, "--mode", "1", "--serial", "1", "--num-threads", "1", "--k", str(g["k"]), "--queries",
                        qf, "--queries-size", str(g["nq"]), "--index-path", idx], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = {}
    for line in r.stdout.splitlines():
        p = line.split("\t")
        if len(p) == 5 and p[0] in ("Query_exact_distance", "Query_exact_node_file_pos"):
            got[(p[0], int(p[3]), int(p[4]))] = p[1]
    for j in range(g["nq"]):
        for r_ in range(g["k"]):
            assert got[("Query_exact_distance", j + 1, r_ + 1)] == g["answers"]["exact_distance"][j][r_]
            assert got[("Query_exact_node_file_pos", j + 1, r_ + 1)] == g["answers"]["exact_node_file_pos"][j][r_]
    # the approximate searches with the reference's flags
    for mode, want in g["approx"].items():
        r = subprocess.run([cli, "--mode", "1", "--serial", "1", "--num-threads", "1", "--k", str(g["k"]),
                            "--queries", qf, "--queries-size", str(g["nq"]), "--index-path", idx, "--delta", "1",
                            *want["args"]], capture_output=True, text=True)
        assert r.returncode == 0, (mode, r.stderr)
        got = {}
        for line in r.stdout.splitlines():
            p = line.split("\t")
            if len(p) == 5 and p[0] in ("Query_exact_distance", "Query_exact_node_file_pos"):
                got[(p[0], int(p[3]), int(p[4]))] = p[1]
        for j in range(g["nq"]):
            assert [got[("Query_exact_distance", j + 1, r_ + 1)] for r_ in range(g["k"])] == \
                want["exact_distance"][j], (mode, j)
            assert [got[("Query_exact_node_file_pos", j + 1, r_ + 1)] for r_ in range(g["k"])] == \
                want["exact_node_file_pos"][j], (mode, j)


def test_device_unit_generator_matches_host(hg, gpu_available):
    import torch
    n, L = 500, 96
    t = torch.empty((n, L), dtype=torch.float32, device="cuda")
    hg.generate_unit_vectors_device(77, n, L, t.data_ptr())
    torch.cuda.synchronize()
    host = hg.generate_unit_vectors(77, n, L)
    assert np.array_equal(t.cpu().numpy().view(np.uint32), host.view(np.uint32))
    sig = np.full(12, 0.1)
    qd = torch.empty((12, L), dtype=torch.float32, device="cuda")
    hg.generate_unit_queries_device(8, t.data_ptr(), n, L, sig, qd.data_ptr())
    torch.cuda.synchronize()
    assert np.array_equal(qd.cpu().numpy().view(np.uint32), hg.generate_unit_queries(8, host, sig).view(np.uint32))
