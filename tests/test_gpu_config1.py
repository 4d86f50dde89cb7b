"""The plain method's CPU-runnable configuration on the GPU, against the
reference's own outputs: 1M z-normalised random walks of length 256 (seed
1184), leaf size 100,000, 100 fresh random-walk queries (seed 14784),
answered one at a time with k = 1 and k = 10.

The golden file (tests/golden/ref_walks1M_L256_leaf100000.json, made by
tests/golden/make_golden.py from the reference compiled from its sources)
holds the reference build's index digests and its CLI's printed answers
(Query_exact_distance = %f of the square root, Query_exact_node_file_pos)."""
import hashlib
import json
import os
import sys

import numpy as np
import pytest

from conftest import golden_path

pytestmark = pytest.mark.gpu

NAME = "ref_walks1M_L256_leaf100000.json"


@pytest.fixture(scope="module")
def config1(hg, gpu_available):
    g = json.load(open(golden_path(NAME)))
    X = hg.generate_walks(g["data_seed"], g["n"], g["L"])
    assert hashlib.sha256(X.tobytes()).hexdigest() == g["data_sha256"]
    Q = hg.generate_walks(g["query_seed"], g["nq"], g["L"])
    assert hashlib.sha256(Q.tobytes()).hexdigest() == g["queries_sha256"]
    ix = hg.HerculesIndex.build(X, g["leaf"])
    yield g, X, Q, ix
    ix.close()


def test_gpu_build_writes_the_reference_index(config1, tmp_path):
    sys.path.insert(0, os.path.dirname(golden_path("")))
    from make_golden import root_fields_digest
    g, X, Q, ix = config1
    d = str(tmp_path) + "/"
    ix.write(d, g["buffer_mb"])
    sha = lambda p: hashlib.sha256(open(p, "rb").read()).hexdigest()
    assert sha(d + "leaves_raw.idx") == g["stock"]["leaves_raw_sha256"]
    assert sha(d + "leaves_sims.idx") == g["stock"]["leaves_sims_sha256"]
    assert root_fields_digest(d + "root.idx") == g["stock"]["root_fields_sha256"]
    assert ix.info.num_leaves == g["num_leaves"]


@pytest.mark.parametrize("k", [1, 10])
@pytest.mark.parametrize("lbsax", [False, True])
def test_plain_path_prints_the_reference_answers(config1, k, lbsax):
    g, X, Q, ix = config1
    want = g["answers"]["k%d" % k]
    d, ids, pos = ix.knn(Q, k, use_lb_sax=lbsax, with_leaf_pos=True)
    for j in range(g["nq"]):
        assert ["%f" % np.sqrt(v) for v in d[j]] == want["exact_distance"][j], (k, j)
        assert [str(int(v)) for v in pos[j]] == want["exact_node_file_pos"][j], (k, j)


def test_batched_path_equals_plain_path(config1):
    """Every query in one batched call, k = 1 and 10 mixed: distances bit for
    bit and ids identical to the plain path's."""
    g, X, Q, ix = config1
    ks = np.array([1, 10] * (g["nq"] // 2), np.uint32)
    bd, bi = ix.knn_batch(Q, ks)
    for k in (1, 10):
        sel = np.nonzero(ks == k)[0]
        d, ids = ix.knn(Q[sel], k)
        assert np.array_equal(bd[sel, :k].view(np.uint32), d.view(np.uint32))
        assert np.array_equal(bi[sel, :k], ids)


def test_fp64_error_at_1M(config1, oracle_mod):
    """Error of the returned FP32 distances against an FP64 brute force over
    all 1M rows, and recall of the ids (first 20 queries, k = 10)."""
    g, X, Q, ix = config1
    d, ids = ix.knn(Q[:20], 10)
    fd, fi = oracle_mod.brute_force_fp64(X, Q[:20], 10)
    rel = np.abs(d.astype(np.float64) - fd) / np.maximum(fd, 1e-30)
    assert rel.max() < 1e-5, rel.max()
    for j in range(20):
        assert set(ids[j].tolist()) == set(fi[j].tolist())
