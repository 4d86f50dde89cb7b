"""bench.py's host-side pieces, on CPU: the reference arm (the reference's
query path over index files the oracle builds) must load nothing of
hercules_b200, and its queries must be the GPU arm's queries."""
import json
import os
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench_args(*argv):
    sys.path.insert(0, ROOT)
    import bench
    old = sys.argv
    sys.argv = ["bench.py", *argv]
    try:
        return bench, bench.parse()
    finally:
        sys.argv = old


def test_host_batches_equal_the_library_generator(hg, oracle_mod):
    """batch_on_host (oracle) == make_batches' recipe through the library's
    host generator: noisy queries of seed QUERY_SEED + i, then fresh walks."""
    bench, args = _bench_args("--n", "5000", "--batch", "64")
    X = hg.generate_walks(bench.DATA_SEED, args.n, args.L)
    for i in (0, 3):
        got, ks = bench.batch_on_host(args, oracle_mod, i)
        nf = bench.fresh_count(args)
        noisy = hg.generate_queries(bench.QUERY_SEED + i, X, bench.sigma2_for(args.batch - nf))
        fresh = hg.generate_walks(bench.FRESH_SEED, nf, args.L, first=i * nf)
        want = np.concatenate([noisy, fresh])
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
        assert list(ks[:9]) == [1, 1, 1, 10, 10, 10, 100, 100, 100]


def test_sample_positions_cover_every_k_and_level():
    bench, args = _bench_args()
    pos = bench.sample_positions(args, 6)
    ks = bench.batch_ks(args)
    assert set(ks[pos].tolist()) == {1, 10, 100}
    nf = bench.fresh_count(args)
    noisy = pos[pos < args.batch - nf]
    assert set((noisy % 3).tolist()) == {0, 1, 2}
    assert pos[-1] >= args.batch - nf


@pytest.mark.skipif(not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "hercules")),
                    reason="reference CLI not built")
def test_reference_arm_runs_without_the_gpu_library(oracle_mod):
    code = ("import sys, runpy; sys.argv = ['bench.py', '--impl', 'reference', '--n', '60000', '--leaf', '5000', "
            "'--steps', '2', '--warmup', '1', '--batch', '256'];\n"
            "try:\n    runpy.run_path('bench.py', run_name='__main__')\n"
            "finally:\n    print('MAPS', 'libhercules_gpu' in open('/proc/self/maps').read(), "
            "'libcuda' in open('/proc/self/maps').read())\n")
    r = subprocess.run([sys.executable, "-c", code], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = r.stdout.strip().splitlines()
    assert lines[-1] == "MAPS False False", lines[-1]
    line = json.loads(lines[-2])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["config"]["queries_per_step"] == 256
    assert set(line["index"]) >= {"root.idx", "leaves_raw.idx", "leaves_sims.idx"}
