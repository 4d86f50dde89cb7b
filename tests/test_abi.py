"""The C ABI library loads and exports every entry point of
include/hercules_gpu.h; host-only entry points behave (no GPU needed)."""
import os
import re

import numpy as np

from conftest import ROOT, golden_path


def declared_symbols():
    h = open(os.path.join(ROOT, "include", "hercules_gpu.h")).read()
    return sorted(set(re.findall(r"HG_API\s+[\w\s\*]+?\b(hg_\w+)\s*\(", h)))


def test_library_exports_every_declared_symbol(hg):
    import subprocess
    syms = declared_symbols()
    assert len(syms) >= 19
    out = subprocess.run(["nm", "-D", "--defined-only", hg.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r"\bT (hg_\w+)", out))
    missing = [s for s in syms if s not in exported]
    assert not missing, missing
    assert sorted(hg.EXPORTED) == syms
    for s in syms:
        assert getattr(hg.lib(), s) is not None


def test_breakpoints_equal_reference_table(hg):
    ref = np.loadtxt(golden_path("sax_breakpoints_card256.txt")).astype(np.float32)
    assert np.array_equal(hg.sax_breakpoints().view(np.uint32), ref.view(np.uint32))


def test_host_generator_is_deterministic_and_znormalised(hg):
    a = hg.generate_walks(1184, 64, 256)
    b = hg.generate_walks(1184, 64, 256)
    c = hg.generate_walks(1184, 32, 256, first=32)
    assert np.array_equal(a, b)
    assert np.array_equal(a[32:], c)
    assert np.allclose(a.mean(1), 0, atol=1e-4)
    assert np.allclose(a.std(1), 1, atol=1e-3)


def test_query_generator(hg):
    X = hg.generate_walks(5, 100, 64)
    q, base = hg.generate_queries(9, X, np.array([0.01, 1.0]), return_base=True)
    assert q.shape == (2, 64) and base.max() < 100
    assert np.allclose(q.std(1), 1, atol=1e-3)
    # small noise keeps the query close to its base row
    assert ((q[0] - X[base[0]]) ** 2).sum() < 10


def test_errors_are_status_codes_not_exits(hg):
    import pytest
    with pytest.raises(hg.HerculesError) as e:
        hg.HerculesIndex.read("/nonexistent/dir/")
    assert e.value.status == -2
    with pytest.raises(hg.HerculesError):
        hg.generate_walks(1, 4, 10)
