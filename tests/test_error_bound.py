"""The certified error bound of the batched BF16 filter, checked on the CPU.

For BF16 roundings q~, x~ (round to nearest even) the filter's estimate
    d~ = |q|^2 + |x|^2 - 2 q~.x~
must stay within
    err = 2 (1 + 2^-20) (|q~| |x - x~| + |q - q~| |x~| + |q - q~| |x - x~| + L 2^-20 |q~| |x~|)
          + (L/8 + 16) 2^-22 (|q|^2 + |x|^2 + D) + 1e-5
of the reference's FP32 distance D (oracle ed, ts.c:83-109 order) for every
pair; the kernel uses per-tile maxima of the row terms, which only widens it.
The FP32 accumulation term is exercised here with the dot product rounded
once to FP32 (the tensor cores' own accumulation error is what L 2^-20 covers).
"""
import numpy as np
import pytest


def bf16(a):
    """float32 -> nearest-even BF16, returned as float32."""
    b = np.ascontiguousarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return r.astype(np.uint32).view(np.float32)


def err_bound(q, x, D):
    L = q.shape[-1]
    qt, xt = bf16(q).astype(np.float64), bf16(x).astype(np.float64)
    q64, x64 = q.astype(np.float64), x.astype(np.float64)
    nqt, nxt = np.linalg.norm(qt), np.linalg.norm(xt)
    rq, rx = np.linalg.norm(q64 - qt), np.linalg.norm(x64 - xt)
    c_acc = L * 2.0 ** -20
    c_sq = (L / 8 + 16) * 2.0 ** -22
    return (2 * (1 + 2 ** -20) * (nqt * rx + rq * nxt + rq * rx + c_acc * nqt * nxt)
            + c_sq * (q64 @ q64 + x64 @ x64 + D) + 1e-5)


def d_tilde(q, x):
    qt, xt = bf16(q).astype(np.float64), bf16(x).astype(np.float64)
    acc = np.float32(qt @ xt)
    return np.float64(np.float32(q.astype(np.float64) @ q)) + np.float64(x.astype(np.float64) @ x) - 2.0 * acc


@pytest.mark.parametrize("L", [64, 256, 1024])
def test_bf16_filter_error_bound_holds(hg, oracle_mod, L):
    X = hg.generate_walks(1184, 400, L)
    sig = np.array([0.01, 0.1, 1.0] * 4)
    Q = np.concatenate([hg.generate_queries(14784, X, sig), hg.generate_walks(99, 4, L)])
    worst = 0.0
    for q in Q:
        for x in X:
            D = float(oracle_mod.ed(q, x))
            e = err_bound(q, x, D)
            gap = abs(d_tilde(q, x) - D)
            assert gap <= e, (gap, e)
            worst = max(worst, gap / e)
    # the bound is not vacuous: the observed error uses a visible share of it
    assert worst > 0.01


def test_bf16_rounding_matches_torch():
    import torch
    a = np.random.default_rng(3).standard_normal(10000).astype(np.float32) * 7
    t = torch.from_numpy(a).to(torch.bfloat16).to(torch.float32).numpy()
    assert np.array_equal(bf16(a).view(np.uint32), t.view(np.uint32))


def test_threshold_split_stays_inside_its_margin():
    """The screening filter subtracts each query's threshold t inside the
    tensor-core accumulation as two BF16 numbers t_hi = bf16(t) and
    t_lo = bf16(t - t_hi).  Their sum misses t by at most 2^-16 |t| (BF16
    keeps 8 significant bits: half an ulp is 2^-8 relative, twice); the
    kernel lowers t first by c_acc |t| + 2^-14 (|t| + |q~| |x~|), which
    covers that split error and the rounding of the larger partial sums."""
    rng = np.random.default_rng(11)
    t = np.concatenate([rng.normal(size=20000) * 10.0 ** rng.integers(-3, 5, size=20000),
                        np.array([0.0, 1.0, -1.0, 127.99, 8191.5])]).astype(np.float32)
    th = bf16(t)
    tl = (t - th).astype(np.float32)  # exact in FP32
    assert np.array_equal(tl.astype(np.float64), t.astype(np.float64) - th.astype(np.float64))
    split_err = np.abs(t.astype(np.float64) - th.astype(np.float64) - bf16(tl).astype(np.float64))
    assert np.all(split_err <= 2.0 ** -16 * np.abs(t.astype(np.float64)))
    for L in (96, 256, 1024, 16384):
        c_acc = L * 2.0 ** -20
        margin = c_acc * np.abs(t) + 2.0 ** -14 * np.abs(t)
        assert np.all(margin >= split_err)
