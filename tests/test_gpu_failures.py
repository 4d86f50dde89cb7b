"""Failure detection on the GPU without a fault: a bounded wait that runs out.

Every mbarrier wait of the tensor-core filter kernel gives up after a time
limit; the kernel then drains its copies and MMAs, frees its tensor memory and
returns, and the host reports HG_ERR_TIMEOUT.  hg_filter_wait_check runs the
kernel with the limit shortened to a millisecond and one operand copy
withheld, so that one barrier phase never completes (a flag that nothing
sets).  Nothing traps or faults; the test then checks that the device still
answers correctly."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HG_OK, HG_ERR_TIMEOUT = 0, -6


def test_filter_wait_runs_out_and_the_device_stays_usable(hg, gpu_available):
    assert hg.filter_wait_check(20000, 0) == HG_OK
    assert hg.filter_wait_check(1000, 1) == HG_ERR_TIMEOUT
    assert "timed out" in hg.lib().hg_last_error().decode()
    # the same kernel, and the whole batched path, still work afterwards
    assert hg.filter_wait_check(20000, 0) == HG_OK
    X = hg.generate_walks(1184, 20000, 64)
    Q = hg.generate_queries(14784, X, np.array([0.01, 0.1, 1.0, 0.1]))
    ix = hg.HerculesIndex.build(X, 1000)
    d, ids = ix.knn(Q, 10)
    bd, bi = ix.knn_batch(Q, 10)
    assert np.array_equal(bd.view(np.uint32), d.view(np.uint32)) and np.array_equal(bi, ids)
    ix.close()


def test_pair_filter_wait_runs_out_and_the_device_stays_usable(hg, gpu_available):
    """The CTA-pair kernel: the odd CTA's first copy is withheld, the leader's
    wait runs out, both CTAs of every pair leave through the final cluster
    barrier and free their tensor memory."""
    assert hg.filter_pair_wait_check(20000, 0) == HG_OK
    assert hg.filter_pair_wait_check(1000, 1) == HG_ERR_TIMEOUT
    assert "timed out" in hg.lib().hg_last_error().decode()
    assert hg.filter_pair_wait_check(20000, 0) == HG_OK
    X = hg.generate_walks(1184, 20000, 64)
    Q = hg.generate_queries(14784, X, np.array([0.01, 0.1, 1.0, 0.1]))
    ix = hg.HerculesIndex.build(X, 1000)
    d, ids = ix.knn(Q, 10)
    for pair in (1, 2):
        ix.set_tuning(filter_cta_pair=pair)
        bd, bi = ix.knn_batch(Q, 10)
        assert np.array_equal(bd.view(np.uint32), d.view(np.uint32)) and np.array_equal(bi, ids)
    ix.close()


def test_filter_wait_check_arguments(hg, gpu_available):
    assert hg.filter_wait_check(0, 1) == -1
    assert hg.filter_wait_check(3000000, 0) == -1
    assert hg.filter_pair_wait_check(0, 1) == -1
    assert hg.filter_pair_wait_check(3000000, 0) == -1
