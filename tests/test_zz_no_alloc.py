"""The allocation-free scan (hg_pscan_noalloc) against the scan of hg_knn.

hg_pscan_noalloc exists for callers that cannot allocate device memory (code
held to a fixed memory-pool budget, or a plugin host that forbids
cudaMalloc/cudaFree on its query threads).  It keeps its working memory in
one static device array, so two calls in a row must not see each other's
state.  This file is collected last so that a failure here stops a `-x` run
only after every other test has run."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


# (rows, length, k, leaf size of the index whose scan mode is the comparison):
# short series with a small k and the largest k; long series (8-lane slots,
# the query staged in up to 64 KB of shared memory) at k = 1, 10 and 224
SHAPES = [(30000, 256, 10, 2000), (30000, 256, 224, 2000), (4000, 4096, 10, 1000),
          (1500, 16384, 1, 500), (1500, 16384, 224, 500)]


@pytest.mark.parametrize("n,L,k,leaf", SHAPES)
def test_pscan_noalloc_matches_pscan_on_two_calls_in_a_row(hg, gpu_available, n, L, k, leaf):
    import torch
    X = hg.generate_walks(1184, n, L)
    Q = hg.generate_queries(14784, X, np.array([0.01, 0.1, 1.0, 0.1, 0.01]))
    ix = hg.HerculesIndex.build(X, leaf)
    want_d, want_id = ix.pscan(Q, k)          # the existing entry point (hg_knn, scan mode)
    ix.close()
    Xd = torch.from_numpy(X).cuda()
    Qd = torch.from_numpy(Q).cuda()
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        for j in range(Q.shape[0]):
            D = torch.full((k,), -1.0, dtype=torch.float32, device="cuda")
            I = torch.full((k,), -7, dtype=torch.int64, device="cuda")
            hg.pscan_noalloc(Xd.data_ptr(), n, L, Qd[j].data_ptr(), k, D.data_ptr(), I.data_ptr(), stream)
            torch.cuda.synchronize()
            assert np.array_equal(D.cpu().numpy().view(np.uint32), want_d[j].view(np.uint32)), (call, j)
            assert np.array_equal(I.cpu().numpy(), want_id[j]), (call, j)


def test_pscan_noalloc_rejects_sizes_beyond_its_limits(hg, gpu_available):
    import torch
    X = torch.zeros((64, 32), dtype=torch.float32, device="cuda")
    D = torch.zeros(300, dtype=torch.float32, device="cuda")
    I = torch.zeros(300, dtype=torch.int64, device="cuda")
    with pytest.raises(hg.HerculesError) as e:
        hg.pscan_noalloc(X.data_ptr(), 64, 32, X[0].data_ptr(), 300, D.data_ptr(), I.data_ptr())
    assert e.value.status == -7
