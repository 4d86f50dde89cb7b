"""Two handles on two GPUs in one process: every kernel's dynamic
shared-memory limit is raised per device (cudaFuncSetAttribute acts on the
current device only), so the second device's first launches must not fail
with the 48 KB default.  Plain per-device memory only; skipped with fewer
than two GPUs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_indexes_and_the_allocation_free_scan_on_two_devices(hg, gpu_available):
    import torch
    if torch.cuda.device_count() < 2:
        pytest.skip("needs two GPUs")
    X = hg.generate_walks(1184, 20000, 256)
    Q = hg.generate_queries(14784, X, np.array([0.01, 0.1, 1.0]))
    answers = []
    for dev in (0, 1):
        ix = hg.HerculesIndex.build(X, 1000, device=dev)
        d, ids = ix.knn(Q, 10, use_lb_sax=True)
        bd, bi = ix.knn_batch(Q, 10)
        assert np.array_equal(bd.view(np.uint32), d.view(np.uint32)) and np.array_equal(bi, ids)
        ix.close()
        with torch.cuda.device(dev):
            Xd = torch.from_numpy(X).cuda(dev)
            Qd = torch.from_numpy(Q).cuda(dev)
            D = torch.empty(10, dtype=torch.float32, device=dev)
            I = torch.empty(10, dtype=torch.int64, device=dev)
            hg.pscan_noalloc(Xd.data_ptr(), X.shape[0], 256, Qd[0].data_ptr(), 10, D.data_ptr(), I.data_ptr(),
                             torch.cuda.current_stream(dev).cuda_stream)
            torch.cuda.synchronize(dev)
            assert np.array_equal(I.cpu().numpy(), ids[0])
        answers.append((d, ids))
    assert np.array_equal(answers[0][0].view(np.uint32), answers[1][0].view(np.uint32))
    assert np.array_equal(answers[0][1], answers[1][1])
