"""Numerics of the tcgen05 tensor-core kernel behind the batched filter: its
products q~.x~ (BF16 roundings, FP32 accumulation in tensor memory) against
a PyTorch FP64 product of the same BF16 values.  The accumulation error must
stay inside the L 2^-20 |q~| |x~| term of the filter's certified bound."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,L,nq", [
    (1000, 256, 300),   # two query tiles (the second partial), resident query tile
    (777, 96, 40),      # K padded by the TMA zero fill (96 = 64 + 32)
    (129, 16, 5),       # one partial K block, one row past a full tile
    (300, 1024, 260),   # query tile streamed with the rows (L > 256)
])
def test_tensor_core_products(hg, gpu_available, n, L, nq):
    import torch
    g = torch.Generator(device="cuda").manual_seed(n * 7 + L)
    X = torch.randn(n, L, device="cuda", generator=g) * 3
    Q = torch.randn(nq, L, device="cuda", generator=g)
    out = torch.full((nq, n), float("nan"), device="cuda")
    hg.bf16_dots_device(X.data_ptr(), n, L, Q.data_ptr(), nq, out.data_ptr())
    torch.cuda.synchronize()
    xb = X.to(torch.bfloat16).double()
    qb = Q.to(torch.bfloat16).double()
    ref = qb @ xb.T
    bound = L * 2.0 ** -20 * qb.norm(dim=1)[:, None] * xb.norm(dim=1)[None, :]
    err = (out.double() - ref).abs()
    assert torch.isfinite(out).all()
    assert (err <= bound).all(), float((err / bound).max())


def test_tensor_core_products_walks(hg, gpu_available):
    """The collection's own kind of data: z-normalised random walks."""
    import torch
    n, L = 5000, 256
    X = hg.generate_walks(1184, n, L)
    Q = hg.generate_queries(14784, X, np.array([0.01, 0.1, 1.0] * 30))
    Xd, Qd = torch.from_numpy(X).cuda(), torch.from_numpy(Q).cuda()
    out = torch.empty((len(Q), n), device="cuda")
    hg.bf16_dots_device(Xd.data_ptr(), n, L, Qd.data_ptr(), len(Q), out.data_ptr())
    torch.cuda.synchronize()
    ref = Qd.to(torch.bfloat16).double() @ Xd.to(torch.bfloat16).double().T
    assert ((out.double() - ref).abs() <= L * 2.0 ** -20 * 16.0 * 16.0 * 1.01).all()
