"""The tcgen05 TF32 GEMM vs a plain PyTorch FP32 matmul.  Needs a B200.

TF32 keeps 10 mantissa bits: products carry ~2^-11 relative error, accumulation is FP32, so
the tolerance is 3e-3 relative (Frobenius) on random data."""

import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("M,N,K,alpha,beta", [(128, 128, 32, 1.0, 0.0), (256, 384, 96, 1.0, 0.0),
                                              (512, 256, 512, -0.5, 1.0), (1024, 1024, 1024, 2.0, -1.0)])
def test_gemm_tf32_matches_torch(M, N, K, alpha, beta):
    import torch

    from pyvl_b200 import _lib
    from pyvl_b200.device import ptr, stream_ptr

    g = torch.Generator(device="cuda").manual_seed(M + N + K)
    A = torch.randn(M, K, device="cuda", generator=g)
    B = torch.randn(K, N, device="cuda", generator=g)
    C = torch.randn(M, N, device="cuda", generator=g)
    want = alpha * (A.double() @ B.double()) + beta * C.double()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.call("pvl_gemm_tf32", M, N, K, alpha, ptr(A), K, ptr(B), N, beta, ptr(C), N, ptr(err), stream_ptr())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    rel = (torch.linalg.norm(C.double() - want) / torch.linalg.norm(want)).item()
    assert rel <= 3e-3, rel


def test_gemm_tf32_rejects_bad_shapes():
    import torch

    from pyvl_b200 import _lib

    x = torch.zeros(16, device="cuda")
    with pytest.raises(ValueError):
        _lib.call("pvl_gemm_tf32", 100, 128, 32, 1.0, x.data_ptr(), 32, x.data_ptr(), 128, 0.0, x.data_ptr(), 128,
                  x.data_ptr(), None)
