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
    Bt = B.t().contiguous()  # the right operand is passed K-major (transposed)
    _lib.call("pvl_gemm_tf32", M, N, K, alpha, ptr(A), K, ptr(Bt), K, beta, ptr(C), N, ptr(err), stream_ptr())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    rel = (torch.linalg.norm(C.double() - want) / torch.linalg.norm(want)).item()
    assert rel <= 3e-3, rel


@pytest.mark.parametrize("M,N,K", [(100, 200, 64), (64, 4096 - 64, 64), (1, 7, 32), (300, 129, 96)])
def test_gemm_tf32_ragged_submatrix(M, N, K):
    """Edges that are not multiples of the 128 x 128 tile, operands and C inside larger
    buffers: the block is updated, nothing outside it is touched."""
    import torch

    from pyvl_b200 import _lib
    from pyvl_b200.device import ptr, stream_ptr

    g = torch.Generator(device="cuda").manual_seed(7 * M + N)
    n4 = (N + 3) // 4 * 4  # leading dimensions: multiples of 4 floats, blocks 16-byte aligned
    lda, ldbt, ldc = K + 8, K + 12, n4 + 20
    A = torch.randn(M + 3, lda, device="cuda", generator=g)
    Bt = torch.randn(N + 2, ldbt, device="cuda", generator=g)
    C = torch.randn(M + 5, ldc, device="cuda", generator=g)
    C0 = C.clone()
    a, bt = A[1:1 + M, 4:4 + K], Bt[2:2 + N, 4:4 + K]  # bt: B transposed, inside a larger buffer
    c = C[2:2 + M, 8:8 + N]
    want = -(a.double() @ bt.double().t()) + c.double()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    _lib.call("pvl_gemm_tf32", M, N, K, -1.0, a.data_ptr(), lda, bt.data_ptr(), ldbt, 1.0, c.data_ptr(), ldc, ptr(err),
              stream_ptr())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    rel = (torch.linalg.norm(c.double() - want) / torch.linalg.norm(want)).item()
    assert rel <= 3e-3, rel
    mask = torch.ones_like(C, dtype=torch.bool)
    mask[2:2 + M, 8:8 + N] = False
    assert torch.equal(C[mask], C0[mask])


def test_gemm_tf32_rejects_bad_shapes():
    import torch

    from pyvl_b200 import _lib

    x = torch.zeros(16, device="cuda")
    with pytest.raises(ValueError):  # K not a multiple of 32: rejected before any launch
        _lib.call("pvl_gemm_tf32", 128, 128, 20, 1.0, x.data_ptr(), 32, x.data_ptr(), 32, 0.0, x.data_ptr(), 128,
                  x.data_ptr(), None)


def test_gemm_tf32_waits_run_out_without_its_copies():
    """The probe runs the same kernel with a short wait limit and a producer that issues no
    copies: every bounded wait runs out, the kernel returns, frees its tensor memory and sets
    the error word; a regular GEMM on the same stream follows and is right."""
    import torch

    from pyvl_b200 import _lib, _probe
    from pyvl_b200.device import ptr, stream_ptr

    A = torch.randn(256, 64, device="cuda")
    Bt = torch.randn(256, 64, device="cuda")
    C = torch.zeros(256, 256, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    _probe.call("pvl_probe_gemm_timeout", 256, 256, 64, ptr(A), 64, ptr(Bt), 64, ptr(C), 256, ptr(err), 4000,
                stream_ptr())
    torch.cuda.synchronize()
    assert int(err.item()) == 1
    assert torch.count_nonzero(C).item() == 0  # no accumulator reached the epilogue
    err.zero_()
    _lib.call("pvl_gemm_tf32", 256, 256, 64, 1.0, ptr(A), 64, ptr(Bt), 64, 0.0, ptr(C), 256, ptr(err), stream_ptr())
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    want = A.double() @ Bt.double().t()
    assert (torch.linalg.norm(C.double() - want) / torch.linalg.norm(want)).item() <= 3e-3
