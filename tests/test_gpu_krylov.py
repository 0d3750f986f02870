"""Building blocks of the mixed solve against plain PyTorch FP64: matrix-vector products with
FP64 and FP32 matrices (vectorised and scalar paths), Gram-Schmidt projection, normalisation
and the basis combination.  Needs a B200."""

import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", ["f64", "f32"])
@pytest.mark.parametrize("rows,cols,ld", [(4096, 4096, 4096), (1000, 999, 1003), (7, 130, 132), (1, 1, 1)])
def test_gemv(dtype, rows, cols, ld):
    import torch

    from pyvl_b200 import _lib
    from pyvl_b200.device import ptr, stream_ptr

    g = torch.Generator(device="cuda").manual_seed(rows + cols)
    tdt = torch.float64 if dtype == "f64" else torch.float32
    M = torch.randn(rows, ld, dtype=tdt, device="cuda", generator=g)
    x = torch.randn(cols, dtype=torch.float64, device="cuda", generator=g)
    y = torch.randn(rows, dtype=torch.float64, device="cuda", generator=g)
    want = -0.5 * (M[:, :cols].double() @ x) + 2.0 * y
    name = "pvl_gemv_f64" if dtype == "f64" else "pvl_gemv_f32mat"
    _lib.call(name, rows, cols, -0.5, ptr(M), ld, ptr(x), 2.0, ptr(y), stream_ptr())
    torch.cuda.synchronize()
    assert torch.allclose(y, want, rtol=1e-12, atol=1e-12 * cols)


def test_gram_schmidt_normalise_combine():
    import torch

    from pyvl_b200 import _lib
    from pyvl_b200.device import ptr, stream_ptr

    n, k = 3000, 5
    g = torch.Generator(device="cuda").manual_seed(0)
    V = torch.linalg.qr(torch.randn(n, k, dtype=torch.float64, device="cuda", generator=g))[0].T.contiguous()
    w = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    w0 = w.clone()
    h = torch.zeros(2 * k, dtype=torch.float64, device="cuda")
    s = stream_ptr()
    _lib.call("pvl_basis_project", n, k, ptr(V), n, ptr(w), ptr(h), s)
    torch.cuda.synchronize()
    assert torch.allclose(h[:k], V @ w0, rtol=1e-12, atol=1e-12)
    assert torch.allclose(w, w0 - V.T @ (V @ w0), rtol=1e-12, atol=1e-12)
    v = torch.zeros(n, dtype=torch.float64, device="cuda")
    nrm = torch.zeros(1, dtype=torch.float64, device="cuda")
    _lib.call("pvl_normalize", n, ptr(w), ptr(v), ptr(nrm), s)
    torch.cuda.synchronize()
    assert abs(nrm.item() - torch.linalg.vector_norm(w).item()) <= 1e-12 * nrm.item()
    assert torch.allclose(v, w / torch.linalg.vector_norm(w), rtol=1e-13, atol=1e-15)
    c = torch.randn(k, dtype=torch.float64, device="cuda", generator=g)
    x = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    want = x + V.T @ c
    _lib.call("pvl_combine", n, k, ptr(V), n, ptr(c), ptr(x), s)
    torch.cuda.synchronize()
    assert torch.allclose(x, want, rtol=1e-13, atol=1e-13)
