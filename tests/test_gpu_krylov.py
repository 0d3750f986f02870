"""Building blocks of the mixed solve against plain PyTorch FP64: matrix-vector products with
FP64 and FP32 matrices (vectorised and scalar paths), Gram-Schmidt projection, normalisation
and the basis combination.  Needs a B200."""

import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", ["f64", "f32", "f32x32"])
@pytest.mark.parametrize("rows,cols,ld", [(4096, 4096, 4096), (1000, 999, 1003), (1000, 1000, 1000),
                                          (7, 130, 132), (3, 2050, 2052), (1, 1, 1)])
@pytest.mark.parametrize("beta", [2.0, 0.0])
def test_gemv(dtype, rows, cols, ld, beta):
    import torch

    from pyvl_b200 import _lib
    from pyvl_b200.device import ptr, stream_ptr

    g = torch.Generator(device="cuda").manual_seed(rows + cols)
    tdt = torch.float64 if dtype == "f64" else torch.float32
    M = torch.randn(rows, ld, dtype=tdt, device="cuda", generator=g)
    x = torch.randn(cols, dtype=torch.float64, device="cuda", generator=g)
    if dtype == "f32x32":  # FP32 vector: the products of each 16-byte group are summed in FP32
        x = x.float()
    y = torch.randn(rows, dtype=torch.float64, device="cuda", generator=g)
    want = -0.5 * (M[:, :cols].double() @ x.double()) + beta * y
    name = {"f64": "pvl_gemv_f64", "f32": "pvl_gemv_f32mat", "f32x32": "pvl_gemv_f32"}[dtype]
    _lib.call(name, rows, cols, -0.5, ptr(M), ld, ptr(x), beta, ptr(y), stream_ptr())
    torch.cuda.synchronize()
    if dtype == "f32x32":
        scale = 0.5 * (M[:, :cols].double().abs() @ x.double().abs())
        assert bool(((y - want).abs() <= 4e-7 * scale + 1e-12).all())
    else:
        assert torch.allclose(y, want, rtol=1e-12, atol=1e-12 * cols)


@pytest.mark.parametrize("n", [1000, 4096, 130])
def test_lu_solve_blocked_matches_wavefront(n):
    """The graph-safe blocked substitution and the wavefront solve of the same factors."""
    import torch

    from pyvl_b200 import _lib
    from pyvl_b200.device import ptr, stream_ptr

    g = torch.Generator(device="cuda").manual_seed(n)
    A = torch.randn(n, n, dtype=torch.float64, device="cuda", generator=g) + 0.5 * n ** 0.5 * torch.eye(
        n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
    LU = A.clone()
    ipiv = torch.zeros(2 * n, dtype=torch.int32, device="cuda")
    info = torch.zeros(1, dtype=torch.int32, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    nb = int(_lib.query("pvl_lu_workspace", n))
    ws = torch.empty(nb, dtype=torch.uint8, device="cuda")
    s = stream_ptr()
    _lib.call("pvl_lu_factor", n, ptr(LU), n, ptr(ipiv), ptr(info), ptr(ws), nb, s)
    x1, x2 = b.clone(), b.clone()
    _lib.call("pvl_lu_solve", n, ptr(LU), n, ptr(ipiv), ptr(x1), ptr(err), ptr(ws), nb, s)
    _lib.call("pvl_lu_solve_blocked", n, ptr(LU), n, ptr(ipiv), ptr(x2), ptr(ws), nb, s)
    torch.cuda.synchronize()
    assert int(info.item()) == 0 and int(err.item()) == 0
    # two substitution orders of the same factors: their difference is bounded by ~cond(A) x
    # eps (the shifted random matrix's spectrum reaches near zero; cond ~1e3 at n = 4096)
    assert float(torch.linalg.vector_norm(x2 - x1) / torch.linalg.vector_norm(x1)) <= 1e-12
    assert float(torch.linalg.vector_norm(A @ x2 - b) / torch.linalg.vector_norm(b)) <= 1e-12


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
