// Building blocks of the mixed-precision solve: FP64 residuals against the FP64 system
// matrix, the FP32 approximate inverse applied as a matrix-vector product, and the
// Gram-Schmidt steps of (flexible) GMRES.  All bandwidth-bound; the host drives the
// iteration and keeps the small Hessenberg least-squares problem.
#include <cstdint>

#include "gemv.cuh"
#include "pvl_common.cuh"

namespace {

inline unsigned blocks_for(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

// c[i] = V_i . w for i < k (one CTA per basis vector).
__global__ void __launch_bounds__(256) basis_dots_kernel(uint32_t n, const double* __restrict__ V, uint32_t ldv,
                                                         const double* __restrict__ w, double* __restrict__ c)
{
    __shared__ double red[8];
    const uint32_t i = blockIdx.x;
    const double* v = V + (size_t)i * ldv;
    double s = 0.0;
    for (uint32_t j = threadIdx.x; j < n; j += blockDim.x)
        s += v[j] * w[j];
    for (int o = 16; o > 0; o >>= 1)
        s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0)
        red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < 8; ++q)
            t += red[q];
        c[i] = t;
    }
}

// w += sign * sum_{i<k} c[i] V_i  (c on the device); with h != NULL, thread 0 also adds c to h.
__global__ void basis_axpy_kernel(uint32_t n, uint32_t k, const double* __restrict__ V, uint32_t ldv,
                                  const double* __restrict__ c, double sign, double* __restrict__ w,
                                  double* __restrict__ h)
{
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (h && j == 0)
        for (uint32_t i = 0; i < k; ++i)
            h[i] += c[i];
    if (j >= n)
        return;
    double s = 0.0;
    for (uint32_t i = 0; i < k; ++i)
        s += c[i] * V[(size_t)i * ldv + j];
    w[j] += sign * s;
}

// nrm[0] = ||w||; v = w / nrm  (one CTA of 1024 threads)
__global__ void __launch_bounds__(1024) normalize_kernel(uint32_t n, const double* __restrict__ w,
                                                         double* __restrict__ v, double* __restrict__ nrm)
{
    __shared__ double red[32];
    __shared__ double s_norm;
    double s = 0.0;
    for (uint32_t j = threadIdx.x; j < n; j += blockDim.x)
        s += w[j] * w[j];
    for (int o = 16; o > 0; o >>= 1)
        s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0)
        red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < 32; ++q)
            t += red[q];
        s_norm = sqrt(t);
        nrm[0] = s_norm;
    }
    __syncthreads();
    const double inv = s_norm > 0.0 ? 1.0 / s_norm : 0.0;
    if (v)
        for (uint32_t j = threadIdx.x; j < n; j += blockDim.x)
            v[j] = w[j] * inv;
}

// b (npad x npad of ldb, FP32) = a (n x n, FP64) padded with the identity.
__global__ void pad_convert_kernel(uint32_t n, const double* __restrict__ a, uint32_t lda, float* __restrict__ b,
                                   uint32_t ldb, uint32_t npad)
{
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)npad * npad)
        return;
    const uint32_t r = (uint32_t)(t / npad), c = (uint32_t)(t % npad);
    b[(size_t)r * ldb + c] = (r < n && c < n) ? (float)a[(size_t)r * lda + c] : (r == c ? 1.0f : 0.0f);
}

__global__ void axpy_kernel(uint32_t n, double alpha, const double* __restrict__ x, double* __restrict__ y)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        y[i] += alpha * x[i];
}

int require(const void* p, const char* what) { return p ? PVL_OK : pvl_fail(PVL_ERR_ARG, "%s is NULL", what); }

}  // namespace

#define PVL_REQUIRE(p)                 \
    do {                               \
        if (int _r = require((p), #p)) \
            return _r;                 \
    } while (0)

extern "C" int pvl_gemv_f64(uint32_t rows, uint32_t cols, double alpha, const double* A, uint32_t lda, const double* x,
                            double beta, double* y, void* stream)
{
    if (rows == 0)
        return PVL_OK;
    PVL_REQUIRE(A); PVL_REQUIRE(x); PVL_REQUIRE(y);
    pvl::launch_gemv<double, double>(rows, cols, alpha, A, lda, x, 0, beta, beta == 0.0 ? nullptr : y, y, 0, nullptr,
                                     (cudaStream_t)stream);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_gemv_f32mat(uint32_t rows, uint32_t cols, double alpha, const float* M, uint32_t ldm,
                               const double* x, double beta, double* y, void* stream)
{
    if (rows == 0)
        return PVL_OK;
    PVL_REQUIRE(M); PVL_REQUIRE(x); PVL_REQUIRE(y);
    pvl::launch_gemv<float, double>(rows, cols, alpha, M, ldm, x, 0, beta, beta == 0.0 ? nullptr : y, y, 0, nullptr,
                                    (cudaStream_t)stream);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_gemv_f32(uint32_t rows, uint32_t cols, double alpha, const float* M, uint32_t ldm, const float* x,
                            double beta, double* y, void* stream)
{
    if (rows == 0)
        return PVL_OK;
    PVL_REQUIRE(M); PVL_REQUIRE(x); PVL_REQUIRE(y);
    pvl::launch_gemv<float, float>(rows, cols, alpha, M, ldm, x, 0, beta, beta == 0.0 ? nullptr : y, y, 0, nullptr,
                                   (cudaStream_t)stream);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_basis_project(uint32_t n, uint32_t k, const double* V, uint32_t ldv, double* w, double* h,
                                 void* stream)
{
    if (n == 0 || k == 0)
        return PVL_OK;
    PVL_REQUIRE(V); PVL_REQUIRE(w); PVL_REQUIRE(h);
    cudaStream_t st = (cudaStream_t)stream;
    double* c = h + k;  // scratch: this pass's coefficients, right after the accumulated ones
    basis_dots_kernel<<<k, 256, 0, st>>>(n, V, ldv, w, c);
    PVL_LAUNCH_CHECK();
    basis_axpy_kernel<<<blocks_for(n, 256), 256, 0, st>>>(n, k, V, ldv, c, -1.0, w, h);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_normalize(uint32_t n, const double* w, double* v, double* nrm, void* stream)
{
    if (n == 0)
        return PVL_OK;
    PVL_REQUIRE(w); PVL_REQUIRE(nrm);
    normalize_kernel<<<1, 1024, 0, (cudaStream_t)stream>>>(n, w, v, nrm);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_combine(uint32_t n, uint32_t k, const double* Z, uint32_t ldz, const double* c, double* x,
                           void* stream)
{
    if (n == 0 || k == 0)
        return PVL_OK;
    PVL_REQUIRE(Z); PVL_REQUIRE(c); PVL_REQUIRE(x);
    basis_axpy_kernel<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(n, k, Z, ldz, c, 1.0, x, nullptr);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_pad_convert_f32(uint32_t n, const double* a, uint32_t lda, float* b, uint32_t ldb,
                                   uint32_t npad, void* stream)
{
    if (npad == 0)
        return PVL_OK;
    PVL_REQUIRE(a); PVL_REQUIRE(b);
    if (npad < n || ldb < npad || lda < n)
        return pvl_fail(PVL_ERR_ARG, "pvl_pad_convert_f32: need n <= npad <= ldb and lda >= n");
    pad_convert_kernel<<<blocks_for((size_t)npad * npad, 256), 256, 0, (cudaStream_t)stream>>>(n, a, lda, b, ldb,
                                                                                             npad);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_axpy_f64(uint32_t n, double alpha, const double* x, double* y, void* stream)
{
    if (n == 0)
        return PVL_OK;
    PVL_REQUIRE(x); PVL_REQUIRE(y);
    axpy_kernel<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(n, alpha, x, y);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}
