// Measurement and test probes (libpvl_probe.so) -- not part of the product's C ABI.
//
// pvl_probe_fma() enqueues a kernel of independent FMA chains whose FLOP count is known
// exactly; timing it gives the FP64 / FP32 non-tensor peak that the compute-bound pair kernels
// are measured against.  pvl_probe_far_series() runs the FP64 reciprocal and arctangent series
// of the pair kernels (pvl::FarSeries) on given arguments, so that a test can hold them to
// their error bounds.  pvl_probe_trsv_timeout() launches the product's wavefront triangular
// solve (trsv.cuh) with a short spin limit and one row block that never publishes its flag,
// so that a test can watch every later block's bounded wait run out and report through the
// error word, with no GPU fault and nothing left running.  pvl_probe_gemm_timeout() runs the
// product's TMA-fed TF32 GEMM (gemm_tc.cuh, through its launcher in libpvl_b200.so) with a
// short wait limit and a producer that issues no copies: every wait runs out, no copy or MMA
// is in flight, and the kernel frees its tensor memory and sets the error word.
#include <cstdarg>
#include <cstdint>
#include <cstdio>

#include "gemm_tc.cuh"
#include "pvl_common.cuh"
#include "pvl_probe.h"
#include "trsv.cuh"

namespace {
thread_local char g_err[512] = "";

int fail(int code, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
    return code;
}

constexpr int kProbeThreads = 256;
constexpr int kChains = 8;

template <typename T>
__global__ void __launch_bounds__(kProbeThreads) fma_probe_kernel(uint32_t iters, T seed, T* __restrict__ sink)
{
    T a[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c)
        a[c] = seed + T(threadIdx.x + c);
    const T m = T(0.999999), k = T(1e-7);
    for (uint32_t i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c)
            a[c] = fma(a[c], m, k);
    }
    T s = T(0);
#pragma unroll
    for (int c = 0; c < kChains; ++c)
        s += a[c];
    if (s == T(-1.2345))  // never true for the chains above; keeps the work observable
        sink[blockIdx.x] = s;
}

__global__ void far_series_kernel(uint32_t n, const double* __restrict__ x, const double* __restrict__ w,
                                  double* __restrict__ rcp, double* __restrict__ sum)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        rcp[i] = pvl::FarSeries<double>::rcp(x[i]);
        sum[i] = pvl::FarSeries<double>::sum(w[i]);
    }
}
}  // namespace

extern "C" const char* pvl_probe_last_error(void) { return g_err; }

extern "C" double pvl_probe_fma(int precision, uint32_t n_blocks, uint32_t iters, void* sink, void* stream)
{
    if (!sink || n_blocks == 0 || iters == 0) {
        fail(PVL_ERR_ARG, "pvl_probe_fma: bad arguments");
        return -1.0;
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (precision == PVL_F32)
        fma_probe_kernel<float><<<n_blocks, kProbeThreads, 0, st>>>(iters, 1.0f, static_cast<float*>(sink));
    else
        fma_probe_kernel<double><<<n_blocks, kProbeThreads, 0, st>>>(iters, 1.0, static_cast<double*>(sink));
    if (cudaGetLastError() != cudaSuccess) {
        fail(PVL_ERR_CUDA, "pvl_probe_fma: launch failed");
        return -1.0;
    }
    return 2.0 * kChains * (double)iters * kProbeThreads * n_blocks;
}

extern "C" int pvl_probe_far_series(uint32_t n, const double* x, const double* w, double* rcp, double* sum,
                                    void* stream)
{
    if (n == 0)
        return PVL_OK;
    if (!x || !w || !rcp || !sum)
        return fail(PVL_ERR_ARG, "pvl_probe_far_series: null pointer argument");
    far_series_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(n, x, w, rcp, sum);
    if (cudaGetLastError() != cudaSuccess)
        return fail(PVL_ERR_CUDA, "pvl_probe_far_series: launch failed");
    return PVL_OK;
}

extern "C" int pvl_probe_trsv_timeout(uint32_t n, const double* LU, uint32_t lda, const double* inv, double* x,
                                      int32_t* flags, int32_t* err, long long spin_limit, int32_t skip_block,
                                      int lower, void* stream)
{
    if (n == 0 || !LU || !inv || !x || !flags || !err || lda < n || spin_limit <= 0)
        return fail(PVL_ERR_ARG, "pvl_probe_trsv_timeout: bad arguments");
    const uint32_t nblk = (n + pvl::trsv::kRB - 1) / pvl::trsv::kRB;
    const void* fn = lower ? (const void*)pvl::trsv::wavefront_kernel<true> : (const void*)pvl::trsv::wavefront_kernel<false>;
    int dev = 0, sms = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, pvl::trsv::kThreads, 0) != cudaSuccess)
        return fail(PVL_ERR_CUDA, "pvl_probe_trsv_timeout: occupancy query failed");
    if ((long long)nblk > (long long)sms * per)
        return fail(PVL_ERR_ARG, "pvl_probe_trsv_timeout: %u blocks cannot be co-resident", nblk);
    cudaStream_t st = (cudaStream_t)stream;
    if (cudaMemsetAsync(flags, 0, sizeof(int32_t) * (nblk + 1), st) != cudaSuccess ||
        cudaMemsetAsync(err, 0, sizeof(int32_t), st) != cudaSuccess)
        return fail(PVL_ERR_CUDA, "pvl_probe_trsv_timeout: memset failed");
    void* args[] = {(void*)&n, (void*)&LU, (void*)&lda, (void*)&inv, (void*)&x, (void*)&flags, (void*)&err,
                    (void*)&spin_limit, (void*)&skip_block};
    if (cudaLaunchCooperativeKernel(fn, dim3(nblk), dim3(pvl::trsv::kThreads), args, 0, st) != cudaSuccess)
        return fail(PVL_ERR_CUDA, "pvl_probe_trsv_timeout: launch failed");
    return PVL_OK;
}

extern "C" int pvl_probe_gemm_timeout(uint32_t M, uint32_t N, uint32_t K, const float* A, uint32_t lda,
                                      const float* Bt, uint32_t ldbt, float* C, uint32_t ldc, int32_t* err,
                                      long long wait_limit, void* stream)
{
    if (!A || !Bt || !C || !err || K == 0 || K % pvl::gemm_tc::kKT || wait_limit <= 0)
        return fail(PVL_ERR_ARG, "pvl_probe_gemm_timeout: bad arguments");
    if (cudaMemsetAsync(err, 0, sizeof(int32_t), (cudaStream_t)stream) != cudaSuccess)
        return fail(PVL_ERR_CUDA, "pvl_probe_gemm_timeout: memset failed");
    const int r = pvl_gemm_tf32_launch(M, N, K, 1.0f, A, lda, Bt, ldbt, 0.0f, C, ldc, err, wait_limit, 1, 1,
                                       (cudaStream_t)stream);
    if (r != PVL_OK)
        return fail(r, "pvl_probe_gemm_timeout: %s", pvl_last_error());
    return PVL_OK;
}
