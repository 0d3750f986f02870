// Measurement helpers of the C ABI: a kernel-launch counter, an FMA-throughput probe and an
// evaluator of the far-field arithmetic.
//
// pvl_launch_count() counts every kernel enqueued through the ABI (incremented at each
// launch site), so a caller can state how many of this library's kernels ran in a timed
// region.  pvl_fma_probe() enqueues a kernel of independent FMA chains whose FLOP count
// is known exactly; timing it gives the FP64 / FP32 non-tensor peak that the
// compute-bound pair kernels are measured against.  pvl_far_series_eval() runs the FP64
// reciprocal and arctangent series of the pair kernels on given arguments, so that a test
// can hold them to their error bounds.
#include <atomic>
#include <cstdint>

#include "pvl_common.cuh"

namespace {
std::atomic<unsigned long long> g_launches{0};

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

void pvl_count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

extern "C" unsigned long long pvl_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }

extern "C" double pvl_fma_probe(int precision, uint32_t n_blocks, uint32_t iters, void* sink, void* stream)
{
    if (!sink || n_blocks == 0 || iters == 0) {
        pvl_fail(PVL_ERR_ARG, "pvl_fma_probe: bad arguments");
        return -1.0;
    }
    cudaStream_t st = (cudaStream_t)stream;
    if (precision == PVL_F32)
        fma_probe_kernel<float><<<n_blocks, kProbeThreads, 0, st>>>(iters, 1.0f, static_cast<float*>(sink));
    else
        fma_probe_kernel<double><<<n_blocks, kProbeThreads, 0, st>>>(iters, 1.0, static_cast<double*>(sink));
    pvl_count_launch();
    if (cudaGetLastError() != cudaSuccess) {
        pvl_fail(PVL_ERR_CUDA, "pvl_fma_probe: launch failed");
        return -1.0;
    }
    return 2.0 * kChains * (double)iters * kProbeThreads * n_blocks;
}

extern "C" int pvl_far_series_eval(uint32_t n, const double* x, const double* w, double* rcp, double* sum,
                                   void* stream)
{
    if (n == 0)
        return PVL_OK;
    if (!x || !w || !rcp || !sum)
        return pvl_fail(PVL_ERR_ARG, "pvl_far_series_eval: null pointer argument");
    far_series_kernel<<<(n + 255) / 256, 256, 0, (cudaStream_t)stream>>>(n, x, w, rcp, sum);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}
