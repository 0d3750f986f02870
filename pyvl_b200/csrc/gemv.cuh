// Matrix-vector products of the mixed-precision solve (sm_100a), shared by krylov.cu and gmres.cu.
//
// y = alpha * M x + beta * b with a row-major FP64 or FP32 matrix M, an FP64 or FP32 vector x
// and FP64 accumulation and output.  One warp per row; each lane keeps UNR 16-byte loads of
// the row in flight.  All of it is HBM streaming (the system matrix is 134 MB at n = 4096,
// larger than L2), so the FP64 matrix is read with the evict-first (streaming) cache
// operator: the FP32 approximate inverse, read in the same Krylov column, then stays in L2.
// Optional device index: x and y advance by index[0] * x_step / y_step, so that a captured
// graph can address the Krylov column the device is currently at.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace pvl {

constexpr int kGemvWarps = 4;

template <typename MT, typename XT> struct GemvVec;
template <> struct GemvVec<double, double> {
    static constexpr int kN = 2, kUnroll = 16;
    static __device__ __forceinline__ double dot(const double* m, const double* x, double s)
    {
        const double2 a = __ldcs(reinterpret_cast<const double2*>(m));
        const double2 b = *reinterpret_cast<const double2*>(x);
        return fma(a.x, b.x, fma(a.y, b.y, s));
    }
};
template <> struct GemvVec<float, double> {
    static constexpr int kN = 4, kUnroll = 8;
    static __device__ __forceinline__ double dot(const float* m, const double* x, double s)
    {
        const float4 a = __ldg(reinterpret_cast<const float4*>(m));
        const double2 b0 = *reinterpret_cast<const double2*>(x);
        const double2 b1 = *reinterpret_cast<const double2*>(x + 2);
        return fma((double)a.x, b0.x, fma((double)a.y, b0.y, fma((double)a.z, b1.x, fma((double)a.w, b1.y, s))));
    }
};
// FP32 matrix and FP32 vector: the four products of a 16-byte vector are summed in FP32
// (an approximate inverse applied to an FP32 copy of the Krylov vector), the row in FP64.
template <> struct GemvVec<float, float> {
    static constexpr int kN = 4, kUnroll = 8;
    static __device__ __forceinline__ double dot(const float* m, const float* x, double s)
    {
        const float4 a = __ldg(reinterpret_cast<const float4*>(m));
        const float4 b = *reinterpret_cast<const float4*>(x);
        return s + (double)fmaf(a.x, b.x, fmaf(a.y, b.y, fmaf(a.z, b.z, a.w * b.w)));
    }
};

template <typename MT, typename XT, bool VEC>
__device__ __forceinline__ double gemv_row(const MT* __restrict__ row, const XT* __restrict__ x, uint32_t n,
                                           uint32_t lane)
{
    using G = GemvVec<MT, XT>;
    constexpr int V = G::kN, U = G::kUnroll, S = 4;  // U loads in flight, S partial sums
    double s[S];
#pragma unroll
    for (int u = 0; u < S; ++u)
        s[u] = 0.0;
    uint32_t j0 = 0;
    if (VEC) {
        const uint32_t nv = n / V;
        uint32_t v = lane;
        for (; v + 32 * (U - 1) < nv; v += 32 * U) {
#pragma unroll
            for (int u = 0; u < U; ++u)
                s[u % S] = G::dot(row + (size_t)(v + 32 * u) * V, x + (size_t)(v + 32 * u) * V, s[u % S]);
        }
        for (; v < nv; v += 32)
            s[0] = G::dot(row + (size_t)v * V, x + (size_t)v * V, s[0]);
        j0 = nv * V;
    }
#pragma unroll 4
    for (uint32_t j = j0 + lane; j < n; j += 32)
        s[1] = fma((double)row[j], (double)x[j], s[1]);
    double t = (s[0] + s[1]) + (s[2] + s[3]);
    for (int o = 16; o > 0; o >>= 1)
        t += __shfl_xor_sync(0xffffffffu, t, o);
    return t;
}

// y[r] = alpha * (M x)[r] + beta * b[r] (b may be y itself, or null for beta = 0).
template <typename MT, typename XT, bool VEC>
__global__ void __launch_bounds__(kGemvWarps * 32, 7) gemv_kernel(uint32_t rows, uint32_t cols, double alpha,
                                                               const MT* __restrict__ M, uint32_t ld, const XT* x,
                                                               size_t x_step, double beta, const double* b, double* y,
                                                               size_t y_step, const uint32_t* __restrict__ index)
{
    const uint32_t r = blockIdx.x * kGemvWarps + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (r >= rows)
        return;
    const size_t k = index ? (size_t)index[0] : 0;
    const double s = gemv_row<MT, XT, VEC>(M + (size_t)r * ld, x + k * x_step, cols, lane);
    if (lane == 0) {
        double* out = y + k * y_step;
        out[r] = b ? fma(alpha, s, beta * b[r]) : alpha * s;
    }
}

// Launch with the vector path when the rows and x are 16-byte aligned.
template <typename MT, typename XT>
inline void launch_gemv(uint32_t rows, uint32_t cols, double alpha, const MT* M, uint32_t ld, const XT* x,
                        size_t x_step, double beta, const double* b, double* y, size_t y_step, const uint32_t* index,
                        cudaStream_t st)
{
    constexpr int V = GemvVec<MT, XT>::kN;
    const bool vec = (ld % V) == 0 && (x_step % V) == 0 && (((uintptr_t)M | (uintptr_t)x) & 15u) == 0;
    const unsigned grid = (unsigned)((rows + kGemvWarps - 1) / kGemvWarps);
    if (vec)
        gemv_kernel<MT, XT, true><<<grid, kGemvWarps * 32, 0, st>>>(rows, cols, alpha, M, ld, x, x_step, beta, b, y,
                                                                    y_step, index);
    else
        gemv_kernel<MT, XT, false><<<grid, kGemvWarps * 32, 0, st>>>(rows, cols, alpha, M, ld, x, x_step, beta, b, y,
                                                                     y_step, index);
}

}  // namespace pvl
