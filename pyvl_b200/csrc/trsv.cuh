// Wavefront triangular solve over 64-row blocks (the solve half of pvl_lu_solve).
//
// One CTA per row block, all co-resident (cooperative launch).  LOWER: unit-lower forward
// substitution, block b needs x of blocks 0..b-1; UPPER: backward substitution, block b needs
// x of blocks nblk-1..b+1.  x holds the right-hand side on entry and the solution on exit.
//
// A CTA keeps the off-diagonal row block it is about to need in registers before the block
// it depends on is published: each of the 256 threads holds 8 rows x 2 columns of the next
// 64 x 64 block (prefetched while the current dependency is consumed), and a row's partial
// sums stay per thread until every dependency is in -- after a flag arrives the work left is
// two loads of x and 16 FMAs per thread.  The inverted diagonal block sits in shared memory
// from the start.  So the chain from one block's flag to the next is a flag poll, an L2 read
// of 64 values, a warp reduction and a 64 x 64 product from shared memory.
//
// Waits are bounded: a CTA that has polled a flag `spin_limit` times sets *err, publishes its
// own flag (so that no later block waits on it in vain) and returns; the solution is then
// invalid and the caller reports PVL_ERR_TIMEOUT.  `skip_block` (normally -1) names a block
// that returns at once without publishing: only a test uses it, to make the waits of every
// later block run out.
#pragma once

#include <cstdint>

namespace pvl {
namespace trsv {

constexpr int kRB = 64;         // rows per block (the LU's panel width)
constexpr int kThreads = 256;   // 8 warps x 8 rows
constexpr long long kSpinLimit = 20000000;  // ~2 s at ~100 ns per poll

__device__ __forceinline__ int32_t ld_acquire(const int32_t* p)
{
    int32_t v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(int32_t* p, int32_t v)
{
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// M: the LU factors (row-major, lda); inv: the inverted diagonal blocks, (nblk, 2, 64, 64) with
// [b][0] = L_bb^-1 and [b][1] = U_bb^-1 (a partial last block padded with identity).
template <bool LOWER>
__global__ void __launch_bounds__(kThreads) wavefront_kernel(uint32_t n, const double* __restrict__ M, uint32_t lda,
                                                             const double* __restrict__ inv, double* __restrict__ x,
                                                             int32_t* __restrict__ flags, int32_t* __restrict__ err,
                                                             long long spin_limit, int32_t skip_block)
{
    __shared__ double s_inv[kRB][kRB + 1];
    __shared__ double s_r[kRB];
    __shared__ double s_acc[kRB];
    __shared__ int s_abort;
    const uint32_t nblk = (n + kRB - 1) / kRB;
    const uint32_t b = LOWER ? blockIdx.x : nblk - 1 - blockIdx.x;
    if ((int32_t)b == skip_block)
        return;
    const uint32_t r0 = b * kRB;
    const uint32_t rows = min((uint32_t)kRB, n - r0);
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double* D = inv + ((size_t)b * 2 + (LOWER ? 0 : 1)) * kRB * kRB;
    for (uint32_t e = threadIdx.x; e < kRB * kRB; e += kThreads)
        s_inv[e / kRB][e % kRB] = D[e];
    if (threadIdx.x == 0)
        s_abort = 0;
    const uint32_t n_dep = LOWER ? b : nblk - 1 - b;
    // this thread's rows (warp w: rows 8w .. 8w+7) and columns (lane, lane + 32) of a 64 x 64 block
    double part[8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
        part[i] = 0.0;
    double cur[8][2], nxt[8][2];
    auto load_block = [&](uint32_t step, double (&dst)[8][2]) {
        const uint32_t c = LOWER ? step : nblk - 1 - step;
        const uint32_t c0 = c * kRB, ccols = min((uint32_t)kRB, n - c0);
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const uint32_t r = 8 * warp + i;
            const double* mrow = M + (size_t)(r0 + r) * lda + c0;
            dst[i][0] = (r < rows && lane < ccols) ? __ldcs(mrow + lane) : 0.0;
            dst[i][1] = (r < rows && lane + 32 < ccols) ? __ldcs(mrow + lane + 32) : 0.0;
        }
    };
    if (n_dep > 0)
        load_block(0, cur);
    // this block's own right-hand side: no other block writes it, so it is read now and not on
    // the chain after the last dependency
    const double rhs_own = threadIdx.x < rows ? __ldcg(x + r0 + threadIdx.x) : 0.0;
    __syncthreads();
    for (uint32_t step = 0; step < n_dep; ++step) {
        if (step + 1 < n_dep)
            load_block(step + 1, nxt);  // in flight while this step waits
        const uint32_t c = LOWER ? step : nblk - 1 - step;
        if (threadIdx.x == 0) {
            long long spins = 0;
            while (ld_acquire(flags + c) == 0) {
                if (++spins > spin_limit) {
                    atomicExch(err, 1);
                    s_abort = 1;
                    break;
                }
                __nanosleep(32);
            }
        }
        __syncthreads();
        if (s_abort) {
            if (threadIdx.x == 0)
                st_release(flags + b, 1);
            return;
        }
        const uint32_t c0 = c * kRB, ccols = min((uint32_t)kRB, n - c0);
        const double x0 = lane < ccols ? __ldcg(x + c0 + lane) : 0.0;
        const double x1 = lane + 32 < ccols ? __ldcg(x + c0 + lane + 32) : 0.0;
#pragma unroll
        for (int i = 0; i < 8; ++i)
            part[i] = fma(cur[i][1], x1, fma(cur[i][0], x0, part[i]));
        if (step + 1 < n_dep) {
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                cur[i][0] = nxt[i][0];
                cur[i][1] = nxt[i][1];
            }
        }
    }
    // row sums of the dependencies, then x_b = inv(D_bb) (r_b - sums)
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        double s = part[i];
        for (int o = 16; o > 0; o >>= 1)
            s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0)
            s_acc[8 * warp + i] = s;
    }
    __syncthreads();
    if (threadIdx.x < kRB)
        s_r[threadIdx.x] = threadIdx.x < rows ? rhs_own - s_acc[threadIdx.x] : 0.0;
    __syncthreads();
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const uint32_t r = 8 * warp + i;
        double s = s_inv[r][lane] * s_r[lane] + s_inv[r][lane + 32] * s_r[lane + 32];
        for (int o = 16; o > 0; o >>= 1)
            s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0 && r < rows)
            x[r0 + r] = s;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0)
        st_release(flags + b, 1);
}

}  // namespace trsv
}  // namespace pvl
