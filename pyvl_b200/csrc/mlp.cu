// The learned warm start of the mixed solve: a per-panel MLP, 12 -> 128 -> 128 -> 1, with
// BF16 weights and BF16 activations and FP32 accumulation.  No reference counterpart: the
// reference solves every step from scratch (python/pyvl/solver.py:223-227).
//
// Kernels:
//   features_kernel -- the 12 normalised inputs of each panel and the base of the prediction
//                      (previous circulation + one Jacobi correction of the new system);
//   forward_tc_kernel -- inference on the tensor cores (tcgen05.mma kind::f16, BF16 operands,
//                      FP32 accumulators in tensor memory), one 128-panel tile per CTA;
//   train_tc_kernel -- forward + backward of the mean squared error over a batch on the tensor
//                      cores, persistent CTAs of 128-sample tiles, the layer-2 weight gradient
//                      accumulated in tensor memory; each CTA writes one partial gradient row
//                      and reduce_kernel sums the rows in a fixed order (deterministic);
//   adam_kernel     -- Adam (Kingma & Ba, 2015) on the FP32 master copy, refreshing the BF16
//                      working copy.
// Parameter vector (FP32 master and BF16 copy alike): W1 (128 x 12), b1 (128), W2 (128 x 128),
// b2 (128), w3 (128), b3 (1).
#include <cuda_bf16.h>

#include <algorithm>
#include <cstdint>

#include "pvl_common.cuh"
#include "umma.cuh"

namespace {

constexpr int kIn = 12;
constexpr int kH = 128;
constexpr int oW1 = 0, oB1 = oW1 + kH * kIn, oW2 = oB1 + kH, oB2 = oW2 + kH * kH, oW3 = oB2 + kH, oB3 = oW3 + kH;
constexpr int kParams = oB3 + 1;
static_assert(oW2 % 8 == 0 && kH % 8 == 0, "W2 rows are read as 16-byte vectors");

inline unsigned blocks_for(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

__device__ __forceinline__ float bf(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }
__device__ __forceinline__ float ldb(const __nv_bfloat16* p) { return __bfloat162float(*p); }

// ---------------------------------------------------------------- inference on the tensor cores
// One CTA of 128 threads per 128-panel tile (the tiles strided over the CTAs).  Layer 1:
// acc1 (TMEM columns 0..127) = X W1^T with X the tile's inputs rounded to BF16 (K = 12 padded
// to one K = 16 step); thread r (TMEM lane r, panel r of the tile) reads its row back, adds b1,
// applies ReLU and rounds to BF16 into H1 in shared memory; layer 2: acc2 (columns 128..255) =
// H1 W2^T, eight K = 16 steps; thread r then forms h2 = bf16(relu(acc2 + b2)) and
// y = b3 + w3 . h2 in FP32.  Operands in the SW128 K-major layout (umma.cuh), MMAs issued by
// one thread (tcgen05.mma kind::f16, BF16 x BF16 -> FP32), completion through mbarriers whose
// waits are bounded: a wait that runs out leaves NaN in the tile's outputs (the seed is then
// rejected by the solve, whose answer does not depend on it).
constexpr int kTcTile = 128;
struct FwdTcSmem {
    unsigned char x[kTcTile * 128];       // X tile: 128 rows x 64 BF16 of K (0..11 used)
    unsigned char w1[kH * 128];           // W1: N = 128 units x 64 BF16 of K (0..11 used)
    unsigned char h1[2][kTcTile * 128];   // H1: K = 128 in two 64-wide column blocks
    unsigned char w2[2][kH * 128];        // W2: N = 128 x K = 128 in two column blocks
    float b1[kH], b2[kH], w3[kH];
    uint64_t bar[2];
    uint32_t tmem;
    int fail;
};

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b)
{
    const uint32_t lo = __bfloat16_as_ushort(__float2bfloat16_rn(a));
    const uint32_t hi = __bfloat16_as_ushort(__float2bfloat16_rn(b));
    return lo | (hi << 16);
}

__global__ void __launch_bounds__(kTcTile) forward_tc_kernel(uint32_t n, const float* __restrict__ X,
                                                             const __nv_bfloat16* __restrict__ P, double scale,
                                                             const double* __restrict__ mul,
                                                             const double* __restrict__ base,
                                                             double* __restrict__ out)
{
    namespace um = pvl::umma;
    extern __shared__ __align__(1024) unsigned char tc_raw[];
    FwdTcSmem& sm = *reinterpret_cast<FwdTcSmem*>(tc_raw + ((1024u - (um::smem_u32(tc_raw) & 1023u)) & 1023u));
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    // weights into the SW128 layout: row j of W1 / W2 is unit j (the N index), K along the row
    for (uint32_t e = tid; e < kH * 8; e += kTcTile) {  // W1: 8 chunks of 8 BF16 per row
        const uint32_t j = e >> 3, c = e & 7u;
        uint32_t w[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint32_t k0 = c * 8 + 2 * q;
            const float a = k0 < kIn ? __bfloat162float(P[oW1 + j * kIn + k0]) : 0.0f;
            const float b = k0 + 1 < kIn ? __bfloat162float(P[oW1 + j * kIn + k0 + 1]) : 0.0f;
            w[q] = pack_bf16x2(a, b);
        }
        *reinterpret_cast<uint4*>(sm.w1 + um::sw128(j, c)) = make_uint4(w[0], w[1], w[2], w[3]);
    }
    for (uint32_t e = tid; e < kH * 16; e += kTcTile) {  // W2: 16 chunks of 8 BF16 per row, two blocks
        const uint32_t j = e >> 4, c = e & 15u;
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(P + oW2 + j * kH + c * 8));  // oW2 % 8 == 0
        *reinterpret_cast<uint4*>(sm.w2[c >> 3] + um::sw128(j, c & 7u)) = v;
    }
    sm.b1[tid] = ldb(P + oB1 + tid);
    sm.b2[tid] = ldb(P + oB2 + tid);
    sm.w3[tid] = ldb(P + oW3 + tid);
    const float b3 = ldb(P + oB3);
    if (tid == 0) {
        um::mbar_init(um::smem_u32(&sm.bar[0]), 1);
        um::mbar_init(um::smem_u32(&sm.bar[1]), 1);
        sm.fail = 0;
    }
    if (warp == 0)
        um::tmem_alloc(&sm.tmem, 2 * kH);
    um::fence_before_sync();
    __syncthreads();
    um::fence_after_sync();
    const uint32_t tmem = sm.tmem;
    const uint32_t lane_base = (32u * warp) << 16;  // this warp's TMEM lanes
    const double sc = mul ? scale * mul[0] : scale;
    constexpr uint32_t kId = pvl::umma::idesc_bf16(kTcTile, kH);
    uint32_t phase = 0;
    for (uint64_t s0 = (uint64_t)blockIdx.x * kTcTile; s0 < n; s0 += (uint64_t)gridDim.x * kTcTile, phase ^= 1u) {
        // the tile's inputs, BF16, two 16-byte chunks per row (K 0..15, 12..15 zero)
        {
            const uint64_t s = s0 + tid;
            float f[16];
#pragma unroll
            for (int i = 0; i < 16; ++i)
                f[i] = (i < kIn && s < n) ? X[s * kIn + i] : 0.0f;
            uint32_t w[8];
#pragma unroll
            for (int q = 0; q < 8; ++q)
                w[q] = pack_bf16x2(f[2 * q], f[2 * q + 1]);
            *reinterpret_cast<uint4*>(sm.x + um::sw128(tid, 0)) = make_uint4(w[0], w[1], w[2], w[3]);
            *reinterpret_cast<uint4*>(sm.x + um::sw128(tid, 1)) = make_uint4(w[4], w[5], w[6], w[7]);
        }
        um::fence_proxy_async();
        um::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            um::fence_after_sync();
            um::mma<false>(tmem, um::sw128_desc(um::smem_u32(sm.x)), um::sw128_desc(um::smem_u32(sm.w1)), kId, 0u);
            um::commit(um::smem_u32(&sm.bar[0]));
        }
        bool ok = um::mbar_wait(um::smem_u32(&sm.bar[0]), phase);
        um::fence_after_sync();
        // H1 row tid: bf16(relu(acc1 + b1)), 16 columns at a time into the two K blocks
#pragma unroll 1
        for (uint32_t c0 = 0; c0 < kH; c0 += 16) {
            float v[16];
            __syncwarp();
            um::tmem_ld16(tmem + lane_base + c0, v);
            uint32_t w[8];
#pragma unroll
            for (int q = 0; q < 8; ++q)
                w[q] = pack_bf16x2(fmaxf(v[2 * q] + sm.b1[c0 + 2 * q], 0.0f),
                                   fmaxf(v[2 * q + 1] + sm.b1[c0 + 2 * q + 1], 0.0f));
            unsigned char* blk = sm.h1[c0 >> 6];
            const uint32_t ch = (c0 & 63u) >> 3;
            *reinterpret_cast<uint4*>(blk + um::sw128(tid, ch)) = make_uint4(w[0], w[1], w[2], w[3]);
            *reinterpret_cast<uint4*>(blk + um::sw128(tid, ch + 1)) = make_uint4(w[4], w[5], w[6], w[7]);
        }
        um::fence_proxy_async();
        um::fence_before_sync();
        if (__syncthreads_or(!ok))
            ok = false;
        if (tid == 0 && ok) {
            um::fence_after_sync();
#pragma unroll
            for (uint32_t ks = 0; ks < kH / 16; ++ks) {  // K = 16 BF16 = 32 bytes per step
                const uint32_t blk = ks >> 2, step = 2u * (ks & 3u);
                um::mma<false>(tmem + kH, um::sw128_desc(um::smem_u32(sm.h1[blk])) + step,
                               um::sw128_desc(um::smem_u32(sm.w2[blk])) + step, kId, ks ? 1u : 0u);
            }
        }
        if (tid == 0)
            um::commit(um::smem_u32(&sm.bar[1]));  // arrives even without MMAs (all earlier ones done)
        ok = um::mbar_wait(um::smem_u32(&sm.bar[1]), phase) && ok;
        um::fence_after_sync();
        float y = b3;
#pragma unroll 1
        for (uint32_t c0 = 0; c0 < kH; c0 += 16) {
            float v[16];
            __syncwarp();
            um::tmem_ld16(tmem + lane_base + kH + c0, v);
#pragma unroll
            for (int i = 0; i < 16; ++i)
                y = fmaf(sm.w3[c0 + i], bf(fmaxf(v[i] + sm.b2[c0 + i], 0.0f)), y);
        }
        const uint64_t s = s0 + tid;
        if (s < n)
            out[s] = ok ? (base ? base[s] : 0.0) + sc * (double)y : __longlong_as_double(0x7FF8000000000000ll);
        um::fence_before_sync();
        __syncthreads();
    }
    um::fence_after_sync();
    if (warp == 0)
        um::tmem_dealloc(tmem, 2 * kH);
}

// ---------------------------------------------------------------- training on the tensor cores
// Forward + backward of mean((y - t)^2) over 128-sample tiles, persistent CTAs of 128 threads
// (thread s = sample s of the tile = TMEM lane s).  Per tile, three stages of tcgen05.mma
// kind::f16 (BF16 operands, FP32 accumulators in tensor memory):
//   1. acc1 = X W1^T (K = 16: the 12 inputs, zero-padded)          -> h1 = bf16(relu(acc1 + b1))
//   2. acc2 = H1 W2^T (K = 128)                                     -> h2, y, dy = 2 (y - t) / n,
//      dh2 = [h2 > 0] dy w3 (rounded to BF16 as an MMA operand)
//   3. dH1 = dH2 W2 (K = 128, into acc1's columns)  and  dW2 += dH2^T H1 (K = 128 samples,
//      accumulated in TMEM over all tiles of the CTA).
// The operands of stage 3 need H1 and dH2 also transposed (samples along K): the epilogue
// threads write both layouts.  db2 and dw3 are per-unit sums over samples: warp reductions
// (halving exchange, 16 shuffles per 16 columns) then a fixed-order sum over the 4 warps;
// db1 and dW1 = sum_s dh1[s][k] x[s][i] on CUDA cores from dh1 staged in shared memory, a
// unit per thread.  Every sum runs in a fixed order: the same data give the same gradient bit
// for bit.  Shared memory is time-shared: X then dH2 in r1, H1 then dH2^T in r2, H1^T in r3,
// and r2 + r3 hold dh1 (FP32) for the CUDA-core phase.  Waits are bounded; one that runs out
// poisons the partial gradient with NaN (training then stops on the loss).
struct TrainTcSmem {
    unsigned char w1[kH * 128];        // W1: N = 128 units x K (12 used)
    unsigned char w2[2][kH * 128];     // W2: N = j x K = k (stage 2's B)
    unsigned char w2t[2][kH * 128];    // W2^T: N = k x K = j (stage 3's B for dH1)
    unsigned char r1[2][kTcTile * 128];
    unsigned char r2[2][kTcTile * 128];
    unsigned char r3[2][kH * 128];
    float xs[kTcTile][kIn];            // the tile's inputs, BF16-rounded
    float b1[kH], b2[kH], w3[kH];
    float red[4][2 * kH];              // per-warp dw3 | db2 partials
    float lred[4];
    uint64_t bar[3];
    uint32_t tmem;
};
static_assert(sizeof(TrainTcSmem) + 1024 <= 227 * 1024, "training tile fits one CTA's shared memory");

// Sum of v[0..15] over the warp's 32 lanes by halving exchanges; lane l ends with the sum for
// column (l >> 1) & 15 (lanes l and l ^ 1 alike).
__device__ __forceinline__ float warp_sum16(float (&v)[16], uint32_t lane)
{
#pragma unroll
    for (int h = 8, o = 16; h >= 1; h >>= 1, o >>= 1) {
#pragma unroll
        for (int i = 0; i < h; ++i) {
            const bool up = (lane & (uint32_t)o) != 0;
            const float send = up ? v[i] : v[i + h];
            const float keep = up ? v[i + h] : v[i];
            v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
        }
    }
    return v[0] + __shfl_xor_sync(0xffffffffu, v[0], 1);
}

// element (row, k) of a BF16 K-major SW128 tile made of 64-wide column blocks of `rows` rows
__device__ __forceinline__ void st_bf16(unsigned char* tile, uint32_t rows, uint32_t row, uint32_t k, float v)
{
    unsigned char* blk = tile + (size_t)(k >> 6) * rows * 128u;
    *reinterpret_cast<__nv_bfloat16*>(blk + pvl::umma::sw128(row, (k & 63u) >> 3) + (k & 7u) * 2u) =
        __float2bfloat16_rn(v);
}

__global__ void __launch_bounds__(kTcTile, 1) train_tc_kernel(uint32_t n, double n_total, const float* __restrict__ X,
                                                              const float* __restrict__ T,
                                                              const __nv_bfloat16* __restrict__ P,
                                                              float* __restrict__ part, float* __restrict__ part_loss)
{
    namespace um = pvl::umma;
    extern __shared__ __align__(1024) unsigned char tr_raw[];
    TrainTcSmem& sm = *reinterpret_cast<TrainTcSmem*>(tr_raw + ((1024u - (um::smem_u32(tr_raw) & 1023u)) & 1023u));
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    // weights: W1 and W2 rows as they are (unit j = N index), W2^T row k = column k of W2
    for (uint32_t e = tid; e < kH * 8; e += kTcTile) {
        const uint32_t j = e >> 3, c = e & 7u;
        uint32_t w[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint32_t k0 = c * 8 + 2 * q;
            const float a = k0 < kIn ? __bfloat162float(P[oW1 + j * kIn + k0]) : 0.0f;
            const float b = k0 + 1 < kIn ? __bfloat162float(P[oW1 + j * kIn + k0 + 1]) : 0.0f;
            w[q] = pack_bf16x2(a, b);
        }
        *reinterpret_cast<uint4*>(sm.w1 + um::sw128(j, c)) = make_uint4(w[0], w[1], w[2], w[3]);
    }
    for (uint32_t e = tid; e < kH * 16; e += kTcTile) {
        const uint32_t j = e >> 4, c = e & 15u;
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(P + oW2 + j * kH + c * 8));
        *reinterpret_cast<uint4*>(sm.w2[c >> 3] + um::sw128(j, c & 7u)) = v;
    }
    for (uint32_t e = tid; e < kH * kH; e += kTcTile) {  // W2^T[k][j] = W2[j][k]
        const uint32_t j = e / kH, k = e % kH;
        const float v = __bfloat162float(P[oW2 + e]);
        st_bf16(&sm.w2t[0][0], kH, k, j, v);
    }
    sm.b1[tid] = ldb(P + oB1 + tid);
    sm.b2[tid] = ldb(P + oB2 + tid);
    sm.w3[tid] = ldb(P + oW3 + tid);
    const float b3 = ldb(P + oB3);
    if (tid == 0)
        for (int i = 0; i < 3; ++i)
            um::mbar_init(um::smem_u32(&sm.bar[i]), 1);
    if (warp == 0)
        um::tmem_alloc(&sm.tmem, 512);
    um::fence_proxy_async();
    um::fence_before_sync();
    __syncthreads();
    um::fence_after_sync();
    const uint32_t tmem = sm.tmem;
    const uint32_t lane_base = (32u * warp) << 16;
    constexpr uint32_t kId = pvl::umma::idesc_bf16(kTcTile, kH);
    const float inv_n = (float)(2.0 / n_total);
    float dW1[kIn], db1 = 0.0f, acc_dw3[8], acc_db2[8], loss = 0.0f, db3 = 0.0f;
#pragma unroll
    for (int i = 0; i < kIn; ++i)
        dW1[i] = 0.0f;
#pragma unroll
    for (int i = 0; i < 8; ++i)
        acc_dw3[i] = acc_db2[i] = 0.0f;
    bool ok = true;
    uint32_t ti = 0;
    for (uint64_t s0 = (uint64_t)blockIdx.x * kTcTile; s0 < n; s0 += (uint64_t)gridDim.x * kTcTile, ++ti) {
        const uint32_t ph = ti & 1u;
        const uint64_t smp = s0 + tid;
        const bool valid = smp < n;
        // ---- inputs: BF16 into X (r1) and as FP32 values for dW1
        {
            float f[16];
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                f[i] = (i < kIn && valid) ? bf(X[smp * kIn + i]) : 0.0f;
                if (i < kIn)
                    sm.xs[tid][i] = f[i];
            }
            uint32_t w[8];
#pragma unroll
            for (int q = 0; q < 8; ++q)
                w[q] = pack_bf16x2(f[2 * q], f[2 * q + 1]);
            *reinterpret_cast<uint4*>(sm.r1[0] + um::sw128(tid, 0)) = make_uint4(w[0], w[1], w[2], w[3]);
            *reinterpret_cast<uint4*>(sm.r1[0] + um::sw128(tid, 1)) = make_uint4(w[4], w[5], w[6], w[7]);
        }
        um::fence_proxy_async();
        um::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            um::fence_after_sync();
            um::mma<false>(tmem, um::sw128_desc(um::smem_u32(sm.r1[0])), um::sw128_desc(um::smem_u32(sm.w1)), kId, 0u);
            um::commit(um::smem_u32(&sm.bar[0]));
        }
        ok = um::mbar_wait(um::smem_u32(&sm.bar[0]), ph) && ok;
        um::fence_after_sync();
        // ---- h1 = bf16(relu(acc1 + b1)) into H1 (r2, rows s) and H1^T (r3, rows k); its ReLU mask
        uint32_t mask[4] = {0u, 0u, 0u, 0u};
#pragma unroll 1
        for (uint32_t c0 = 0; c0 < kH; c0 += 16) {
            float v[16];
            __syncwarp();
            um::tmem_ld16(tmem + lane_base + c0, v);
            uint32_t w[8];
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                v[i] = bf(fmaxf(v[i] + sm.b1[c0 + i], 0.0f));
                if (v[i] > 0.0f)
                    mask[(c0 + i) >> 5] |= 1u << ((c0 + i) & 31u);
                st_bf16(&sm.r3[0][0], kH, c0 + i, tid, v[i]);
            }
#pragma unroll
            for (int q = 0; q < 8; ++q)
                w[q] = pack_bf16x2(v[2 * q], v[2 * q + 1]);
            unsigned char* blk = sm.r2[c0 >> 6];
            const uint32_t ch = (c0 & 63u) >> 3;
            *reinterpret_cast<uint4*>(blk + um::sw128(tid, ch)) = make_uint4(w[0], w[1], w[2], w[3]);
            *reinterpret_cast<uint4*>(blk + um::sw128(tid, ch + 1)) = make_uint4(w[4], w[5], w[6], w[7]);
        }
        um::fence_proxy_async();
        um::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            um::fence_after_sync();
#pragma unroll
            for (uint32_t ks = 0; ks < kH / 16; ++ks) {
                const uint32_t blk = ks >> 2, step = 2u * (ks & 3u);
                um::mma<false>(tmem + kH, um::sw128_desc(um::smem_u32(sm.r2[blk])) + step,
                               um::sw128_desc(um::smem_u32(sm.w2[blk])) + step, kId, ks ? 1u : 0u);
            }
            um::commit(um::smem_u32(&sm.bar[1]));
        }
        ok = um::mbar_wait(um::smem_u32(&sm.bar[1]), ph) && ok;
        um::fence_after_sync();
        // ---- output, loss and dy
        float y = b3;
#pragma unroll 1
        for (uint32_t c0 = 0; c0 < kH; c0 += 16) {
            float v[16];
            __syncwarp();
            um::tmem_ld16(tmem + lane_base + kH + c0, v);
#pragma unroll
            for (int i = 0; i < 16; ++i)
                y = fmaf(sm.w3[c0 + i], bf(fmaxf(v[i] + sm.b2[c0 + i], 0.0f)), y);
        }
        float dy = 0.0f;
        if (valid) {
            const float r = y - T[smp];
            loss += r * r;
            dy = r * inv_n;
        }
        db3 += dy;
        // ---- dh2 = [h2 > 0] dy w3 into dH2 (r1, rows s) and dH2^T (r2, rows j); dw3 and db2 sums
#pragma unroll 1
        for (uint32_t c0 = 0; c0 < kH; c0 += 16) {
            float v[16], g[16], hv[16];
            __syncwarp();
            um::tmem_ld16(tmem + lane_base + kH + c0, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) {
                const float h2 = bf(fmaxf(v[i] + sm.b2[c0 + i], 0.0f));
                g[i] = h2 > 0.0f ? dy * sm.w3[c0 + i] : 0.0f;
                hv[i] = dy * h2;
                st_bf16(&sm.r1[0][0], kTcTile, tid, c0 + i, g[i]);
                st_bf16(&sm.r2[0][0], kH, c0 + i, tid, g[i]);
            }
            const uint32_t slot = c0 >> 4;
            acc_dw3[slot] += warp_sum16(hv, lane);
            acc_db2[slot] += warp_sum16(g, lane);
        }
        um::fence_proxy_async();
        um::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            um::fence_after_sync();
#pragma unroll
            for (uint32_t ks = 0; ks < kH / 16; ++ks) {  // dH1 = dH2 W2 (acc1's columns)
                const uint32_t blk = ks >> 2, step = 2u * (ks & 3u);
                um::mma<false>(tmem, um::sw128_desc(um::smem_u32(sm.r1[blk])) + step,
                               um::sw128_desc(um::smem_u32(sm.w2t[blk])) + step, kId, ks ? 1u : 0u);
            }
#pragma unroll
            for (uint32_t ks = 0; ks < kTcTile / 16; ++ks) {  // dW2 += dH2^T H1 over the tile's samples
                const uint32_t blk = ks >> 2, step = 2u * (ks & 3u);
                um::mma<false>(tmem + 2 * kH, um::sw128_desc(um::smem_u32(sm.r2[blk])) + step,
                               um::sw128_desc(um::smem_u32(sm.r3[blk])) + step, kId, (ti | ks) ? 1u : 0u);
            }
            um::commit(um::smem_u32(&sm.bar[2]));
        }
        ok = um::mbar_wait(um::smem_u32(&sm.bar[2]), ph) && ok;
        um::fence_after_sync();
        // ---- dh1 = [h1 > 0] dH1, staged FP32 (r2 + r3, 16-byte chunks XOR-swizzled by row)
        float* D = reinterpret_cast<float*>(sm.r2);
#pragma unroll 1
        for (uint32_t c0 = 0; c0 < kH; c0 += 16) {
            float v[16];
            __syncwarp();
            um::tmem_ld16(tmem + lane_base + c0, v);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                float4 o;
                float* op = &o.x;
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const uint32_t k = c0 + 4 * q + i;
                    op[i] = (mask[k >> 5] >> (k & 31u)) & 1u ? v[4 * q + i] : 0.0f;
                }
                const uint32_t chunk = ((c0 >> 2) + q) ^ (tid & 31u);
                *reinterpret_cast<float4*>(D + tid * kH + chunk * 4) = o;
            }
        }
        um::fence_before_sync();
        __syncthreads();
        // ---- unit k = tid: db1, dW1 over the tile's samples
        for (uint32_t s_ = 0; s_ < (uint32_t)kTcTile; ++s_) {
            const float g = D[s_ * kH + ((((tid >> 2) ^ (s_ & 31u)) << 2) | (tid & 3u))];
            db1 += g;
#pragma unroll
            for (int i = 0; i < kIn; ++i)
                dW1[i] = fmaf(g, sm.xs[s_][i], dW1[i]);
        }
        __syncthreads();  // r1..r3 and xs are rewritten by the next tile
    }
    // ---- this CTA's partial gradient
    um::fence_after_sync();
    float* g = part + (size_t)blockIdx.x * kParams;
    if (ti > 0) {
#pragma unroll 1
        for (uint32_t c0 = 0; c0 < kH; c0 += 16) {  // dW2 row j = tid (TMEM lane)
            float v[16];
            __syncwarp();
            um::tmem_ld16(tmem + lane_base + 2 * kH + c0, v);
#pragma unroll
            for (int i = 0; i < 16; ++i)
                g[oW2 + tid * kH + c0 + i] = ok ? v[i] : __int_as_float(0x7FC00000);
        }
    } else {
        for (uint32_t k = 0; k < kH; ++k)
            g[oW2 + tid * kH + k] = 0.0f;
    }
    if ((lane & 1u) == 0)
#pragma unroll
        for (int slot = 0; slot < 8; ++slot) {
            sm.red[warp][slot * 16 + ((lane >> 1) & 15u)] = acc_dw3[slot];
            sm.red[warp][kH + slot * 16 + ((lane >> 1) & 15u)] = acc_db2[slot];
        }
    float lsum = loss, d3 = db3;
    for (int o = 16; o > 0; o >>= 1) {
        lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
        d3 += __shfl_xor_sync(0xffffffffu, d3, o);
    }
    __syncthreads();
    const float dw3 = ((sm.red[0][tid] + sm.red[1][tid]) + sm.red[2][tid]) + sm.red[3][tid];
    const float db2 = ((sm.red[0][kH + tid] + sm.red[1][kH + tid]) + sm.red[2][kH + tid]) + sm.red[3][kH + tid];
    const float bad = ok ? 0.0f : __int_as_float(0x7FC00000);
#pragma unroll
    for (int i = 0; i < kIn; ++i)
        g[oW1 + tid * kIn + i] = dW1[i] + bad;
    g[oB1 + tid] = db1 + bad;
    g[oB2 + tid] = db2 + bad;
    g[oW3 + tid] = dw3 + bad;
    __syncthreads();
    if (lane == 0) {
        sm.red[warp][0] = lsum;
        sm.red[warp][1] = d3;
    }
    __syncthreads();
    if (tid == 0) {
        g[oB3] = ((sm.red[0][1] + sm.red[1][1]) + sm.red[2][1]) + sm.red[3][1] + bad;
        part_loss[blockIdx.x] = ((sm.red[0][0] + sm.red[1][0]) + sm.red[2][0]) + sm.red[3][0] + bad;
    }
    um::fence_before_sync();
    __syncthreads();
    um::fence_after_sync();
    if (warp == 0)
        um::tmem_dealloc(tmem, 512);
}

// grad[p] = sum over CTAs of part[c * kParams + p], in CTA order; loss likewise (thread 0).
__global__ void reduce_kernel(uint32_t n_parts, const float* __restrict__ part, const float* __restrict__ part_loss,
                              double n_total, float* __restrict__ grad, float* __restrict__ loss)
{
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < kParams) {
        float s = 0.0f;
        for (uint32_t c = 0; c < n_parts; ++c)
            s += part[(size_t)c * kParams + p];
        grad[p] = s;
    }
    if (p == 0 && loss) {
        double s = 0.0;
        for (uint32_t c = 0; c < n_parts; ++c)
            s += part_loss[c];
        *loss = (float)(s / n_total);
    }
}

__global__ void adam_kernel(float* __restrict__ w, __nv_bfloat16* __restrict__ wb, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, float lr, float b1, float b2, float eps,
                            float c1, float c2)
{
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= kParams)
        return;
    const float gp = g[p];
    const float mp = b1 * m[p] + (1.0f - b1) * gp;
    const float vp = b2 * v[p] + (1.0f - b2) * gp * gp;
    m[p] = mp;
    v[p] = vp;
    const float wn = w[p] - lr * (mp / c1) / (sqrtf(vp / c2) + eps);
    w[p] = wn;
    wb[p] = __float2bfloat16_rn(wn);
}

__global__ void to_bf16_kernel(uint32_t n, const float* __restrict__ w, __nv_bfloat16* __restrict__ wb)
{
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p < n)
        wb[p] = __float2bfloat16_rn(w[p]);
}

// Inputs of panel i (before normalisation):
//   0 g0            1 g0 - g1        2 rem0           3 r_i / A_ii (r = b - A g0: one Jacobi step)
//   4 b_i           5 b_i - bprev_i  6 A_ii + 2 pi    7..9 normal
//   10 normal . control-point velocity               11 rem1
// where rem0 / rem1 are what the last two steps' solutions added to their own Jacobi
// corrections (gamma - base), the quantity the network predicts for this step.  The
// increments (1, 2, 3, 5, 11) are divided by the step scale s = ||r|| / sqrt(n), so that the
// network sees the shape of this step's change, not its size (s = 1 when r = 0).
// X[i][f] = (v_f - mean_f) * inv_std_f; base[i] = g0_i + r_i / A_ii.
__global__ void features_kernel(uint32_t n, const double* __restrict__ g0, const double* __restrict__ g1,
                                const double* __restrict__ rem0, const double* __restrict__ rem1,
                                const double* __restrict__ resid, const double* __restrict__ rnorm,
                                const double* __restrict__ A, uint32_t lda,
                                const double* __restrict__ rhs, const double* __restrict__ rhs_prev,
                                const double* __restrict__ nrm, const double* __restrict__ cpv,
                                const float* __restrict__ mean, const float* __restrict__ inv_std,
                                float* __restrict__ X, double* __restrict__ base)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    const double aii = A[(size_t)i * lda + i];
    const double jac = aii != 0.0 ? resid[i] / aii : 0.0;
    const double nx = nrm[3 * (size_t)i], ny = nrm[3 * (size_t)i + 1], nz = nrm[3 * (size_t)i + 2];
    const double rn = rnorm[0] / sqrt((double)n);
    const double inv_s = rn > 0.0 ? 1.0 / rn : 1.0;
    double f[kIn];
    f[0] = g0[i];
    f[1] = (g0[i] - g1[i]) * inv_s;
    f[2] = rem0[i] * inv_s;
    f[3] = jac * inv_s;
    f[4] = rhs[i];
    f[5] = (rhs[i] - rhs_prev[i]) * inv_s;
    f[6] = aii + 6.283185307179586;
    f[7] = nx;
    f[8] = ny;
    f[9] = nz;
    f[10] = nx * cpv[3 * (size_t)i] + ny * cpv[3 * (size_t)i + 1] + nz * cpv[3 * (size_t)i + 2];
    f[11] = rem1[i] * inv_s;
#pragma unroll
    for (int k = 0; k < kIn; ++k)
        X[(size_t)i * kIn + k] = (float)((f[k] - (double)mean[k]) * (double)inv_std[k]);
    base[i] = g0[i] + jac;
}

int set_attrs()
{
    PVL_SMEM_OPTIN(forward_tc_kernel, sizeof(FwdTcSmem) + 1024);
    PVL_SMEM_OPTIN(train_tc_kernel, sizeof(TrainTcSmem) + 1024);
    return PVL_OK;
}

}  // namespace

extern "C" uint32_t pvl_mlp_param_count(void) { return kParams; }

extern "C" uint32_t pvl_mlp_input_count(void) { return kIn; }

extern "C" size_t pvl_mlp_train_workspace(uint32_t n_ctas)
{
    return ((size_t)n_ctas * kParams + n_ctas + kParams + 64) * sizeof(float);
}

extern "C" int pvl_mlp_features(uint32_t n, const double* g0, const double* g1, const double* rem0,
                                const double* rem1, const double* resid, const double* rnorm, const double* A,
                                uint32_t lda,
                                const double* rhs, const double* rhs_prev, const double* normals, const double* cp_vel,
                                const float* mean, const float* inv_std, float* X, double* base, void* stream)
{
    if (n == 0)
        return PVL_OK;
    if (!g0 || !g1 || !rem0 || !rem1 || !resid || !rnorm || !A || !rhs || !rhs_prev || !normals || !cp_vel || !mean ||
        !inv_std || !X || !base)
        return pvl_fail(PVL_ERR_ARG, "pvl_mlp_features: null pointer argument");
    if (lda < n)
        return pvl_fail(PVL_ERR_ARG, "pvl_mlp_features: lda < n");
    features_kernel<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(n, g0, g1, rem0, rem1, resid, rnorm, A, lda, rhs,
                                                                         rhs_prev, normals, cp_vel, mean, inv_std, X,
                                                                         base);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_mlp_forward(uint32_t n, const float* X, const void* params_bf16, double scale, const double* mul,
                               const double* base, double* out, void* stream)
{
    if (n == 0)
        return PVL_OK;
    if (!X || !params_bf16 || !out)
        return pvl_fail(PVL_ERR_ARG, "pvl_mlp_forward: null pointer argument");
    if (int r = set_attrs())
        return r;
    const unsigned grid = (unsigned)std::min<uint64_t>(blocks_for(n, kTcTile), 148ull * 2);
    forward_tc_kernel<<<grid, kTcTile, sizeof(FwdTcSmem) + 1024, (cudaStream_t)stream>>>(
        n, X, static_cast<const __nv_bfloat16*>(params_bf16), scale, mul, base, out);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_mlp_gradient(uint32_t n, const float* X, const float* T, const void* params_bf16, uint32_t n_ctas,
                                float* grad, float* loss, void* ws, size_t ws_bytes, void* stream)
{
    if (!X || !T || !params_bf16 || !grad || !ws)
        return pvl_fail(PVL_ERR_ARG, "pvl_mlp_gradient: null pointer argument");
    if (n == 0 || n_ctas == 0)
        return pvl_fail(PVL_ERR_ARG, "pvl_mlp_gradient: empty batch or no CTAs");
    if (ws_bytes < pvl_mlp_train_workspace(n_ctas))
        return pvl_fail(PVL_ERR_ALLOC, "pvl_mlp_gradient: workspace too small");
    if (int r = set_attrs())
        return r;
    cudaStream_t st = (cudaStream_t)stream;
    float* part = static_cast<float*>(ws);
    float* part_loss = part + (size_t)n_ctas * kParams;
    const unsigned grid = (unsigned)std::min<uint64_t>(n_ctas, blocks_for(n, kTcTile));
    train_tc_kernel<<<grid, kTcTile, sizeof(TrainTcSmem) + 1024, st>>>(
        n, (double)n, X, T, static_cast<const __nv_bfloat16*>(params_bf16), part, part_loss);
    PVL_LAUNCH_CHECK();
    reduce_kernel<<<blocks_for(kParams, 256), 256, 0, st>>>(grid, part, part_loss, (double)n, grad, loss);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_mlp_adam(float* params, void* params_bf16, const float* grad, float* m, float* v, uint32_t step,
                            float lr, float beta1, float beta2, float eps, void* stream)
{
    if (!params || !params_bf16 || !grad || !m || !v)
        return pvl_fail(PVL_ERR_ARG, "pvl_mlp_adam: null pointer argument");
    if (step == 0)
        return pvl_fail(PVL_ERR_ARG, "pvl_mlp_adam: steps count from 1");
    const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
    adam_kernel<<<blocks_for(kParams, 256), 256, 0, (cudaStream_t)stream>>>(
        params, static_cast<__nv_bfloat16*>(params_bf16), grad, m, v, lr, beta1, beta2, eps, c1, c2);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_mlp_to_bf16(const float* params, void* params_bf16, void* stream)
{
    if (!params || !params_bf16)
        return pvl_fail(PVL_ERR_ARG, "pvl_mlp_to_bf16: null pointer argument");
    to_bf16_kernel<<<blocks_for(kParams, 256), 256, 0, (cudaStream_t)stream>>>(
        kParams, params, static_cast<__nv_bfloat16*>(params_bf16));
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}
