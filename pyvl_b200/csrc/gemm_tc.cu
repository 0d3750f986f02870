// Tensor-core GEMM on sm_100a: C = alpha * A * B + beta * C with FP32 storage, TF32 inputs
// and FP32 accumulation (tcgen05.mma kind::tf32, accumulator in tensor memory).
//
// Used by the low-precision preconditioner (the approximate inverse of the system matrix,
// rebuilt when it goes stale, and the trailing update of the FP32 LU).  Row-major A (M x K),
// B (K x N), C (M x N); any M and N (rows and columns past the edge of a tile are staged as
// zeros and not stored), K a multiple of 32, leading dimensions multiples of 4 floats,
// 16-byte aligned bases.
//
// One CTA = one 128 x 128 output tile, 128 threads.  The K loop runs over 32-wide tiles in two
// shared-memory stages of 32 KB (A tile and B^T tile, both stored K-major in the canonical
// 128-byte-swizzled UMMA layout: row r of an 8-row group at byte (r/8)*1024 + (r%8)*128, its
// 16-byte chunk c at chunk c ^ (r%8)).  All threads stage a tile (A straight from its rows,
// B transposed on the way); thread 0 issues four K=8 MMAs per tile and commits them to the
// stage's mbarrier, which the threads wait on before overwriting that stage.  After the last
// tile the four warps read their 32 TMEM lanes (rows) back with tcgen05.ld into a shared FP32
// tile, and then combine it with C in coalesced rows.  Every wait is bounded; a time-out sets *err and the CTA still waits (bounded) for
// its own MMAs and frees its tensor memory before returning.
#include <cstdint>

#include "pvl_common.cuh"

namespace {

constexpr int kTile = 128;       // M and N of a CTA tile (one UMMA 128 x 128)
constexpr int kKT = 32;          // K per shared-memory stage (128 bytes of TF32)
constexpr int kStages = 2;
constexpr int kThreads = 128;
constexpr int kStageBytes = 2 * kTile * kKT * 4;  // A + B^T tiles
constexpr long long kWaitLimit = 1ll << 22;       // polls (each may suspend briefly) before a wait gives up

__device__ __forceinline__ uint32_t smem_u32(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of (row, 16-byte chunk) inside a 128-row x 128-byte SW128 K-major tile.
__device__ __forceinline__ uint32_t sw128(uint32_t row, uint32_t chunk)
{
    return (row >> 3) * 1024u + (row & 7u) * 128u + ((chunk ^ (row & 7u)) << 4);
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t sw128_desc(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);   // start address (16-byte units)
    d |= (uint64_t)1u << 16;                   // leading byte offset (unused for swizzled K-major)
    d |= (uint64_t)(1024u >> 4) << 32;         // stride byte offset: next 8-row group
    d |= (uint64_t)1u << 46;                   // descriptor version for sm_100
    d |= (uint64_t)2u << 61;                   // layout: 128-byte swizzle
    return d;
}

// Instruction descriptor: D FP32, A and B TF32, both K-major, M = 128, N = 128.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTile >> 3) << 17) |
                            ((uint32_t)(kTile >> 4) << 24);

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity)
{
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(parity)
        : "memory");
    return done != 0;
}

// Bounded wait for the phase with the given parity; false on time-out.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    for (long long i = 0; i < kWaitLimit; ++i)
        if (mbar_try_wait(bar, parity))
            return true;
    return false;
}

__device__ __forceinline__ void umma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint32_t bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
                 : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i)
        v[i] = __uint_as_float(r[i]);
}

__global__ void __launch_bounds__(kThreads) gemm_tf32_kernel(uint32_t M, uint32_t N, uint32_t K, float alpha,
                                                             const float* __restrict__ A, uint32_t lda,
                                                             const float* __restrict__ B, uint32_t ldb, float beta,
                                                             float* __restrict__ C, uint32_t ldc,
                                                             int32_t* __restrict__ err)
{
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // 1024-byte aligned stage buffers (the swizzle pattern is anchored at 1024 B)
    unsigned char* smem = smem_raw + ((1024u - (smem_u32(smem_raw) & 1023u)) & 1023u);
    __shared__ __align__(8) uint64_t bars[kStages];
    __shared__ uint32_t tmem_base;
    __shared__ int s_fail;

    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t m0 = blockIdx.y * kTile, n0 = blockIdx.x * kTile;
    if (tid == 0) {
        for (int s = 0; s < kStages; ++s)
            mbar_init(smem_u32(&bars[s]), 1);
        s_fail = 0;
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                     "r"((uint32_t)kTile)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base;

    const uint32_t n_kt = K / kKT;
    int32_t last_committed = -1;  // tile whose commit covers every MMA issued so far
    for (uint32_t kt = 0; kt < n_kt; ++kt) {
        const uint32_t s = kt % kStages;
        unsigned char* sa = smem + s * kStageBytes;
        unsigned char* sb = sa + kTile * kKT * 4;
        if (kt >= kStages) {
            // the MMAs that last read this stage (tile kt - kStages) must be done
            const uint32_t parity = ((kt - kStages) / kStages) & 1u;
            if (!mbar_wait(smem_u32(&bars[s]), parity))
                atomicExch(&s_fail, 1);
        }
        __syncthreads();
        if (s_fail)
            break;
        const uint32_t k0 = kt * kKT;
        // A tile: 128 rows x 32 floats, 8 chunks of 16 B per row
#pragma unroll
        for (int g = 0; g < (kTile * kKT / 4) / kThreads; ++g) {
            const uint32_t idx = tid + g * kThreads;
            const uint32_t r = idx >> 3, c = idx & 7u;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (m0 + r < M)
                v = *reinterpret_cast<const float4*>(A + (size_t)(m0 + r) * lda + k0 + 4 * c);
            *reinterpret_cast<float4*>(sa + sw128(r, c)) = v;
        }
        // B^T tile: row n holds B[k0 .. k0+31][n0 + n]; four consecutive k per 16-byte chunk
#pragma unroll
        for (int g = 0; g < (kTile * kKT / 4) / kThreads; ++g) {
            const uint32_t idx = tid + g * kThreads;
            const uint32_t n = idx & (kTile - 1), c = idx >> 7;
            float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
            if (n0 + n < N) {
                const float* src = B + (size_t)(k0 + 4 * c) * ldb + n0 + n;
                v.x = src[0];
                v.y = src[(size_t)ldb];
                v.z = src[2 * (size_t)ldb];
                v.w = src[3 * (size_t)ldb];
            }
            *reinterpret_cast<float4*>(sb + sw128(n, c)) = v;
        }
        // generic-proxy stores -> visible to the tensor core's async proxy
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint64_t da = sw128_desc(smem_u32(sa)), db = sw128_desc(smem_u32(sb));
#pragma unroll
            for (uint32_t ks = 0; ks < kKT / 8; ++ks)  // K = 8 TF32 (32 bytes) per MMA
                umma_tf32(tmem, da + 2u * ks, db + 2u * ks, kIdesc, (kt | ks) ? 1u : 0u);
            umma_commit(smem_u32(&bars[s]));
        }
        last_committed = (int32_t)kt;
    }
    // wait for the last MMAs this CTA issued (their commit covers all earlier ones)
    __syncthreads();
    bool ok = !s_fail && last_committed == (int32_t)n_kt - 1;
    if (last_committed >= 0) {
        const uint32_t last = (uint32_t)last_committed, s = last % kStages;
        if (!mbar_wait(smem_u32(&bars[s]), (last / kStages) & 1u))
            ok = false;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (!ok) {
        if (tid == 0)
            atomicExch(err, 1);
    } else if (n_kt > 0) {
        // epilogue, two phases through the (now idle) stage buffers:
        // 1. warp w reads its 32 TMEM lanes (rows 32w .. 32w+31) and stores them row-wise into a
        //    128 x 128 FP32 tile, 16-byte chunks XOR-swizzled by (row & 7) (conflict-free);
        // 2. each warp walks rows w, w+4, ..., lane l owning columns 4l .. 4l+3, so that C is read
        //    and written in 512-byte coalesced rows.
        float* tile = reinterpret_cast<float*>(smem);
        const uint32_t trow = 32 * warp + lane;
#pragma unroll 1
        for (uint32_t c0 = 0; c0 < kTile; c0 += 16) {
            float v[16];
            __syncwarp();
            tmem_ld16(tmem + ((32u * warp) << 16) + c0, v);
#pragma unroll
            for (int q = 0; q < 4; ++q) {
                const uint32_t chunk = (c0 >> 2) + q;
                *reinterpret_cast<float4*>(tile + trow * kTile + ((chunk ^ (trow & 7u)) << 2)) =
                    make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]);
            }
        }
        __syncthreads();
        const uint32_t col = n0 + 4 * lane;
#pragma unroll 1
        for (uint32_t r = warp; r < kTile; r += kThreads / 32) {
            const uint32_t grow = m0 + r;
            if (grow >= M || col >= N)
                continue;
            const float4 a = *reinterpret_cast<const float4*>(tile + r * kTile + ((lane ^ (r & 7u)) << 2));
            float* crow = C + (size_t)grow * ldc + col;
            if (col + 4 <= N) {
                float4 o = beta == 0.0f ? make_float4(0.f, 0.f, 0.f, 0.f) : *reinterpret_cast<const float4*>(crow);
                o.x = alpha * a.x + beta * o.x;
                o.y = alpha * a.y + beta * o.y;
                o.z = alpha * a.z + beta * o.z;
                o.w = alpha * a.w + beta * o.w;
                *reinterpret_cast<float4*>(crow) = o;
            } else {
                const float av[4] = {a.x, a.y, a.z, a.w};
                for (uint32_t i = 0; i < 4 && col + i < N; ++i)
                    crow[i] = alpha * av[i] + (beta == 0.0f ? 0.0f : beta * crow[i]);
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)kTile)
                     : "memory");
}

}  // namespace

extern "C" int pvl_gemm_tf32(uint32_t M, uint32_t N, uint32_t K, float alpha, const float* A, uint32_t lda,
                             const float* B, uint32_t ldb, float beta, float* C, uint32_t ldc, int32_t* err,
                             void* stream)
{
    if (M == 0 || N == 0)
        return PVL_OK;
    if (!A || !B || !C || !err)
        return pvl_fail(PVL_ERR_ARG, "pvl_gemm_tf32: null pointer argument");
    if (K % kKT)
        return pvl_fail(PVL_ERR_ARG, "pvl_gemm_tf32: K must be a multiple of %d (got %u)", kKT, K);
    if (lda % 4 || ldb % 4 || ldc % 4 || lda < K || ldb < N || ldc < N)
        return pvl_fail(PVL_ERR_ARG, "pvl_gemm_tf32: leading dimensions must be >= the row length and multiples of 4");
    if (((uintptr_t)A | (uintptr_t)B | (uintptr_t)C) & 15u)
        return pvl_fail(PVL_ERR_ARG, "pvl_gemm_tf32: A, B and C must be 16-byte aligned");
    const size_t smem = (size_t)kStages * kStageBytes + 1024;
    static bool attr = false;
    if (!attr) {
        PVL_CUDA_CHECK(cudaFuncSetAttribute(gemm_tf32_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr = true;
    }
    dim3 grid((N + kTile - 1) / kTile, (M + kTile - 1) / kTile);
    if (grid.y > 65535)
        return pvl_fail(PVL_ERR_ARG, "pvl_gemm_tf32: M too large");
    gemm_tf32_kernel<<<grid, kThreads, smem, (cudaStream_t)stream>>>(M, N, K, alpha, A, lda, B, ldb, beta, C, ldc,
                                                                     err);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}
