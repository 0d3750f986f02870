// Tensor-core GEMM on sm_100a: C = alpha * A * B + beta * C with FP32 storage, TF32 inputs
// and FP32 accumulation (tcgen05.mma kind::tf32, accumulators in tensor memory).
//
// Used by the low-precision preconditioner of the mixed solve: the trailing updates of the
// FP32 LU and the rank-64 updates of its triangular inversion.  Row-major A (M x K) and B given
// as its transpose Bt (N x K, row-major), so that both operands are K-major; row-major C
// (M x N).  Any M and N, K a multiple of 32, leading dimensions multiples of 4 floats, 16-byte
// aligned bases.
//
// Persistent, warp-specialised: one CTA per SM walks the 128 x 128 output tiles.
//   warp 0       TMA producer: each 32-wide K slice of A and Bt (16 KB each) is brought into a
//                four-stage ring of shared memory by cp.async.bulk.tensor (128-byte swizzle,
//                the canonical UMMA K-major layout), completion counted on the stage's
//                "full" mbarrier;
//   warp 1       allocates 256 TMEM columns (two 128 x 128 FP32 accumulators) and issues the
//                MMAs (four K = 8 steps per slice) from one thread, each slice's commit freeing
//                its stage, each tile's commit handing its accumulator to the epilogue;
//   warps 2..5   epilogue: each thread first requests its 32 four-float pieces of the tile's
//                C (kept in registers: one memory round trip per tile), then moves the
//                accumulator's rows through tcgen05.ld into a shared staging tile (the TMEM
//                buffer is released at once, so the next tile's MMAs run during the rest of
//                the epilogue) and writes C in 512-byte coalesced rows.
// Every wait is bounded.  A wait that runs out sets *err and stops the CTA's roles; before
// the CTA frees its tensor memory it waits (bounded) for its own copies and MMAs in flight.
// A TMA load never reads another GPU's memory here and none uses cluster multicast.
#include <cuda.h>

#include <cstdint>
#include <mutex>

#include "gemm_tc.cuh"
#include "pvl_common.cuh"
#include "umma.cuh"

namespace pvl {
namespace gemm_tc {

struct Smem {
    unsigned char stage[kStages][kStageBytes];  // 1024-byte aligned (the swizzle is anchored there)
    float out[kTile * kTile];                   // epilogue staging, 16-byte chunks XOR-swizzled by row
    uint64_t full[kStages], empty[kStages], acc_full[2], acc_empty[2], drain;
    uint32_t tmem;
    int fail;
};

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* tm, int x, int y, uint32_t bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            umma::smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(tm)), "r"(x), "r"(y), "r"(bar)
        : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void epi_sync() { asm volatile("bar.sync 1, 128;" ::: "memory"); }

// Barrier of the 128 epilogue threads that also returns the OR of `v` over them, so that they
// leave their loop together.
__device__ __forceinline__ bool epi_sync_or(bool v)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.or.pred q, 1, 128, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)v)
        : "memory");
    return r != 0;
}

__device__ __forceinline__ void set_fail(Smem& s, int32_t* err)
{
    if (atomicExch(&s.fail, 1) == 0)
        atomicExch(err, 1);
}

__device__ __forceinline__ bool failed(const Smem& s) { return *((volatile const int*)&s.fail) != 0; }

// skip_loads (tests only): the producer issues no copies, so every wait on a stage runs out.
__global__ void __launch_bounds__(kThreads, 1) gemm_tf32_kernel(const __grid_constant__ CUtensorMap tma,
                                                                const __grid_constant__ CUtensorMap tmb, uint32_t M,
                                                                uint32_t N, uint32_t K, float alpha, float beta,
                                                                float* __restrict__ C, uint32_t ldc,
                                                                int32_t* __restrict__ err, long long wait_limit,
                                                                int skip_loads)
{
    extern __shared__ __align__(1024) unsigned char gemm_raw[];
    Smem& s = *reinterpret_cast<Smem*>(gemm_raw + ((1024u - (umma::smem_u32(gemm_raw) & 1023u)) & 1023u));
    const uint32_t tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const uint32_t tiles_n = (N + kTile - 1) / kTile, n_tiles = tiles_n * ((M + kTile - 1) / kTile);
    const uint32_t n_kt = K / kKT;
    if (tid == 0) {
        for (int i = 0; i < kStages; ++i) {
            umma::mbar_init(umma::smem_u32(&s.full[i]), 1);
            umma::mbar_init(umma::smem_u32(&s.empty[i]), 1);
        }
        for (int i = 0; i < 2; ++i) {
            umma::mbar_init(umma::smem_u32(&s.acc_full[i]), 1);
            umma::mbar_init(umma::smem_u32(&s.acc_empty[i]), 1);
        }
        umma::mbar_init(umma::smem_u32(&s.drain), 1);
        s.fail = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1)
        umma::tmem_alloc(&s.tmem, 2 * kTile);
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    const uint32_t tmem = s.tmem;

    if (warp == 0) {
        // ------------------------------------------------------------ TMA producer
        if (lane == 0) {
            uint32_t it = 0;
            int pending[kStages] = {0, 0, 0, 0};  // a fill in flight that this thread has not seen land
            for (uint32_t t = blockIdx.x; t < n_tiles && !failed(s); t += gridDim.x) {
                const int m0 = (int)((t / tiles_n) * kTile), n0 = (int)((t % tiles_n) * kTile);
                for (uint32_t kt = 0; kt < n_kt; ++kt, ++it) {
                    const uint32_t st = it % kStages, use = it / kStages;
                    if (use > 0) {
                        if (!umma::mbar_wait(umma::smem_u32(&s.empty[st]), (use - 1) & 1u, wait_limit)) {
                            set_fail(s, err);
                            break;
                        }
                        pending[st] = 0;  // its consumer has released it, so the fill landed
                    }
                    if (failed(s))
                        break;
                    if (skip_loads)
                        continue;
                    const uint32_t bar = umma::smem_u32(&s.full[st]);
                    umma::mbar_arrive_expect_tx(bar, kStageBytes);
                    tma_load_2d(s.stage[st], &tma, (int)(kt * kKT), m0, bar);
                    tma_load_2d(s.stage[st] + kHalfBytes, &tmb, (int)(kt * kKT), n0, bar);
                    pending[st] = 1 + (int)(use & 1u);  // remembers the parity of the fill
                }
            }
            // copies still in flight land before the CTA may exit (bounded)
            for (int st = 0; st < kStages; ++st)
                if (pending[st] && !umma::mbar_wait(umma::smem_u32(&s.full[st]), (uint32_t)(pending[st] - 1), wait_limit))
                    set_fail(s, err);
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0) {
            constexpr uint32_t kId = umma::idesc_tf32(kTile, kTile);
            uint32_t it = 0, ti = 0;
            bool issued = false;
            for (uint32_t t = blockIdx.x; t < n_tiles && !failed(s); t += gridDim.x, ++ti) {
                const uint32_t a = ti & 1u, use_a = ti >> 1;
                if (use_a > 0 && !umma::mbar_wait(umma::smem_u32(&s.acc_empty[a]), (use_a - 1) & 1u, wait_limit)) {
                    set_fail(s, err);
                    break;
                }
                umma::fence_after_sync();
                bool ok = true;
                for (uint32_t kt = 0; kt < n_kt; ++kt, ++it) {
                    const uint32_t st = it % kStages;
                    if (!umma::mbar_wait(umma::smem_u32(&s.full[st]), (it / kStages) & 1u, wait_limit)) {
                        set_fail(s, err);
                        ok = false;
                        break;
                    }
                    umma::fence_after_sync();
                    const uint64_t da = umma::sw128_desc(umma::smem_u32(s.stage[st]));
                    const uint64_t db = umma::sw128_desc(umma::smem_u32(s.stage[st] + kHalfBytes));
#pragma unroll
                    for (uint32_t ks = 0; ks < kKT / 8; ++ks)  // K = 8 TF32 (32 bytes) per MMA
                        umma::mma<true>(tmem + a * kTile, da + 2u * ks, db + 2u * ks, kId, (kt | ks) ? 1u : 0u);
                    issued = true;
                    umma::commit(umma::smem_u32(&s.empty[st]));
                }
                if (!ok)
                    break;
                umma::commit(umma::smem_u32(&s.acc_full[a]));
            }
            if (issued) {  // every MMA of this CTA completes before its tensor memory is freed (bounded)
                umma::commit(umma::smem_u32(&s.drain));
                if (!umma::mbar_wait(umma::smem_u32(&s.drain), 0u, wait_limit))
                    set_fail(s, err);
            }
        }
    } else {
        // ------------------------------------------------------------ epilogue (128 threads)
        const uint32_t q = warp & 3u;            // TMEM lane quarter this warp may read
        const uint32_t row = 32u * q + lane;     // accumulator row of this thread
        const uint32_t ew = warp - 2;            // 0..3: rows ew, ew + 4, ... in the coalesced phase
        uint32_t ti = 0;
        for (uint32_t t = blockIdx.x; t < n_tiles; t += gridDim.x, ++ti) {
            const uint32_t a = ti & 1u;
            const uint32_t m0 = (t / tiles_n) * kTile, n0 = (t % tiles_n) * kTile;
            const uint32_t col = n0 + 4 * lane;
            // this thread's 32 four-float pieces of C (rows ew, ew + 4, ...), all requested
            // before the accumulator is awaited, so that one memory round trip per tile (not
            // one per row) overlaps the tile's MMAs
            float4 cin[kTile / 4];
            const bool full_cols = col + 4 <= N;
#pragma unroll
            for (int i = 0; i < kTile / 4; ++i) {
                const uint32_t grow = m0 + ew + 4u * i;
                cin[i] = make_float4(0.f, 0.f, 0.f, 0.f);
                if (beta != 0.0f && full_cols && grow < M)
                    cin[i] = *reinterpret_cast<const float4*>(C + (size_t)grow * ldc + col);
            }
            const bool ok = umma::mbar_wait(umma::smem_u32(&s.acc_full[a]), (ti >> 1) & 1u, wait_limit);
            if (!ok)
                set_fail(s, err);
            if (epi_sync_or(!ok || failed(s)))
                break;
            umma::fence_after_sync();
#pragma unroll 1
            for (uint32_t c0 = 0; c0 < kTile; c0 += 16) {
                float v[16];
                __syncwarp();
                umma::tmem_ld16(tmem + a * kTile + ((32u * q) << 16) + c0, v);
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const uint32_t chunk = (c0 >> 2) + c;
                    *reinterpret_cast<float4*>(s.out + row * kTile + ((chunk ^ (row & 7u)) << 2)) =
                        make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
                }
            }
            umma::fence_before_sync();
            epi_sync();
            if (ew == 0 && lane == 0)
                mbar_arrive(umma::smem_u32(&s.acc_empty[a]));  // the accumulator may take the next tile
#pragma unroll
            for (int i = 0; i < kTile / 4; ++i) {
                const uint32_t r = ew + 4u * i, grow = m0 + r;
                if (grow >= M || col >= N)
                    continue;
                const float4 v = *reinterpret_cast<const float4*>(s.out + r * kTile + ((lane ^ (r & 7u)) << 2));
                float* crow = C + (size_t)grow * ldc + col;
                if (full_cols) {
                    float4 o = cin[i];
                    o.x = alpha * v.x + beta * o.x;
                    o.y = alpha * v.y + beta * o.y;
                    o.z = alpha * v.z + beta * o.z;
                    o.w = alpha * v.w + beta * o.w;
                    *reinterpret_cast<float4*>(crow) = o;
                } else {
                    const float av[4] = {v.x, v.y, v.z, v.w};
                    for (uint32_t e = 0; e < 4 && col + e < N; ++e)
                        crow[e] = alpha * av[e] + (beta == 0.0f ? 0.0f : beta * crow[e]);
                }
            }
            epi_sync();  // the staging tile is free for the next tile
        }
    }
    umma::fence_before_sync();
    __syncthreads();
    umma::fence_after_sync();
    if (warp == 1)
        umma::tmem_dealloc(tmem, 2 * kTile);
}

}  // namespace gemm_tc
}  // namespace pvl

namespace {

using namespace pvl::gemm_tc;

using EncodeTiled = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                 const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiled encode_fn()
{
    static EncodeTiled fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<EncodeTiled>(p);
    }();
    return fn;
}

}  // namespace

// Tensor map of a row-major FP32 matrix (rows x k, leading dimension ld floats) in 32 x 128
// boxes (32 floats of K = 128 bytes, the swizzle span; 128 rows), 128-byte swizzle, rows past
// the end read as zero.
int pvl_tf32_tensor_map(CUtensorMap* tm, const float* base, uint32_t rows, uint32_t k, uint32_t ld)
{
    EncodeTiled enc = encode_fn();
    if (!enc)
        return pvl_fail(PVL_ERR_CUDA, "cuTensorMapEncodeTiled is not available");
    const cuuint64_t dims[2] = {k, rows};
    const cuuint64_t strides[1] = {(cuuint64_t)ld * sizeof(float)};
    const cuuint32_t box[2] = {kKT, kTile};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = enc(tm, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS)
        return pvl_fail(PVL_ERR_CUDA, "cuTensorMapEncodeTiled failed (%d)", (int)r);
    return PVL_OK;
}

int pvl_gemm_tf32_launch(uint32_t M, uint32_t N, uint32_t K, float alpha, const float* A, uint32_t lda, const float* Bt,
                         uint32_t ldbt, float beta, float* C, uint32_t ldc, int32_t* err, long long wait_limit,
                         int skip_loads, uint32_t max_ctas, cudaStream_t st)
{
    CUtensorMap ta, tb;
    if (int r = pvl_tf32_tensor_map(&ta, A, M, K, lda))
        return r;
    if (int r = pvl_tf32_tensor_map(&tb, Bt, N, K, ldbt))
        return r;
    const size_t smem = sizeof(pvl::gemm_tc::Smem) + 1024;
    PVL_SMEM_OPTIN(pvl::gemm_tc::gemm_tf32_kernel, smem);
    int dev = 0, sms = 0;
    PVL_CUDA_CHECK(cudaGetDevice(&dev));
    PVL_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const uint32_t tiles = ((M + kTile - 1) / kTile) * ((N + kTile - 1) / kTile);
    uint32_t grid = tiles < (uint32_t)sms ? tiles : (uint32_t)sms;
    if (max_ctas && grid > max_ctas)
        grid = max_ctas;
    pvl::gemm_tc::gemm_tf32_kernel<<<grid, kThreads, smem, st>>>(ta, tb, M, N, K, alpha, beta, C, ldc, err,
                                                                 wait_limit, skip_loads);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_gemm_tf32(uint32_t M, uint32_t N, uint32_t K, float alpha, const float* A, uint32_t lda,
                             const float* Bt, uint32_t ldbt, float beta, float* C, uint32_t ldc, int32_t* err,
                             void* stream)
{
    if (M == 0 || N == 0)
        return PVL_OK;
    if (!A || !Bt || !C || !err)
        return pvl_fail(PVL_ERR_ARG, "pvl_gemm_tf32: null pointer argument");
    if (K == 0 || K % kKT)
        return pvl_fail(PVL_ERR_ARG, "pvl_gemm_tf32: K must be a positive multiple of %d (got %u)", kKT, K);
    if (lda % 4 || ldbt % 4 || ldc % 4 || lda < K || ldbt < K || ldc < N)
        return pvl_fail(PVL_ERR_ARG, "pvl_gemm_tf32: leading dimensions must be >= the row length and multiples of 4");
    if (((uintptr_t)A | (uintptr_t)Bt | (uintptr_t)C) & 15u)
        return pvl_fail(PVL_ERR_ARG, "pvl_gemm_tf32: A, Bt and C must be 16-byte aligned");
    return pvl_gemm_tf32_launch(M, N, K, alpha, A, lda, Bt, ldbt, beta, C, ldc, err, pvl::umma::kWaitLimit, 0, 0,
                                (cudaStream_t)stream);
}
