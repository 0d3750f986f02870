// Shapes of the persistent TMA-fed TF32 GEMM of gemm_tc.cu and its internal launcher (reached
// by the test probes, which run the kernel with a short wait limit and no loads).
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>


namespace pvl {
namespace gemm_tc {

constexpr int kTile = 128;                         // M and N of an output tile (one UMMA 128 x 128)
constexpr int kKT = 32;                            // K per stage: 32 TF32 = 128 bytes, the swizzle span
constexpr int kStages = 4;
constexpr int kThreads = 192;                      // warp 0 TMA, warp 1 MMA, warps 2..5 epilogue
constexpr uint32_t kHalfBytes = kTile * kKT * 4;   // one operand slice (16 KB)
constexpr uint32_t kStageBytes = 2 * kHalfBytes;   // A and Bt slices

}  // namespace gemm_tc
}  // namespace pvl

// Launcher of the kernel above (gemm_tc.cu); wait_limit in polls, skip_loads for tests,
// max_ctas = 0 for one CTA per SM (at most one per tile).
int pvl_gemm_tf32_launch(uint32_t M, uint32_t N, uint32_t K, float alpha, const float* A, uint32_t lda, const float* Bt,
                         uint32_t ldbt, float beta, float* C, uint32_t ldc, int32_t* err, long long wait_limit,
                         int skip_loads, uint32_t max_ctas, cudaStream_t st);
