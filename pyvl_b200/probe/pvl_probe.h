/* Measurement and test probes of pyvl_b200 (libpvl_probe.so).  Not part of the product's
 * C ABI (include/pvl_b200.h): benchmarks and tests load this library beside it.  Status codes
 * as in pvl_b200.h; pvl_probe_last_error() gives the calling thread's last message. */
#ifndef PVL_PROBE_H
#define PVL_PROBE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

const char* pvl_probe_last_error(void);

/* Enqueue a kernel of n_blocks x 256 threads, each running 8 independent FMA chains of `iters`
 * steps in `precision` (PVL_F64 / PVL_F32); returns the exact FLOP count (2 per FMA), or a
 * negative value on error.  `sink`: a device buffer of n_blocks elements (never written in
 * practice).  Timed with events it gives the GPU's non-tensor FMA peak. */
double pvl_probe_fma(int precision, uint32_t n_blocks, uint32_t iters, void* sink, void* stream);

/* rcp[i] = the FP64 pair kernels' 1/x[i] (hardware seed and one third-order refinement) and
 * sum[i] = their arctangent series sum_k (-w)^k / (2k + 1) at w[i] (w in [0, 0.1]), for n
 * device values. */
int pvl_probe_far_series(uint32_t n, const double* x, const double* w, double* rcp, double* sum, void* stream);

/* One pass of the wavefront triangular solve of pvl_lu_solve (lower: unit-lower forward,
 * else backward) on factors LU (lda) with the inverted diagonal blocks `inv`, x in place, with
 * a spin limit of `spin_limit` polls per wait and block `skip_block` (or -1) returning without
 * publishing its flag.  flags: n / 64 + 1 int32 (zeroed here); *err is zeroed here and set to
 * 1 by every block whose wait ran out. */
int pvl_probe_trsv_timeout(uint32_t n, const double* LU, uint32_t lda, const double* inv, double* x, int32_t* flags,
                           int32_t* err, long long spin_limit, int32_t skip_block, int lower, void* stream);

/* The TF32 GEMM of pvl_gemm_tf32 (C = A Bt^T) with a wait limit of `wait_limit` polls and a
 * producer that issues no copies, on one CTA: every wait runs out and *err is set to 1 (zeroed
 * here first); C is not written. */
int pvl_probe_gemm_timeout(uint32_t M, uint32_t N, uint32_t K, const float* A, uint32_t lda, const float* Bt,
                           uint32_t ldbt, float* C, uint32_t ldc, int32_t* err, long long wait_limit, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PVL_PROBE_H */
