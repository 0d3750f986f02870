// Dense FP64 LU with partial pivoting (GEPP) and the matching solve, for the row-major
// system matrix the induction kernels write.  Replaces the reference's
// scipy.linalg.lu_factor / lu_solve (python/pyvl/solver.py:223-227).
//
// Right-looking blocked factorisation, panel width NB = 64.  Per panel (k0, nb):
//   1. panel_spec_kernel -- speculative factorisation of the whole panel with the diagonal as
//      pivot.  Every CTA factors the same nb x nb top block (one row per thread, rows held in
//      registers) together with its own 64 rows below it, so no CTA waits for another.  Per
//      column it records the largest |entry| below the diagonal at the moment the column is
//      eliminated.
//   2. panel_pivot_kernel -- one CTA: if every diagonal entry is non-zero and no entry below
//      it is larger, partial pivoting would have chosen exactly these pivots (LAPACK's idamax
//      returns the first maximal entry and the diagonal comes first), so the speculative
//      factors ARE the GEPP factors: commit them with identity pivots.  Otherwise restore the
//      panel from the backup and factor it with explicit partial pivoting in getf2 order.
//   3. trsm_kernel -- applies the panel's interchanges to the other columns and forms
//      U12 = L11^-1 A12 (one column per thread, held in registers).
//   4. gemm_update_kernel -- A22 -= L21 U12, FP64, 128 x 128 tiles, 8 x 8 outputs per thread,
//      128-bit conflict-free shared loads.
// Diagonally dominant systems (the vortex-ring matrices are close to -2 pi I) take the
// speculative path on every panel; a bordered closed-body system falls back on the panel
// holding the zero-diagonal border.
//
// The solve runs two wavefront kernels (forward with unit-lower L, backward with U) over
// row blocks, one CTA per block, co-resident through a cooperative launch; each CTA stages
// its diagonal block in shared memory before waiting, and every wait on an earlier block is
// bounded and reports a time-out through a device error word.
#include <algorithm>
#include <cstdint>

#include "pvl_common.cuh"
#include "dmma.cuh"
#include "trsv.cuh"

namespace {

constexpr int NB = 64;               // panel width
constexpr int kSlabRows = 64;        // rows below the top block per CTA in panel_spec_kernel
constexpr int kRB = 64;              // rows per block in the wavefront solves
static_assert(kRB == pvl::trsv::kRB, "the solve's row blocks are the inverted diagonal blocks");
static_assert(NB == pvl::dmma::K, "the tensor-core products have K = the panel width");
constexpr int kSolveThreads = pvl::trsv::kThreads;

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }
inline unsigned blocks_for(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

struct LuWs {
    double* backup;         // (n, NB) copy of the current panel before speculation
    double* top_out;        // (NB, NB) speculative top block
    int32_t* reject;        // per panel: the speculation failed
    int32_t* ok;            // per panel: speculative factors accepted
    int32_t* flags;         // wavefront flags (solve)
    double* tmp;            // (n) solve vector
    double* inv;            // (n_blocks, 2, kRB, kRB): inverses of the diagonal blocks of L and U
    double* backup_row;     // (NB, n) copy of the panel's row block right of it (FP64 path)
    double* linv;           // (NB, NB) inverse of the panel's unit-lower L11 (FP64 path)
    double* uinv;           // (NB, NB) inverse of the panel's U11 (FP64 path)
};

size_t lu_ws_bytes(uint32_t n)
{
    return align256((size_t)n * NB * sizeof(double)) + align256((size_t)NB * NB * sizeof(double)) +
           align256(((size_t)n / NB + 2) * sizeof(int32_t)) +
           align256(((size_t)n / NB + 2) * sizeof(int32_t)) + align256(((size_t)n / kRB + 2) * sizeof(int32_t)) +
           align256((size_t)n * sizeof(double)) + align256(((size_t)n + kRB - 1) / kRB * 2 * kRB * kRB * sizeof(double)) +
           align256((size_t)NB * n * sizeof(double)) + 2 * align256((size_t)NB * NB * sizeof(double));
}

LuWs carve(void* ws, uint32_t n)
{
    char* p = static_cast<char*>(ws);
    LuWs w;
    w.backup = reinterpret_cast<double*>(p);
    p += align256((size_t)n * NB * sizeof(double));
    w.top_out = reinterpret_cast<double*>(p);
    p += align256((size_t)NB * NB * sizeof(double));
    w.reject = reinterpret_cast<int32_t*>(p);
    p += align256(((size_t)n / NB + 2) * sizeof(int32_t));
    w.ok = reinterpret_cast<int32_t*>(p);
    p += align256(((size_t)n / NB + 2) * sizeof(int32_t));
    w.flags = reinterpret_cast<int32_t*>(p);
    p += align256(((size_t)n / kRB + 2) * sizeof(int32_t));
    w.tmp = reinterpret_cast<double*>(p);
    p += align256((size_t)n * sizeof(double));
    w.inv = reinterpret_cast<double*>(p);
    p += align256(((size_t)n + kRB - 1) / kRB * 2 * kRB * kRB * sizeof(double));
    w.backup_row = reinterpret_cast<double*>(p);
    p += align256((size_t)NB * n * sizeof(double));
    w.linv = reinterpret_cast<double*>(p);
    p += align256((size_t)NB * NB * sizeof(double));
    w.uinv = reinterpret_cast<double*>(p);
    return w;
}

__global__ void init_perm_kernel(uint32_t n, int32_t* __restrict__ perm)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        perm[i] = (int32_t)i;
}

// ---------------------------------------------------------------- 1+2. speculative panel
// grid.x = max(1, ceil(below / kSlabRows)); 128 threads: threads 0..63 hold the 64 rows of
// the top block (every CTA factors the same top block, so no CTA waits for another), threads
// 64..127 hold this CTA's rows below it.  Each thread keeps its row in registers (columns
// beyond nb are zero; missing top rows are unit rows) and eliminates column j with the row
// that thread j publishes in shared memory, scaling by the reciprocal of the pivot as getf2
// does -- the recurrence of getf2 without interchanges.  Partial pivoting would keep the
// diagonal in column j iff no entry below it is larger in magnitude at that moment; every
// thread checks this for its own row, and any violation (or a zero/NaN pivot) marks the panel.
// Slab rows are backed up and overwritten in place; the factored top block goes to `top_out`
// (committed by panel_pivot_kernel) so that no CTA can read a half-written top block.
template <typename T>
__global__ void __launch_bounds__(2 * kSlabRows) panel_spec_kernel(uint32_t n, uint32_t k0, uint32_t nb,
                                                                   T* __restrict__ A, uint32_t lda,
                                                                   T* __restrict__ backup,
                                                                   T* __restrict__ top_out,
                                                                   int32_t* __restrict__ reject)
{
    __shared__ T U[NB][NB + 1];
    __shared__ T s_rcp[NB];
    const uint32_t tid = threadIdx.x;
    const bool is_top = tid < NB;
    const uint32_t r_begin = k0 + nb + blockIdx.x * kSlabRows;
    // global row of this thread (top: k0 + tid, slab: r_begin + tid - 64)
    const uint32_t grow = is_top ? k0 + tid : r_begin + (tid - NB);
    const bool valid = is_top ? tid < nb : grow < n;
    T row[NB];
#pragma unroll
    for (int c = 0; c < NB; ++c) {
        T v = T(0);
        if (valid && (uint32_t)c < nb)
            v = A[(size_t)grow * lda + k0 + c];
        else if (is_top && !valid && (uint32_t)c == tid)
            v = T(1);  // unit row standing in for a missing top row
        row[c] = v;
    }
    if (!is_top && valid)
#pragma unroll
        for (int c = 0; c < NB; ++c)
            if ((uint32_t)c < nb)
                backup[(size_t)(grow - k0) * NB + c] = row[c];
    bool bad = false;
#pragma unroll
    for (int j = 0; j < NB; ++j) {
        if (tid == (uint32_t)j) {
#pragma unroll
            for (int c = j; c < NB; ++c)
                U[j][c] = row[c];
            s_rcp[j] = T(1) / row[j];
            bad |= !(fabs(row[j]) > T(0));
        }
        __syncthreads();
        const bool act = is_top ? tid > (uint32_t)j : valid;
        if (act) {
            const T v = row[j];
            bad |= !(fabs(v) <= fabs(U[j][j]));
            const T x = v * s_rcp[j];
            row[j] = x;
#pragma unroll
            for (int c = j + 1; c < NB; ++c)
                row[c] -= x * U[j][c];
        }
    }
    if (__syncthreads_or(bad) && tid == 0)
        atomicExch(reject, 1);
    if (is_top) {
        if (blockIdx.x == 0 && valid)
#pragma unroll
            for (int c = 0; c < NB; ++c)
                if ((uint32_t)c < nb)
                    top_out[(size_t)tid * NB + c] = row[c];
    } else if (valid) {
#pragma unroll
        for (int c = 0; c < NB; ++c)
            if ((uint32_t)c < nb)
                A[(size_t)grow * lda + k0 + c] = row[c];
    }
}

// ---------------------------------------------------------------- 3. accept or pivot
template <typename T>
__global__ void __launch_bounds__(1024) panel_pivot_kernel(uint32_t n, uint32_t k0, uint32_t nb, T* __restrict__ A,
                                                           uint32_t lda, const T* __restrict__ backup,
                                                           const T* __restrict__ top_out,
                                                           const int32_t* __restrict__ reject,
                                                           int32_t* __restrict__ ok, uint32_t panel,
                                                           int32_t* __restrict__ ipiv, int32_t* __restrict__ perm,
                                                           int32_t* __restrict__ info,
                                                           const T* __restrict__ backup_row)
{
    __shared__ T s_val[32];
    __shared__ uint32_t s_idx[32];
    __shared__ uint32_t s_piv;
    __shared__ T s_prow[NB];
    const int bad = reject[panel];
    if (!bad) {
        if (threadIdx.x == 0)
            ok[panel] = 1;
        for (uint32_t t = threadIdx.x; t < nb * nb; t += blockDim.x) {
            const uint32_t r = t / nb, c = t % nb;
            A[(size_t)(k0 + r) * lda + k0 + c] = top_out[(size_t)r * NB + c];
        }
        for (uint32_t j = threadIdx.x; j < nb; j += blockDim.x)
            ipiv[k0 + j] = (int32_t)(k0 + j);
        return;
    }
    if (threadIdx.x == 0)
        ok[panel] = 0;
    // the top block of A was never written; restore the rows below it, then LAPACK getf2:
    // first row of maximal |a|, swap, scale, update
    for (size_t t = threadIdx.x; t < (size_t)(n - k0 - nb) * nb; t += blockDim.x) {
        const uint32_t r = (uint32_t)(t / nb) + nb, c = (uint32_t)(t % nb);
        A[(size_t)(k0 + r) * lda + k0 + c] = backup[(size_t)r * NB + c];
    }
    if (backup_row)  // the FP64 path also replaced the row block right of the panel by U12
        for (size_t t = threadIdx.x; t < (size_t)nb * (n - k0 - nb); t += blockDim.x) {
            const uint32_t r = (uint32_t)(t / (n - k0 - nb)), c = k0 + nb + (uint32_t)(t % (n - k0 - nb));
            A[(size_t)(k0 + r) * lda + c] = backup_row[(size_t)r * n + c];
        }
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t j = 0; j < nb; ++j) {
        const uint32_t col = k0 + j;
        T best = T(-1);
        uint32_t bidx = 0xFFFFFFFFu;
        for (uint32_t r = col + threadIdx.x; r < n; r += blockDim.x) {
            const T v = fabs(A[(size_t)r * lda + col]);
            if (v > best) {
                best = v;
                bidx = r;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const T ov = __shfl_xor_sync(0xffffffffu, best, o);
            const uint32_t oi = __shfl_xor_sync(0xffffffffu, bidx, o);
            if (ov > best || (ov == best && oi < bidx)) {
                best = ov;
                bidx = oi;
            }
        }
        if (lane == 0) {
            s_val[warp] = best;
            s_idx[warp] = bidx;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            T b = T(-1);
            uint32_t bi = col;
            for (uint32_t w = 0; w < blockDim.x / 32; ++w)
                if (s_val[w] > b || (s_val[w] == b && s_idx[w] < bi)) {
                    b = s_val[w];
                    bi = s_idx[w];
                }
            s_piv = bi;
            ipiv[col] = (int32_t)bi;
            if (bi != col) {
                const int32_t t = perm[col];
                perm[col] = perm[bi];
                perm[bi] = t;
            }
        }
        __syncthreads();
        const uint32_t p = s_piv;
        if (p != col)
            for (uint32_t c = threadIdx.x; c < nb; c += blockDim.x) {
                const T a = A[(size_t)col * lda + k0 + c];
                A[(size_t)col * lda + k0 + c] = A[(size_t)p * lda + k0 + c];
                A[(size_t)p * lda + k0 + c] = a;
            }
        __syncthreads();
        for (uint32_t c = threadIdx.x; c < nb; c += blockDim.x)
            s_prow[c] = A[(size_t)col * lda + k0 + c];
        __syncthreads();
        const T piv = s_prow[j];
        if (piv == T(0)) {
            if (threadIdx.x == 0)
                atomicCAS(info, 0, (int32_t)(col + 1));
            __syncthreads();
            continue;
        }
        const T rcp = T(1) / piv;
        for (uint32_t r = col + 1 + threadIdx.x; r < n; r += blockDim.x) {
            T* row = A + (size_t)r * lda + k0;
            const T l = row[j] * rcp;
            row[j] = l;
            for (uint32_t c = j + 1; c < nb; ++c)
                row[c] -= l * s_prow[c];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------- 3. swaps + U12
// One thread per column outside the panel: apply the panel's interchanges (if any); columns
// right of the panel then solve L11 x = a (unit lower).  The 64 x 128 column block is staged
// through shared memory with coalesced row accesses; each thread keeps its column in
// registers during the substitution.
constexpr int kTrsmCols = 128;

template <typename T>
__global__ void __launch_bounds__(kTrsmCols, 1) trsm_kernel(uint32_t n, uint32_t k0, uint32_t nb,
                                                            T* __restrict__ A, uint32_t lda,
                                                            const int32_t* __restrict__ ok, uint32_t panel,
                                                            const int32_t* __restrict__ ipiv, int fast_u12)
{
    if (fast_u12 && ok[panel])
        return;  // the FP64 path formed U12 = L11^-1 A12 already and nothing was interchanged
    extern __shared__ double tsm_raw[];
    T* tsm = reinterpret_cast<T*>(tsm_raw);
    T(*L)[NB + 1] = reinterpret_cast<T(*)[NB + 1]>(tsm);                        // [NB][NB + 1]
    T(*X)[kTrsmCols + 1] = reinterpret_cast<T(*)[kTrsmCols + 1]>(tsm + NB * (NB + 1));  // [NB][129]
    const bool swapped = !ok[panel];
    const uint32_t t = blockIdx.x * kTrsmCols + threadIdx.x;
    const uint32_t n_out = n - nb;
    const uint32_t col = t < k0 ? t : t + nb;
    if (t < n_out && swapped)
        for (uint32_t j = 0; j < nb; ++j) {
            const uint32_t r1 = k0 + j, r2 = (uint32_t)ipiv[k0 + j];
            if (r1 != r2) {
                const T a = A[(size_t)r1 * lda + col];
                A[(size_t)r1 * lda + col] = A[(size_t)r2 * lda + col];
                A[(size_t)r2 * lda + col] = a;
            }
        }
    // the columns right of the panel start at k0 + nb; this CTA's first such column:
    const uint32_t c_first = blockIdx.x * kTrsmCols;  // in t-space
    if (c_first + kTrsmCols <= k0 || c_first >= n_out)
        return;  // CTA-uniform: only left-of-panel columns (already swapped) or none
    __syncthreads();  // swaps of this CTA's columns are visible before staging
    for (uint32_t e = threadIdx.x; e < NB * NB; e += kTrsmCols) {
        const uint32_t r = e / NB, c = e % NB;
        L[r][c] = (r < nb && c < nb) ? A[(size_t)(k0 + r) * lda + k0 + c] : T(0);
    }
    for (uint32_t e = threadIdx.x; e < NB * kTrsmCols; e += kTrsmCols) {
        const uint32_t r = e / kTrsmCols, c = e % kTrsmCols;
        const uint32_t tt = c_first + c;
        const uint32_t cc = tt < k0 ? tt : tt + nb;
        X[r][c] = (r < nb && tt < n_out && cc >= k0 + nb) ? A[(size_t)(k0 + r) * lda + cc] : T(0);
    }
    __syncthreads();
    T x[NB];
#pragma unroll
    for (int r = 0; r < NB; ++r)
        x[r] = X[r][threadIdx.x];
#pragma unroll
    for (int q = 0; q < NB - 1; ++q) {
        const T xq = x[q];
#pragma unroll
        for (int r = q + 1; r < NB; ++r)
            x[r] -= L[r][q] * xq;
    }
#pragma unroll
    for (int r = 0; r < NB; ++r)
        X[r][threadIdx.x] = x[r];
    __syncthreads();
    for (uint32_t e = threadIdx.x; e < NB * kTrsmCols; e += kTrsmCols) {
        const uint32_t r = e / kTrsmCols, c = e % kTrsmCols;
        const uint32_t tt = c_first + c;
        const uint32_t cc = tt < k0 ? tt : tt + nb;
        if (r >= 1 && r < nb && tt < n_out && cc >= k0 + nb)
            A[(size_t)(k0 + r) * lda + cc] = X[r][c];
    }
}

// ---------------------------------------------------------------- FP64 panel on the tensor cores
// The FP64 factorisation first factors each panel without interchanges and then checks that
// partial pivoting would have made none: with no interchange before column j, GEPP keeps the
// diagonal in column j exactly when no entry below it is larger in magnitude at that moment,
// i.e. when every multiplier l_ij (i > j) has |l_ij| <= 1 (LAPACK's idamax returns the first
// maximal entry, and the diagonal comes first).  The multipliers are formed by blocks:
//   top_factor_kernel   L11 U11 = A11 (one CTA, the 64 x 64 diagonal block, in registers),
//                       the check inside the block, and L11^-1, U11^-1;
//   panel_apply_kernel  L21 = A21 U11^-1 (with the check on every multiplier) and
//                       U12 = L11^-1 A12, both as FP64 tensor-core tiles (dmma.cuh), the
//                       overwritten operands backed up;
//   panel_pivot_kernel  commits the top block -- or, if any check failed, restores the panel and
//                       its row block and refactors the panel with explicit partial pivoting in
//                       getf2 order, after which trsm_kernel applies the interchanges and forms
//                       U12 by substitution;
//   dmma_update_kernel  A22 -= L21 U12 on the FP64 tensor cores: 64 x 64 tiles, each CTA a
//                       run of them with the next tile's operands loading during the MMAs.
// Every product has K = 64, the panel width; the multipliers and U12 are the blocked forms of
// getf2's and trsm's, equal to them up to rounding.
// Columns per thread of the top-block kernel: 16 (256 threads), 8 (512) or 4 (1024); more
// threads shorten each column step's chain of dependent instructions per warp.
#ifndef PVL_TOP_CPT
#define PVL_TOP_CPT 16
#endif
constexpr int kTopCpt = PVL_TOP_CPT;
constexpr int kTopGroups = NB / kTopCpt;          // threads per row (neighbouring lanes)
constexpr int kTopThreads = NB * kTopGroups;
constexpr int kTopGs = kTopCpt + 2;               // doubles per column group of a broadcast row:
                                                  // the groups' 16-byte loads fall in distinct banks
static_assert(kTopCpt == 16 || kTopCpt == 8 || kTopCpt == 4, "16, 8 or 4 columns per thread");

constexpr double kPivotLo = 0x1p-1000, kPivotHi = 0x1p+1000;

// 1/p for a pivot with kPivotLo <= |p| <= kPivotHi: the hardware's approximate reciprocal r
// (rcp.approx.ftz.f64, relative error d < 2^-19) refined by one third-order step of the
// geometric series 1/p = r / (1 - e), e = 1 - p r:  r + r (e + e^2) = (1/p)(1 - d^3), within an
// ulp of the rounded quotient.  Pivots outside the range take the exact (pivoting) path.
__device__ __forceinline__ double pivot_rcp(double p)
{
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(p));
    const double e = fma(-p, r, 1.0);
    return fma(r, fma(e, e, e), r);
}

// One CTA: the 64 x 64 diagonal block (a partial block padded with identity) factored without
// interchanges, with X = L11^-1 and Y = U11^-1 formed in the same 64 column steps.  Thread
// (r, g) holds row r, columns C g .. C g + C - 1 (C = kTopCpt), of T, X and Y in registers (the
// threads of a row are neighbouring lanes); the column loop is unrolled by C, so every register
// index is a constant.  Step j: row j is final and sits in shared memory (published by its
// threads at the end of step j - 1, double-buffered by parity, one barrier per step).  A row
// r > j takes its multiplier l = T[r][j] / U[j][j] (by the pivot's reciprocal, as getf2) from
// the thread that holds column j, checks it, and applies T[r][c] -= l U[j][c] (c > j) and
// X[r] -= l X[j].  A row r <= j finishes Y[r][j] = (delta_rj - sum_{k<j} Y[r][k] U[k][j]) /
// U[j][j] (the sum has been accumulated in y by the earlier steps) and applies
// Y[r][c] -= Y[r][j] U[j][c] (c > j), the same broadcast row.  The threads of row j + 1 then
// publish it with its pivot's reciprocal.
__global__ void __launch_bounds__(kTopThreads) top_factor_kernel(uint32_t k0, uint32_t nb,
                                                                 const double* __restrict__ A, uint32_t lda,
                                                                 double* __restrict__ top_out,
                                                                 double* __restrict__ linv,
                                                                 double* __restrict__ uinv,
                                                                 int32_t* __restrict__ reject)
{
    constexpr int C = kTopCpt, G = kTopGroups;
    __shared__ __align__(16) double prow[2][G][kTopGs];  // row j of T
    __shared__ __align__(16) double xrow[2][G][kTopGs];  // row j of X
    __shared__ double rd[NB];                            // 1 / U[q][q]
    const uint32_t tid = threadIdx.x, row = tid / G, g = tid % G;
    const int src = (int)(tid & 31u & ~(uint32_t)(G - 1));  // lane of this row's group 0
    double t[C], x[C], y[C];
#pragma unroll
    for (int k = 0; k < C; ++k) {
        const uint32_t c = C * g + k;
        t[k] = (row < nb && c < nb) ? A[(size_t)(k0 + row) * lda + k0 + c] : (row == c ? 1.0 : 0.0);
        x[k] = y[k] = row == c ? 1.0 : 0.0;
    }
    bool bad = false;
    if (row == 0) {
#pragma unroll
        for (int k = 0; k < C; k += 2) {
            *reinterpret_cast<double2*>(&prow[0][g][k]) = make_double2(t[k], t[k + 1]);
            *reinterpret_cast<double2*>(&xrow[0][g][k]) = make_double2(x[k], x[k + 1]);
        }
        if (g == 0) {
            bad |= !(fabs(t[0]) >= kPivotLo && fabs(t[0]) <= kPivotHi);  // zero, tiny, huge or NaN pivot
            rd[0] = pivot_rcp(t[0]);
        }
    }
    __syncthreads();
#pragma unroll 1
    for (uint32_t gj = 0; gj < (uint32_t)G; ++gj) {
#pragma unroll
        for (int kj = 0; kj < C; ++kj) {
            const uint32_t j = C * gj + kj;
            const int b = kj & 1;
            const bool below = row > j;
            const double a = __shfl_sync(0xffffffffu, below ? t[kj] : y[kj], src + (int)gj) * rd[j];
            if (g == gj) {
                if (below) {
                    bad |= !(fabs(a) < pvl::dmma::kMultLimit);
                    t[kj] = a;
                } else {
                    y[kj] = a;
                }
            }
            if (g >= gj) {  // columns right of j: k > kj in group gj, every k in later groups
                const bool later = g > gj;
                if (below) {
#pragma unroll
                    for (int k = 0; k < C; k += 2) {
                        const double2 p = *reinterpret_cast<const double2*>(&prow[b][g][k]);
                        if (k > kj || later)
                            t[k] = fma(-a, p.x, t[k]);
                        if (k + 1 > kj || later)
                            t[k + 1] = fma(-a, p.y, t[k + 1]);
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < C; k += 2) {
                        const double2 p = *reinterpret_cast<const double2*>(&prow[b][g][k]);
                        if (k > kj || later)
                            y[k] = fma(-a, p.x, y[k]);
                        if (k + 1 > kj || later)
                            y[k + 1] = fma(-a, p.y, y[k + 1]);
                    }
                }
            }
            if (below && g <= gj) {  // X[j][c] = 0 for c > j
#pragma unroll
                for (int k = 0; k < C; k += 2) {
                    const double2 p = *reinterpret_cast<const double2*>(&xrow[b][g][k]);
                    x[k] = fma(-a, p.x, x[k]);
                    x[k + 1] = fma(-a, p.y, x[k + 1]);
                }
            }
            if (row == j + 1) {  // row j + 1 is final: publish it (never true after the last step)
                const int kn = (kj + 1) % C;
                const uint32_t gn = gj + (kj == C - 1 ? 1u : 0u);
#pragma unroll
                for (int k = 0; k < C; k += 2) {
                    *reinterpret_cast<double2*>(&prow[b ^ 1][g][k]) = make_double2(t[k], t[k + 1]);
                    *reinterpret_cast<double2*>(&xrow[b ^ 1][g][k]) = make_double2(x[k], x[k + 1]);
                }
                if (g == gn) {
                    bad |= !(fabs(t[kn]) >= kPivotLo && fabs(t[kn]) <= kPivotHi);
                    rd[j + 1] = pivot_rcp(t[kn]);
                }
            }
            __syncthreads();
        }
    }
    if (__syncthreads_or(bad) && tid == 0)
        atomicExch(reject, 1);
    const size_t o = (size_t)row * NB + C * g;
#pragma unroll
    for (int k = 0; k < C; k += 2) {
        *reinterpret_cast<double2*>(linv + o + k) = make_double2(x[k], x[k + 1]);
        *reinterpret_cast<double2*>(uinv + o + k) = make_double2(y[k], y[k + 1]);
    }
    if (row < nb) {
#pragma unroll
        for (int k = 0; k < C; ++k)
            if (C * g + k < nb)
                top_out[o + k] = t[k];
    }
}

constexpr int kApplyRows = 32;  // L21 tile: 32 rows x 64
constexpr int kApplyCols = 32;  // U12 tile: 64 x 32 columns
constexpr size_t kApplySmem = sizeof(pvl::dmma::Smem<64, 32>) > sizeof(pvl::dmma::Smem<32, 64>)
                                  ? sizeof(pvl::dmma::Smem<64, 32>) : sizeof(pvl::dmma::Smem<32, 64>);

// CTAs 0 .. n_ltiles-1: a 32-row tile of L21 = A21 U11^-1; the rest: a 32-column tile of
// U12 = L11^-1 A12.  Both in place, the old values backed up for the pivoting fallback.
template <bool VEC>
__global__ void __launch_bounds__(pvl::dmma::kThreads) panel_apply_kernel(uint32_t n, uint32_t k0,
                                                                          double* __restrict__ A, uint32_t lda,
                                                                          const double* __restrict__ linv,
                                                                          const double* __restrict__ uinv,
                                                                          double* __restrict__ backup,
                                                                          double* __restrict__ backup_row,
                                                                          int32_t* __restrict__ reject,
                                                                          uint32_t n_ltiles)
{
    using namespace pvl::dmma;
    extern __shared__ __align__(16) double apply_smem[];
    const uint32_t base = k0 + NB;
    if (blockIdx.x < n_ltiles) {
        auto& sm = *reinterpret_cast<Smem<kApplyRows, 64>*>(apply_smem);
        const uint32_t r0 = base + blockIdx.x * kApplyRows;
        tile<kApplyRows, 64, kLowerMul, VEC>(sm, A, lda, r0, k0, uinv, NB, 0, 0, A, lda, r0, k0,
                                             min((uint32_t)kApplyRows, n - r0), NB, backup, k0, 0, 0, reject);
    } else {
        auto& sm = *reinterpret_cast<Smem<64, kApplyCols>*>(apply_smem);
        const uint32_t c0 = base + (blockIdx.x - n_ltiles) * kApplyCols;
        tile<64, kApplyCols, kUpperMul, VEC>(sm, linv, NB, 0, 0, A, lda, k0, c0, A, lda, k0, c0, NB,
                                             min((uint32_t)kApplyCols, n - c0), backup_row, 0, 0, n, nullptr);
    }
}

// One rectangle of the trailing update A22 -= L21 U12: C = rows row0 .. row0 + m, columns
// col0 .. col0 + nn; A = the panel's L21 (columns a_col ..) on C's rows, B = its U12 (rows
// b_row ..) on C's columns.  `slots` runs of `per` 64 x 64 tiles.
struct UpdRect {
    uint32_t row0, col0, m, nn, a_col, b_row, per, slots;
};

UpdRect upd_rect(uint32_t row0, uint32_t col0, uint32_t m, uint32_t nn, uint32_t k0, uint32_t max_slots)
{
    const uint32_t tiles = blocks_for(m, pvl::dmma::kUpdTile) * blocks_for(nn, pvl::dmma::kUpdTile);
    UpdRect r{row0, col0, m, nn, k0, k0, 0, 0};
    r.per = tiles ? blocks_for(tiles, std::max(1u, max_slots)) : 1;
    r.slots = blocks_for(tiles, r.per);
    return r;
}

// One CTA per SM, each a run of tiles (dmma.cuh update_tiles: C and A blocks stream into shared
// memory one tile ahead of the MMAs).  CTA s < r0.slots runs tiles [s per, (s + 1) per) of r0,
// the CTAs after them those of r1 (each rectangle's tiles in column-major order).
template <bool VEC>
__global__ void __launch_bounds__(pvl::dmma::kUpdThreads, 1) dmma_update_kernel(double* __restrict__ A, uint32_t lda,
                                                                            UpdRect r0, UpdRect r1)
{
    extern __shared__ __align__(16) double upd_smem[];
    auto& sm = *reinterpret_cast<pvl::dmma::UpdSmem*>(upd_smem);
    uint32_t slot = blockIdx.x;
    const bool first = slot < r0.slots;
    const UpdRect r = first ? r0 : r1;
    if (!first)
        slot -= r0.slots;
    if (slot >= r.slots)
        return;
    constexpr uint32_t T = pvl::dmma::kUpdTile;
    const uint32_t tiles = ((r.m + T - 1) / T) * ((r.nn + T - 1) / T);
    const uint32_t t0 = slot * r.per, t1 = min(tiles, t0 + r.per);
    pvl::dmma::update_tiles<VEC>(sm, A, lda, r.row0, r.col0, r.m, r.nn, r.a_col, r.b_row, t0, t1);
}

// SMs left free while the bulk of a panel's trailing update runs on the side stream: the next
// panel's top block, apply and pivot kernels run there meanwhile.
constexpr int kLookaheadSms = 8;

// A second stream and two events per thread and device for the look-ahead fork and join (a
// stream may take part in one capture at a time: per thread, since captures here are
// thread-local).  Created on first use in a context and kept; a new context (after a device
// reset) gets new ones.
struct SideStream {
    void* ctx = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};

int side_stream(int dev, SideStream*& out)
{
    thread_local SideStream cache[64];
    if (dev < 0 || dev >= 64)
        return pvl_fail(PVL_ERR_ARG, "pvl_lu_factor: device %d out of range", dev);
    void* ctx = nullptr;
    if (int rc = pvl_current_context(&ctx))
        return rc;
    SideStream& c = cache[dev];
    if (!c.s || c.ctx != ctx) {
        c = SideStream{};
        PVL_CUDA_CHECK(cudaStreamCreateWithFlags(&c.s, cudaStreamNonBlocking));
        PVL_CUDA_CHECK(cudaEventCreateWithFlags(&c.fork, cudaEventDisableTiming));
        PVL_CUDA_CHECK(cudaEventCreateWithFlags(&c.join, cudaEventDisableTiming));
        c.ctx = ctx;
    }
    out = &c;
    return PVL_OK;
}

// ---------------------------------------------------------------- diagonal-block inverses
// One CTA per kRB-row block b: threads 0..63 form column c of L_bb^-1 (unit lower, forward
// substitution), threads 64..127 column c of U_bb^-1 (backward substitution), each column
// held in registers.  A partial last block is padded with identity.  The wavefront solves
// then apply each diagonal block as one parallel matrix-vector product.
template <typename T>
__global__ void __launch_bounds__(2 * kRB, 1) diag_inverse_kernel(uint32_t n, const T* __restrict__ M,
                                                                  uint32_t lda, T* __restrict__ inv)
{
    __shared__ T D[kRB][kRB + 1];
    const uint32_t b = blockIdx.x, r0 = b * kRB;
    const uint32_t rows = min((uint32_t)kRB, n - r0);
    for (uint32_t e = threadIdx.x; e < kRB * kRB; e += blockDim.x) {
        const uint32_t r = e / kRB, c = e % kRB;
        D[r][c] = (r < rows && c < rows) ? M[(size_t)(r0 + r) * lda + r0 + c] : (r == c ? T(1) : T(0));
    }
    __syncthreads();
    const bool lower = threadIdx.x < kRB;
    const int c = (int)(threadIdx.x & (kRB - 1));
    T y[kRB];
    if (lower) {
#pragma unroll
        for (int r = 0; r < kRB; ++r)
            y[r] = r == c ? T(1) : T(0);
#pragma unroll
        for (int q = 0; q < kRB - 1; ++q) {
            const T yq = y[q];
#pragma unroll
            for (int r = q + 1; r < kRB; ++r)
                y[r] -= D[r][q] * yq;
        }
    } else {
#pragma unroll
        for (int r = 0; r < kRB; ++r)
            y[r] = r == c ? T(1) : T(0);
#pragma unroll
        for (int q = kRB - 1; q >= 0; --q) {
            const T yq = y[q] / D[q][q];
            y[q] = yq;
#pragma unroll
            for (int r = 0; r < q; ++r)
                y[r] -= D[r][q] * yq;
        }
    }
    T* out = inv + ((size_t)b * 2 + (lower ? 0 : 1)) * kRB * kRB;
#pragma unroll
    for (int r = 0; r < kRB; ++r)
        out[(size_t)r * kRB + c] = y[r];
}

// ---------------------------------------------------------------- solve
__global__ void gather_kernel(uint32_t n, const int32_t* __restrict__ perm, const double* __restrict__ b,
                              double* __restrict__ out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n)
        out[i] = b[perm[i]];
}

// Blocked substitution with one launch per step and no inter-CTA waits (so that it can sit in a
// conditional body of a CUDA graph, where the wavefront's co-resident launch is not available):
// x_b = inv(D_bb) x_b for one diagonal block (one CTA), then the block's column slice updates
// the rows still to be solved (one warp per row).  Same inverted diagonal blocks as the wavefront.
template <bool LOWER>
__global__ void __launch_bounds__(kRB) diag_apply_kernel(uint32_t n, uint32_t b, const double* __restrict__ inv,
                                                         double* __restrict__ x)
{
    __shared__ double s[kRB];
    const uint32_t r0 = b * kRB, rows = min((uint32_t)kRB, n - r0), t = threadIdx.x;
    s[t] = t < rows ? x[r0 + t] : 0.0;
    __syncthreads();
    if (t < rows) {
        const double* D = inv + ((size_t)b * 2 + (LOWER ? 0 : 1)) * kRB * kRB + (size_t)t * kRB;
        double acc = 0.0;
#pragma unroll 8
        for (int c = 0; c < kRB; ++c)
            acc = fma(D[c], s[c], acc);
        x[r0 + t] = acc;
    }
}

template <bool LOWER>
__global__ void __launch_bounds__(256) block_update_kernel(uint32_t n, uint32_t b, const double* __restrict__ M,
                                                           uint32_t lda, double* __restrict__ x)
{
    const uint32_t c0 = b * kRB, cols = min((uint32_t)kRB, n - c0);
    const uint32_t first = LOWER ? c0 + cols : 0, count = LOWER ? n - first : c0;
    const uint32_t i = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (i >= count)
        return;
    const uint32_t r = first + i;
    const double* row = M + (size_t)r * lda + c0;
    double s = 0.0;
    for (uint32_t c = lane; c < cols; c += 32)
        s = fma(row[c], x[c0 + c], s);
    for (int o = 16; o > 0; o >>= 1)
        s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0)
        x[r] -= s;
}

int coresident_blocks(const void* fn, int threads)
{
    int dev = 0, sms = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
        return 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, threads, 0) != cudaSuccess)
        return 0;
    return sms * per;
}

}  // namespace

extern "C" size_t pvl_lu_workspace(uint32_t n) { return lu_ws_bytes(n); }

extern "C" int pvl_lu_factor(uint32_t n, double* A, uint32_t lda, int32_t* ipiv, int32_t* info, void* ws,
                             size_t ws_bytes, void* stream)
{
    if (n == 0)
        return PVL_OK;
    if (!A || !ipiv || !info || !ws)
        return pvl_fail(PVL_ERR_ARG, "pvl_lu_factor: null pointer argument");
    if (lda < n)
        return pvl_fail(PVL_ERR_ARG, "pvl_lu_factor: lda %u < n %u", lda, n);
    if (ws_bytes < lu_ws_bytes(n))
        return pvl_fail(PVL_ERR_ALLOC, "pvl_lu_factor: workspace %zu < %zu", ws_bytes, lu_ws_bytes(n));
    cudaStream_t st = (cudaStream_t)stream;
    LuWs w = carve(ws, n);
    const size_t trsm_smem = (size_t)(NB * (NB + 1) + NB * (kTrsmCols + 1)) * sizeof(double);
    const size_t upd_smem = sizeof(pvl::dmma::UpdSmem);
    int dev = 0, sms = 0;
    PVL_CUDA_CHECK(cudaGetDevice(&dev));
    PVL_CUDA_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    SideStream* side = nullptr;
    if (int rc = side_stream(dev, side))
        return rc;
    // 16-byte operand copies and stores need even row strides and an even width
    const bool vec = (lda % 2 == 0) && (n % 2 == 0) && (((uintptr_t)A & 15u) == 0);
    const void* apply_fn = vec ? (const void*)panel_apply_kernel<true> : (const void*)panel_apply_kernel<false>;
    const void* upd_fn = vec ? (const void*)dmma_update_kernel<true> : (const void*)dmma_update_kernel<false>;
    PVL_SMEM_OPTIN(trsm_kernel<double>, trsm_smem);
    PVL_SMEM_OPTIN(apply_fn, kApplySmem);
    PVL_SMEM_OPTIN(upd_fn, upd_smem);
    auto update = [&](cudaStream_t s, const UpdRect& r0, const UpdRect& r1) -> int {
        const uint32_t ctas = r0.slots + r1.slots;
        if (ctas == 0)
            return PVL_OK;
        void* args[] = {(void*)&A, (void*)&lda, (void*)&r0, (void*)&r1};
        PVL_CUDA_CHECK(cudaLaunchKernel(upd_fn, dim3(ctas), dim3(pvl::dmma::kUpdThreads), args, upd_smem, s));
        pvl_count_launch();
        return PVL_OK;
    };
    const UpdRect none{0, 0, 0, 0, 0, 0, 1, 0};
    const uint32_t all_slots = (uint32_t)sms;  // one CTA per SM
    const uint32_t bulk_slots = (uint32_t)std::max(1, sms - kLookaheadSms);
    int32_t* perm = ipiv + n;
    PVL_CUDA_CHECK(cudaMemsetAsync(info, 0, sizeof(int32_t), st));
    init_perm_kernel<<<blocks_for(n, 256), 256, 0, st>>>(n, perm);
    PVL_LAUNCH_CHECK();
    const uint32_t n_panels = (n + NB - 1) / NB;
    PVL_CUDA_CHECK(cudaMemsetAsync(w.reject, 0, sizeof(int32_t) * (n_panels + 1), st));
    // Look-ahead: panel p's trailing update is split into the next panel's column and row
    // blocks (the L shape next to this panel, on `st`) and the rest (on the side stream, on all
    // but kLookaheadSms SMs).  Panel p + 1's top block, apply and pivot kernels touch only its
    // own columns and row block, so they run on `st` while the rest of panel p's update is in
    // flight; its trsm kernel (whose fallback interchanges reach every column) and everything
    // after wait for it.
    bool pending = false;
    for (uint32_t p = 0; p < n_panels; ++p) {
        const uint32_t k0 = p * NB;
        const uint32_t nb = std::min<uint32_t>(NB, n - k0);
        const uint32_t below = n - k0 - nb;  // nonzero only for full panels (nb == NB)
        top_factor_kernel<<<1, kTopThreads, 0, st>>>(k0, nb, A, lda, w.top_out, w.linv, w.uinv, w.reject + p);
        PVL_LAUNCH_CHECK();
        if (below > 0) {
            const uint32_t nl = blocks_for(below, kApplyRows), nu = blocks_for(below, kApplyCols);
            double* bk = w.backup;
            double* bkr = w.backup_row;
            const double* li = w.linv;
            const double* ui = w.uinv;
            int32_t* rj = w.reject + p;
            void* args[] = {(void*)&n, (void*)&k0, (void*)&A, (void*)&lda, (void*)&li, (void*)&ui, (void*)&bk,
                            (void*)&bkr, (void*)&rj, (void*)&nl};
            PVL_CUDA_CHECK(cudaLaunchKernel(apply_fn, dim3(nl + nu), dim3(pvl::dmma::kThreads), args, kApplySmem, st));
            pvl_count_launch();
        }
        panel_pivot_kernel<double><<<1, 1024, 0, st>>>(n, k0, nb, A, lda, w.backup, w.top_out, w.reject, w.ok, p, ipiv,
                                                       perm, info, below > 0 ? w.backup_row : nullptr);
        PVL_LAUNCH_CHECK();
        if (pending) {  // the rest of the previous panel's update
            PVL_CUDA_CHECK(cudaEventRecord(side->join, side->s));
            PVL_CUDA_CHECK(cudaStreamWaitEvent(st, side->join, 0));
            pending = false;
        }
        if (n > nb) {
            trsm_kernel<double><<<blocks_for(n - nb, kTrsmCols), kTrsmCols, trsm_smem, st>>>(n, k0, nb, A, lda, w.ok, p,
                                                                                           ipiv, 1);
            PVL_LAUNCH_CHECK();
        }
        if (below == 0)
            continue;
        const uint32_t base = k0 + NB;
        if (below <= (uint32_t)pvl::dmma::kUpdTile) {  // one tile column: no look-ahead split
            if (int rc = update(st, upd_rect(base, base, below, below, k0, all_slots), none))
                return rc;
            continue;
        }
        const uint32_t step = pvl::dmma::kUpdTile;
        if (int rc = update(st, upd_rect(base, base, below, step, k0, all_slots),
                            upd_rect(base, base + step, step, below - step, k0, all_slots)))
            return rc;
        PVL_CUDA_CHECK(cudaEventRecord(side->fork, st));
        PVL_CUDA_CHECK(cudaStreamWaitEvent(side->s, side->fork, 0));
        if (int rc = update(side->s, upd_rect(base + step, base + step, below - step, below - step, k0, bulk_slots),
                            none))
            return rc;
        pending = true;
    }
    if (pending) {
        PVL_CUDA_CHECK(cudaEventRecord(side->join, side->s));
        PVL_CUDA_CHECK(cudaStreamWaitEvent(st, side->join, 0));
    }
    diag_inverse_kernel<double><<<(n + kRB - 1) / kRB, 2 * kRB, 0, st>>>(n, A, lda, w.inv);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" size_t pvl_lu_solve_workspace(uint32_t n) { return lu_ws_bytes(n); }

extern "C" int pvl_lu_solve(uint32_t n, const double* LU, uint32_t lda, const int32_t* ipiv, double* b,
                            int32_t* err, void* ws, size_t ws_bytes, void* stream)
{
    if (n == 0)
        return PVL_OK;
    if (!LU || !ipiv || !b || !ws || !err)
        return pvl_fail(PVL_ERR_ARG, "pvl_lu_solve: null pointer argument");
    if (ws_bytes < lu_ws_bytes(n))
        return pvl_fail(PVL_ERR_ALLOC, "pvl_lu_solve: workspace too small");
    const uint32_t nblk = (n + kRB - 1) / kRB;
    const void* fwd = (const void*)pvl::trsv::wavefront_kernel<true>;
    const void* bwd = (const void*)pvl::trsv::wavefront_kernel<false>;
    if ((int)nblk > coresident_blocks(fwd, kSolveThreads) || (int)nblk > coresident_blocks(bwd, kSolveThreads))
        return pvl_fail(PVL_ERR_ARG, "pvl_lu_solve: n = %u needs %u co-resident blocks", n, nblk);
    cudaStream_t st = (cudaStream_t)stream;
    LuWs w = carve(ws, n);
    const int32_t* perm = ipiv + n;
    PVL_CUDA_CHECK(cudaMemsetAsync(err, 0, sizeof(int32_t), st));
    gather_kernel<<<blocks_for(n, 256), 256, 0, st>>>(n, perm, b, w.tmp);
    PVL_LAUNCH_CHECK();
    long long spin = pvl::trsv::kSpinLimit;
    int32_t skip = -1;
    for (int pass = 0; pass < 2; ++pass) {
        PVL_CUDA_CHECK(cudaMemsetAsync(w.flags, 0, sizeof(int32_t) * (nblk + 1), st));
        double* xt = w.tmp;
        int32_t* fl = w.flags;
        const double* iv = w.inv;
        void* args[] = {(void*)&n, (void*)&LU, (void*)&lda, (void*)&iv, (void*)&xt, (void*)&fl, (void*)&err,
                        (void*)&spin, (void*)&skip};
        PVL_CUDA_CHECK(cudaLaunchCooperativeKernel(pass == 0 ? fwd : bwd, dim3(nblk), dim3(kSolveThreads), args, 0, st));
        pvl_count_launch();
    }
    PVL_CUDA_CHECK(cudaMemcpyAsync(b, w.tmp, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    return PVL_OK;
}

extern "C" int pvl_lu_solve_blocked(uint32_t n, const double* LU, uint32_t lda, const int32_t* ipiv, double* b,
                                    void* ws, size_t ws_bytes, void* stream)
{
    if (n == 0)
        return PVL_OK;
    if (!LU || !ipiv || !b || !ws)
        return pvl_fail(PVL_ERR_ARG, "pvl_lu_solve_blocked: null pointer argument");
    if (ws_bytes < lu_ws_bytes(n))
        return pvl_fail(PVL_ERR_ALLOC, "pvl_lu_solve_blocked: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    LuWs w = carve(ws, n);
    const uint32_t nblk = (n + kRB - 1) / kRB;
    gather_kernel<<<blocks_for(n, 256), 256, 0, st>>>(n, ipiv + n, b, w.tmp);
    PVL_LAUNCH_CHECK();
    for (uint32_t k = 0; k < nblk; ++k) {
        diag_apply_kernel<true><<<1, kRB, 0, st>>>(n, k, w.inv, w.tmp);
        PVL_LAUNCH_CHECK();
        const uint32_t below = n - std::min(n, (k + 1) * kRB);
        if (below) {
            block_update_kernel<true><<<blocks_for(below, 8), 256, 0, st>>>(n, k, LU, lda, w.tmp);
            PVL_LAUNCH_CHECK();
        }
    }
    for (uint32_t k = nblk; k-- > 0;) {
        diag_apply_kernel<false><<<1, kRB, 0, st>>>(n, k, w.inv, w.tmp);
        PVL_LAUNCH_CHECK();
        if (k) {
            block_update_kernel<false><<<blocks_for(k * kRB, 8), 256, 0, st>>>(n, k, LU, lda, w.tmp);
            PVL_LAUNCH_CHECK();
        }
    }
    PVL_CUDA_CHECK(cudaMemcpyAsync(b, w.tmp, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    return PVL_OK;
}

// ================================================================ FP32 LU (TF32 trailing update)
// The low-precision factorisation behind the mixed path's preconditioner.  Speculative panel
// (panel_spec_kernel), pivot and TRSM kernels instantiated for float, with the trailing update
// A22 -= L21 U12 on the tensor cores (U12 transposed into a K-major operand, then
// pvl_gemm_tf32: TMA-fed tcgen05 MMAs, TF32 products, FP32 accumulation).  The explicit inverse U^-1 L^-1 is then formed from the factors by blocked
// triangular inversion: the 64 x 64 diagonal-block products on CUDA cores in FP32, every
// rank-64 update on the tensor cores.  Applying the preconditioner is then one FP32
// matrix-vector product per Krylov iteration instead of two latency-bound triangular solves.
namespace {

// out[r][j] = sum_k D[r][k] in[k][j] for the 64 rows of a block (FP32, CUDA cores: the
// diagonal blocks of the inverse carry the O(1) entries whose TF32 rounding would dominate
// the preconditioner's error).  One thread per column, D staged in shared memory.
__global__ void __launch_bounds__(128) block_apply_kernel(uint32_t cols, const float* __restrict__ D,
                                                          const float* __restrict__ in, uint32_t ldi,
                                                          float* __restrict__ out, uint32_t ldo)
{
    __shared__ float sD[kRB][kRB];
    for (uint32_t e = threadIdx.x; e < kRB * kRB; e += blockDim.x)
        sD[e / kRB][e % kRB] = D[e];
    __syncthreads();
    const uint32_t j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= cols)
        return;
    float x[kRB];
#pragma unroll
    for (int k = 0; k < kRB; ++k)
        x[k] = in[(size_t)k * ldi + j];
#pragma unroll 4
    for (int r = 0; r < kRB; ++r) {
        float s = 0.0f;
#pragma unroll
        for (int k = 0; k < kRB; ++k)
            s = fmaf(sD[r][k], x[k], s);
        out[(size_t)r * ldo + j] = s;
    }
}

__global__ void set_identity_kernel(uint32_t n, float* __restrict__ X, uint32_t ldx)
{
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)n * n)
        return;
    const uint32_t r = (uint32_t)(t / n), c = (uint32_t)(t % n);
    X[(size_t)r * ldx + c] = r == c ? 1.0f : 0.0f;
}

// out[r][perm[c]] = X[r][c]: the inverse's columns permuted, so that A^-1 b = out b.
__global__ void permute_columns_kernel(uint32_t n, const float* __restrict__ X, uint32_t ldx,
                                       const int32_t* __restrict__ perm, float* __restrict__ out, uint32_t ldo)
{
    const size_t t = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (size_t)n * n)
        return;
    const uint32_t r = (uint32_t)(t / n), c = (uint32_t)(t % n);
    const uint32_t q = (uint32_t)perm[c];
    if (q < n)  // a valid factorisation never maps outside [0, n)
        out[(size_t)r * ldo + q] = X[(size_t)r * ldx + c];
}

// dst (cols x 64, row-major) = the transpose of the 64 x cols block src (leading dimension
// lds): the K-major form of a rank-64 update's right operand for the tensor-core GEMM.
__global__ void __launch_bounds__(256) transpose64_kernel(uint32_t cols, const float* __restrict__ src, uint32_t lds,
                                                          float* __restrict__ dst)
{
    __shared__ float t[32][33];
    const uint32_t c0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
    const uint32_t tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
    for (uint32_t k = ty; k < 32; k += 8)
        t[k][tx] = c0 + tx < cols ? src[(size_t)(k0 + k) * lds + c0 + tx] : 0.0f;
    __syncthreads();
    for (uint32_t c = ty; c < 32; c += 8)
        if (c0 + c < cols)
            dst[(size_t)(c0 + c) * kRB + k0 + tx] = t[tx][c];
}

}  // namespace

extern "C" int pvl_gemm_tf32(uint32_t M, uint32_t N, uint32_t K, float alpha, const float* A, uint32_t lda,
                             const float* Bt, uint32_t ldbt, float beta, float* C, uint32_t ldc, int32_t* err,
                             void* stream);

namespace {
// C (M x cols) -= A (M x 64, lda) * B where B is the 64 x cols block at src (lds): B is
// transposed into bt (cols x 64) first, then the tensor-core GEMM runs on K-major operands.
int rank64_update(uint32_t M, uint32_t cols, const float* A, uint32_t lda, const float* src, uint32_t lds, float* bt,
                  float* C, uint32_t ldc, int32_t* err, cudaStream_t st)
{
    transpose64_kernel<<<dim3(blocks_for(cols, 32), kRB / 32), 256, 0, st>>>(cols, src, lds, bt);
    PVL_LAUNCH_CHECK();
    return pvl_gemm_tf32(M, cols, kRB, -1.0f, A, lda, bt, kRB, 1.0f, C, ldc, err, st);
}
}  // namespace

extern "C" size_t pvl_lu32_workspace(uint32_t n) { return lu_ws_bytes(n); }

extern "C" int pvl_lu32_factor(uint32_t n, float* A, uint32_t lda, int32_t* ipiv, int32_t* info, int32_t* err,
                               void* ws, size_t ws_bytes, void* stream)
{
    if (n == 0)
        return PVL_OK;
    if (!A || !ipiv || !info || !err || !ws)
        return pvl_fail(PVL_ERR_ARG, "pvl_lu32_factor: null pointer argument");
    if (lda < n || lda % 4 || ((uintptr_t)A & 15u))
        return pvl_fail(PVL_ERR_ARG, "pvl_lu32_factor: lda must be >= n and a multiple of 4, A 16-byte aligned");
    if (ws_bytes < lu_ws_bytes(n))
        return pvl_fail(PVL_ERR_ALLOC, "pvl_lu32_factor: workspace %zu < %zu", ws_bytes, lu_ws_bytes(n));
    cudaStream_t st = (cudaStream_t)stream;
    LuWs w = carve(ws, n);
    float* backup = reinterpret_cast<float*>(w.backup);
    float* top_out = reinterpret_cast<float*>(w.top_out);
    float* inv = reinterpret_cast<float*>(w.inv);
    float* ut = reinterpret_cast<float*>(w.backup_row);  // U12 transposed for the tensor-core updates
    const size_t trsm_smem = (size_t)(NB * (NB + 1) + NB * (kTrsmCols + 1)) * sizeof(float);
    PVL_SMEM_OPTIN(trsm_kernel<float>, trsm_smem);
    int32_t* perm = ipiv + n;
    PVL_CUDA_CHECK(cudaMemsetAsync(info, 0, sizeof(int32_t), st));
    PVL_CUDA_CHECK(cudaMemsetAsync(err, 0, sizeof(int32_t), st));
    init_perm_kernel<<<blocks_for(n, 256), 256, 0, st>>>(n, perm);
    PVL_LAUNCH_CHECK();
    const uint32_t n_panels = (n + NB - 1) / NB;
    PVL_CUDA_CHECK(cudaMemsetAsync(w.reject, 0, sizeof(int32_t) * (n_panels + 1), st));
    for (uint32_t p = 0; p < n_panels; ++p) {
        const uint32_t k0 = p * NB;
        const uint32_t nb = std::min<uint32_t>(NB, n - k0);
        const uint32_t below = n - k0 - nb;
        const uint32_t ctas = std::max<uint32_t>(1, (below + kSlabRows - 1) / kSlabRows);
        panel_spec_kernel<float><<<ctas, 2 * kSlabRows, 0, st>>>(n, k0, nb, A, lda, backup, top_out, w.reject + p);
        PVL_LAUNCH_CHECK();
        panel_pivot_kernel<float><<<1, 1024, 0, st>>>(n, k0, nb, A, lda, backup, top_out, w.reject, w.ok, p, ipiv,
                                                      perm, info, nullptr);
        PVL_LAUNCH_CHECK();
        if (n > nb) {
            trsm_kernel<float><<<blocks_for(n - nb, kTrsmCols), kTrsmCols, trsm_smem, st>>>(n, k0, nb, A, lda, w.ok, p,
                                                                                          ipiv, 0);
            PVL_LAUNCH_CHECK();
        }
        if (below > 0) {
            // every panel with rows below it is a full NB = 64 wide, so K = 64 (a multiple of 32)
            float* a22 = A + (size_t)(k0 + nb) * lda + k0 + nb;
            if (int r = rank64_update(below, below, A + (size_t)(k0 + nb) * lda + k0, lda, A + (size_t)k0 * lda + k0 + nb,
                                      lda, ut, a22, lda, err, st))
                return r;
        }
    }
    diag_inverse_kernel<float><<<(n + kRB - 1) / kRB, 2 * kRB, 0, st>>>(n, A, lda, inv);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_lu32_inverse(uint32_t n, const float* LU, uint32_t lda, const int32_t* perm, float* X,
                                uint32_t ldx, float* Y, uint32_t ldy, int32_t* err, void* ws, size_t ws_bytes,
                                void* stream)
{
    if (n == 0)
        return PVL_OK;
    if (!LU || !X || !Y || !err || !ws)
        return pvl_fail(PVL_ERR_ARG, "pvl_lu32_inverse: null pointer argument");
    if (n % kRB)
        return pvl_fail(PVL_ERR_ARG, "pvl_lu32_inverse: n = %u must be a multiple of %d", n, kRB);
    if (lda < n || ldx < n || ldy < n || lda % 4 || ldx % 4 || ldy % 4 ||
        (((uintptr_t)LU | (uintptr_t)X | (uintptr_t)Y) & 15u))
        return pvl_fail(PVL_ERR_ARG, "pvl_lu32_inverse: leading dimensions must be >= n and multiples of 4, "
                                     "arrays 16-byte aligned");
    if (ws_bytes < lu_ws_bytes(n))
        return pvl_fail(PVL_ERR_ALLOC, "pvl_lu32_inverse: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    LuWs w = carve(ws, n);
    const float* inv = reinterpret_cast<const float*>(w.inv);  // written by pvl_lu32_factor
    float* bt = reinterpret_cast<float*>(w.backup_row);         // transposed update operands
    const uint32_t nblk = n / kRB;
    // forward: Y = L^-1, with X as the working right-hand side (starts as I)
    set_identity_kernel<<<blocks_for((size_t)n * n, 256), 256, 0, st>>>(n, X, ldx);
    PVL_LAUNCH_CHECK();
    PVL_CUDA_CHECK(cudaMemset2DAsync(Y, (size_t)ldy * sizeof(float), 0, (size_t)n * sizeof(float), n, st));
    for (uint32_t k = 0; k < nblk; ++k) {
        const uint32_t r0 = k * kRB, cols = r0 + kRB;  // L^-1 is zero right of the diagonal block
        block_apply_kernel<<<blocks_for(cols, 128), 128, 0, st>>>(cols, inv + (size_t)k * 2 * kRB * kRB,
                                                                 X + (size_t)r0 * ldx, ldx, Y + (size_t)r0 * ldy, ldy);
        PVL_LAUNCH_CHECK();
        if (cols < n)
            if (int r = rank64_update(n - cols, cols, LU + (size_t)cols * lda + r0, lda, Y + (size_t)r0 * ldy, ldy, bt,
                                      X + (size_t)cols * ldx, ldx, err, st))
                return r;
    }
    // backward: X = U^-1 Y, with Y as the working right-hand side
    for (uint32_t kk = nblk; kk-- > 0;) {
        const uint32_t r0 = kk * kRB;
        block_apply_kernel<<<blocks_for(n, 128), 128, 0, st>>>(n, inv + ((size_t)kk * 2 + 1) * kRB * kRB,
                                                              Y + (size_t)r0 * ldy, ldy, X + (size_t)r0 * ldx, ldx);
        PVL_LAUNCH_CHECK();
        if (r0 > 0)
            if (int r = rank64_update(r0, n, LU + r0, lda, X + (size_t)r0 * ldx, ldx, bt, Y, ldy, err, st))
                return r;
    }
    if (perm) {
        // A^-1 = U^-1 L^-1 P with (P b)[i] = b[perm[i]]: fold P into the columns
        permute_columns_kernel<<<blocks_for((size_t)n * n, 256), 256, 0, st>>>(n, X, ldx, perm, Y, ldy);
        PVL_LAUNCH_CHECK();
        PVL_CUDA_CHECK(cudaMemcpy2DAsync(X, (size_t)ldx * sizeof(float), Y, (size_t)ldy * sizeof(float),
                                         (size_t)n * sizeof(float), n, cudaMemcpyDeviceToDevice, st));
    }
    return PVL_OK;
}
