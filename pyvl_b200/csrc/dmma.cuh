// FP64 tensor-core tiles (mma.sync m16n8k8 .f64) for the LU's rank-64 products.
//
// A CTA of 128 threads (2 x 2 warps) computes a BM x BN tile of A (M x 64) * B (64 x N), all
// row-major FP64, with the whole K = 64 staged in shared memory by cp.async (8-byte copies when
// a leading dimension is odd, 16-byte ones otherwise).  Shared rows are padded to 68 doubles,
// so the fragment loads of a half-warp (groupID 0..3, thread-in-group 0..3) hit 16 distinct
// 8-byte bank pairs.  Fragment layout of mma.m16n8k8 .f64 (g = lane / 4, t = lane % 4):
//   A 16 x 8: a0 (g, t), a1 (g + 8, t), a2 (g, t + 4), a3 (g + 8, t + 4)
//   B 8 x 8:  b0 (t, g), b1 (t + 4, g)
//   C 16 x 8: c0 (g, 2t), c1 (g, 2t + 1), c2 (g + 8, 2t), c3 (g + 8, 2t + 1)
// Modes:
//   kUpdate   C -= A B (the trailing update): C is loaded into the accumulators (negated)
//             while the operands are in flight, so the epilogue only stores.
//   kLowerMul C = A B where C aliases A (A21 := A21 U11^-1, the panel's multipliers): the CTA's
//             A rows go to a backup first; any |C| >= kMultLimit or non-finite sets *flag.
//   kUpperMul C = A B where C aliases B (A12 := L11^-1 A12): the CTA's B columns go to a backup.
#pragma once

#include <cstdint>

namespace pvl {
namespace dmma {

constexpr int K = 64;            // the panel width: the inner dimension of every product here
constexpr int kPad = 68;         // shared row stride in doubles (68 = 4 mod 16: conflict-free fragments)
constexpr int kThreads = 128;
// A multiplier at least this large (or a NaN) means partial pivoting might have chosen another
// row at that column: the panel is refactored with explicit pivoting.  The margin below 1
// sends near-ties to the exact getf2 order as well.
constexpr double kMultLimit = 1.0 - 1e-12;

enum Mode { kUpdate = 0, kLowerMul = 1, kUpperMul = 2 };

__device__ __forceinline__ void mma16x8x8(double (&c)[4], const double (&a)[4], const double (&b)[2])
{
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

__device__ __forceinline__ uint32_t smem_addr(const void* p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Copy BYTES (8 or 16) from global to shared; zero-fill when !valid (src is then not read).
template <int BYTES>
__device__ __forceinline__ void cp_async(void* dst, const void* src, bool valid)
{
    const uint32_t d = smem_addr(dst);
    const uint32_t n = valid ? BYTES : 0;
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(n) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;" ::"r"(d), "l"(src), "r"(n) : "memory");
}

__device__ __forceinline__ void cp_async_wait_all()
{
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// rows x 64 block at (row0, col0) of a row-major matrix into sm[rows][kPad]; rows past
// row_end read as zero.
// NTHR threads copy, tid = 0 .. NTHR - 1 the caller's index among them.
template <int ROWS, bool VEC, int NTHR = kThreads>
__device__ __forceinline__ void stage_rows(double* sm, const double* __restrict__ g, uint32_t ld, uint32_t row0,
                                           uint32_t row_end, uint32_t col0, uint32_t tid = threadIdx.x)
{
    constexpr int PER = VEC ? 2 : 1;           // doubles per copy
    constexpr int CHUNKS = K / PER;            // copies per row
    for (uint32_t e = tid; e < (uint32_t)(ROWS * CHUNKS); e += NTHR) {
        const uint32_t r = e / CHUNKS, c = (e % CHUNKS) * PER;
        const bool ok = row0 + r < row_end;
        const double* src = ok ? g + (size_t)(row0 + r) * ld + col0 + c : g;
        cp_async<8 * PER>(sm + r * kPad + c, src, ok);
    }
}

// 64 x COLS block at (row0, col0) into sm[64][kPad] (columns past col_end read as zero).
template <int COLS, bool VEC, int NTHR = kThreads>
__device__ __forceinline__ void stage_cols(double* sm, const double* __restrict__ g, uint32_t ld, uint32_t row0,
                                           uint32_t col0, uint32_t col_end, uint32_t tid = threadIdx.x)
{
    constexpr int PER = VEC ? 2 : 1;
    constexpr int CHUNKS = COLS / PER;
    for (uint32_t e = tid; e < (uint32_t)(K * CHUNKS); e += NTHR) {
        const uint32_t r = e / CHUNKS, c = (e % CHUNKS) * PER;
        const bool ok = col0 + c < col_end;  // col_end and c are even when VEC
        const double* src = ok ? g + (size_t)(row0 + r) * ld + col0 + c : g;
        cp_async<8 * PER>(sm + r * kPad + c, src, ok);
    }
}

template <int BM, int BN>
struct Smem {
    double a[BM * kPad];
    double b[K * kPad];
};

// One BM x BN tile.  A: rows [a_row0, a_row0 + BM) x cols [a_col0, a_col0 + 64) of (lda);
// B: rows [b_row0, b_row0 + 64) x cols [b_col0, b_col0 + BN) of (ldb); C: rows [c_row0, ...) x
// cols [c_col0, ...) of (ldc), valid below m_end / n_end (tile-relative bounds in M and N).
// bk: backup of the aliased operand (kLowerMul: A rows at bk[(row - bk_row0) * 64 + k];
// kUpperMul: B at bk[k * bk_ld + col - bk_col0]).
template <int BM, int BN, int MODE, bool VEC>
__device__ __forceinline__ void tile(Smem<BM, BN>& s, const double* A, uint32_t lda, uint32_t a_row0, uint32_t a_col0,
                                     const double* B, uint32_t ldb, uint32_t b_row0, uint32_t b_col0, double* C,
                                     uint32_t ldc, uint32_t c_row0, uint32_t c_col0, uint32_t m_end, uint32_t n_end,
                                     double* bk, uint32_t bk_row0, uint32_t bk_col0, uint32_t bk_ld, int32_t* flag)
{
    constexpr int WM = BM / 2, WN = BN / 2;    // warp tile
    constexpr int MT = WM / 16, NT = WN / 8;   // MMA tiles per warp
    static_assert(MT >= 1 && NT >= 1 && WM % 16 == 0 && WN % 8 == 0, "tile shape");
    const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t g = lane >> 2, t = lane & 3;
    const uint32_t wm0 = (warp >> 1) * WM, wn0 = (warp & 1) * WN;
    stage_rows<BM, VEC>(s.a, A, lda, a_row0, a_row0 + m_end, a_col0);
    stage_cols<BN, VEC>(s.b, B, ldb, b_row0, b_col0, b_col0 + n_end);
    double acc[MT][NT][4];
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j) {
#pragma unroll
            for (int q = 0; q < 4; ++q)
                acc[i][j][q] = 0.0;
            if (MODE == kUpdate) {  // acc = -C while the operands are in flight
                const uint32_t col = wn0 + 8 * j + 2 * t;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const uint32_t row = wm0 + 16 * i + g + 8 * h;
                    if (row < m_end) {
                        const double* cp = C + (size_t)(c_row0 + row) * ldc + c_col0 + col;
                        if (VEC && col + 1 < n_end) {
                            const double2 v = *reinterpret_cast<const double2*>(cp);
                            acc[i][j][2 * h] = -v.x;
                            acc[i][j][2 * h + 1] = -v.y;
                        } else {
                            if (col < n_end)
                                acc[i][j][2 * h] = -cp[0];
                            if (col + 1 < n_end)
                                acc[i][j][2 * h + 1] = -cp[1];
                        }
                    }
                }
            }
        }
    cp_async_wait_all();
    __syncthreads();
    if (MODE == kLowerMul) {  // backup of the A rows about to be overwritten
        for (uint32_t e = threadIdx.x; e < (uint32_t)(BM * K); e += kThreads) {
            const uint32_t r = e / K, k = e % K;
            if (r < m_end)
                bk[(size_t)(a_row0 + r - bk_row0) * K + k] = s.a[r * kPad + k];
        }
    } else if (MODE == kUpperMul) {
        for (uint32_t e = threadIdx.x; e < (uint32_t)(K * BN); e += kThreads) {
            const uint32_t k = e / BN, c = e % BN;
            if (c < n_end)
                bk[(size_t)k * bk_ld + b_col0 + c - bk_col0] = s.b[k * kPad + c];
        }
    }
#pragma unroll
    for (int k0 = 0; k0 < K; k0 += 8) {
        double af[MT][4], bf[NT][2];
#pragma unroll
        for (int i = 0; i < MT; ++i) {
            const double* p = s.a + (wm0 + 16 * i + g) * kPad + k0 + t;
            af[i][0] = p[0];
            af[i][1] = p[8 * kPad];
            af[i][2] = p[4];
            af[i][3] = p[8 * kPad + 4];
        }
#pragma unroll
        for (int j = 0; j < NT; ++j) {
            const double* p = s.b + (k0 + t) * kPad + wn0 + 8 * j + g;
            bf[j][0] = p[0];
            bf[j][1] = p[4 * kPad];
        }
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < NT; ++j)
                mma16x8x8(acc[i][j], af[i], bf[j]);
    }
    bool bad = false;
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j) {
            const uint32_t col = wn0 + 8 * j + 2 * t;
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const uint32_t row = wm0 + 16 * i + g + 8 * h;
                double v0 = acc[i][j][2 * h], v1 = acc[i][j][2 * h + 1];
                if (MODE == kUpdate) {
                    v0 = -v0;
                    v1 = -v1;
                }
                if (row >= m_end)
                    continue;
                if (MODE == kLowerMul) {
                    if (col < n_end)
                        bad |= !(fabs(v0) < kMultLimit);
                    if (col + 1 < n_end)
                        bad |= !(fabs(v1) < kMultLimit);
                }
                double* cp = C + (size_t)(c_row0 + row) * ldc + c_col0 + col;
                if (VEC && col + 1 < n_end) {
                    *reinterpret_cast<double2*>(cp) = make_double2(v0, v1);
                } else {
                    if (col < n_end)
                        cp[0] = v0;
                    if (col + 1 < n_end)
                        cp[1] = v1;
                }
            }
        }
    if (MODE == kLowerMul && __syncthreads_or(bad) && threadIdx.x == 0)
        atomicExch(flag, 1);
}

// ---------------------------------------------------------------- pipelined trailing update
// C -= A B over a run of 64 x 64 tiles of one M x N block C (rows row0.., columns col0..),
// A: the 64 columns a_col.. of C's rows, B: the 64 rows b_row.. of C's columns.  Tiles in
// column-major order, so that consecutive tiles of a run share their B block.  One CTA of
// kUpdWarps warps (8: warp tile 32 x 16; 4: 32 x 32) per SM.  The C and A blocks of each tile
// stream into a two-deep ring of shared memory by cp.async, issued one whole tile ahead: while
// tile t is multiplied, tile t + 1's blocks are already there and tile t + 2's are in flight;
// the accumulators start from -C (shared memory) and the result goes from registers to global
// memory.  So every tile costs its MMAs, two barriers and a few shared loads, and the HBM
// traffic (C in and out) runs underneath.
#ifndef PVL_UPD_WARPS
#define PVL_UPD_WARPS 8
#endif
constexpr int kUpdTile = 64;
constexpr int kUpdWarps = PVL_UPD_WARPS;
constexpr int kUpdThreads = 32 * kUpdWarps;
static_assert(kUpdWarps == 4 || kUpdWarps == 8, "2 x 2 or 2 x 4 warps over a 64 x 64 tile");
struct UpdSmem {
    double a[2][kUpdTile * kPad];
    double c[2][kUpdTile * kPad];
    double b[K * kPad];
};

// ROWS x COLS block at (row0, col0) of a row-major matrix into sm[ROWS][kPad]; rows past
// row_end and columns past col_end are not copied (their contents are never used).
template <int ROWS, int COLS, bool VEC, int NTHR>
__device__ __forceinline__ void stage_tile(double* sm, const double* __restrict__ g, uint32_t ld, uint32_t row0,
                                           uint32_t row_end, uint32_t col0, uint32_t col_end, uint32_t tid)
{
    constexpr int PER = VEC ? 2 : 1;
    constexpr int CHUNKS = COLS / PER;
    for (uint32_t e = tid; e < (uint32_t)(ROWS * CHUNKS); e += NTHR) {
        const uint32_t r = e / CHUNKS, c = (e % CHUNKS) * PER;
        if (row0 + r < row_end && col0 + c < col_end)  // col_end and c are even when VEC
            cp_async<8 * PER>(sm + r * kPad + c, g + (size_t)(row0 + r) * ld + col0 + c, true);
    }
}

template <bool VEC>
__device__ __forceinline__ void update_tiles(UpdSmem& s, double* __restrict__ Cm, uint32_t ld, uint32_t row0,
                                             uint32_t col0, uint32_t m, uint32_t nn, uint32_t a_col, uint32_t b_row,
                                             uint32_t t_begin, uint32_t t_end)
{
    constexpr int WN = kUpdWarps / 2;     // warps along N
    constexpr int MT = 2, NT = 8 / WN;    // warp tile 32 x (64 / WN)
    const uint32_t tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t g = lane >> 2, t4 = lane & 3;
    const uint32_t wm0 = (warp / WN) * 32, wn0 = (warp % WN) * (8 * NT);
    const uint32_t tiles_i = (m + kUpdTile - 1) / kUpdTile;
    if (t_begin >= t_end)
        return;
    auto coords = [&](uint32_t t, uint32_t& i0, uint32_t& j0, uint32_t& me, uint32_t& ne) {
        i0 = (t % tiles_i) * kUpdTile;
        j0 = (t / tiles_i) * kUpdTile;
        me = min((uint32_t)kUpdTile, m - i0);
        ne = min((uint32_t)kUpdTile, nn - j0);
    };
    // tile t's A block (rows of C, the panel's columns) and C block into ring slot `buf`
    auto stage_ac = [&](uint32_t t, int buf) {
        uint32_t i0, j0, me, ne;
        coords(t, i0, j0, me, ne);
        stage_tile<kUpdTile, K, VEC, kUpdThreads>(s.a[buf], Cm, ld, row0 + i0, row0 + i0 + me, a_col, a_col + K, tid);
        stage_tile<kUpdTile, kUpdTile, VEC, kUpdThreads>(s.c[buf], Cm, ld, row0 + i0, row0 + i0 + me, col0 + j0,
                                                         col0 + j0 + ne, tid);
    };
    auto stage_b = [&](uint32_t t) {
        uint32_t i0, j0, me, ne;
        coords(t, i0, j0, me, ne);
        stage_cols<kUpdTile, VEC, kUpdThreads>(s.b, Cm, ld, b_row, col0 + j0, col0 + j0 + ne, tid);
    };
    auto commit = [] { asm volatile("cp.async.commit_group;" ::: "memory"); };
    // prologue: {B, A/C of the first tile}, {A/C of the second} -- one commit group each
    stage_b(t_begin);
    stage_ac(t_begin, 0);
    commit();
    if (t_begin + 1 < t_end)
        stage_ac(t_begin + 1, 1);
    commit();
    bool b_new = false;  // the most recent group holds a new B block
    for (uint32_t t = t_begin; t < t_end; ++t) {
        const int cur = (int)((t - t_begin) & 1u);
        // this tile's group is the second most recent, unless the most recent one holds its B
        if (b_new)
            asm volatile("cp.async.wait_group 0;" ::: "memory");
        else
            asm volatile("cp.async.wait_group 1;" ::: "memory");
        __syncthreads();
        uint32_t i0, j0, me, ne;
        coords(t, i0, j0, me, ne);
        double acc[MT][NT][4];
        const double* cs = s.c[cur];
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < NT; ++j)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const uint32_t row = wm0 + 16 * i + g + 8 * h, col = wn0 + 8 * j + 2 * t4;
                    const double2 v = *reinterpret_cast<const double2*>(cs + row * kPad + col);
                    acc[i][j][2 * h] = -v.x;  // rows / columns outside the block: never stored
                    acc[i][j][2 * h + 1] = -v.y;
                }
        const double* as = s.a[cur];
#pragma unroll
        for (int k0 = 0; k0 < K; k0 += 8) {
            double af[MT][4], bf[NT][2];
#pragma unroll
            for (int i = 0; i < MT; ++i) {
                const double* p = as + (wm0 + 16 * i + g) * kPad + k0 + t4;
                af[i][0] = p[0];
                af[i][1] = p[8 * kPad];
                af[i][2] = p[4];
                af[i][3] = p[8 * kPad + 4];
            }
#pragma unroll
            for (int j = 0; j < NT; ++j) {
                const double* p = s.b + (k0 + t4) * kPad + wn0 + 8 * j + g;
                bf[j][0] = p[0];
                bf[j][1] = p[4 * kPad];
            }
#pragma unroll
            for (int i = 0; i < MT; ++i)
#pragma unroll
                for (int j = 0; j < NT; ++j)
                    mma16x8x8(acc[i][j], af[i], bf[j]);
        }
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
            for (int j = 0; j < NT; ++j) {
                const uint32_t col = wn0 + 8 * j + 2 * t4;
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const uint32_t row = wm0 + 16 * i + g + 8 * h;
                    if (row >= me)
                        continue;
                    double* cp = Cm + (size_t)(row0 + i0 + row) * ld + col0 + j0 + col;
                    const double v0 = -acc[i][j][2 * h], v1 = -acc[i][j][2 * h + 1];
                    if (VEC && col + 1 < ne) {
                        *reinterpret_cast<double2*>(cp) = make_double2(v0, v1);
                    } else {
                        if (col < ne)
                            cp[0] = v0;
                        if (col + 1 < ne)
                            cp[1] = v1;
                    }
                }
            }
        __syncthreads();  // slot `cur` (and B, if the next tile starts a column) may be refilled
        b_new = t + 1 < t_end && (t + 1) / tiles_i != t / tiles_i;
        if (b_new)
            stage_b(t + 1);
        if (t + 2 < t_end)
            stage_ac(t + 2, cur);
        commit();
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");  // nothing in flight when the CTA exits
}

}  // namespace dmma
}  // namespace pvl
