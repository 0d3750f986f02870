// Shared device helpers for the pyvl_b200 CUDA kernels (sm_100a).
//
// Geometry ids follow the reference's geo_id_t (src/core/common.h:46-56): low 31 bits
// index, bit 31 = reversed orientation, INVALID_ID = 0x7FFFFFFF.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "pvl_status.h"

#define PVL_IDX(g) ((g) & 0x7FFFFFFFu)
#define PVL_REV(g) ((g) >> 31)
#define PVL_INVALID 0x7FFFFFFFu

namespace pvl {

// One vortex segment prepared for pair evaluation: start point r1, unit direction
// d = (r2 - r1)/len, length and its square, the segment circulation gamma and glen = gamma * len
// (the end point itself is never needed: dr2 = dr1 - len d).
// A segment shorter than the cut-off radius contributes nothing (src/core/flow_solver.c:107-112):
// it is stored with d = 0 and len = 0, so every point sees h^2 = |dr1 x d|^2 = 0 below the
// cut-off and skips it without a separate test.
template <typename T>
struct __align__(16) Segment {
    T r1x, r1y, r1z;
    T len2, pad0, pad1;
    T dx, dy, dz;
    T len;
    T gamma;
    T glen;
};

// Squared cut-off radius as the kernels compare it: tol^2, but at least the smallest normal
// number, so that a disabled segment (h^2 = 0 exactly) is skipped even for tol = 0.
template <typename T>
__host__ __device__ inline T cutoff2(double tol)
{
    const double t2 = tol * tol;
    const double lo = sizeof(T) == sizeof(float) ? 1.1754943508222875e-38 : 2.2250738585072014e-308;
    return T(t2 > lo ? t2 : lo);
}

template <typename T> struct Vec3 { T x, y, z; };

// Far-field evaluation of ang / h (see segment_induction).  For x = h^2 + t1 t2 > 0 the angle
// is atan(z) with z = -h len / x, and the Taylor series of the arctangent,
//   atan(z) = z (1 - w/3 + w^2/5 - w^3/7 + ...),  w = z^2,
// gives ang / h = -(len / x) S(w) with w = h^2 len^2 / x^2 -- no square root and no atan2.
// The series is used only for w <= kW, where the first omitted term bounds the relative
// truncation error: double, 16 terms for w <= 0.1 (0.1^16 / 33 < 4e-18), 8 terms for
// w <= 0.01 (0.01^8 / 17 < 1e-17) and 4 terms for w <= 1e-4 (1e-16 / 9 < 1.2e-17); float,
// 5 terms for w <= 0.04 (0.04^5 / 11 < 1e-8).
// Closer pairs (larger w, or x <= 0) take the atan2 form.
// Comparisons of non-negative values (or +NaN) through their bit patterns: for IEEE numbers of
// one sign, the order of the bit patterns is the order of the values, and the integer compare
// runs on the ALU pipe instead of the FP64 pipe that bounds the FP64 sweeps.  lt_nn(a, b):
// a < b, exactly (the cut-off).
__device__ __forceinline__ bool lt_nn(double a, double b) { return __double_as_longlong(a) < __double_as_longlong(b); }
// Threshold tests that only choose between two evaluations that are both accurate near the
// threshold (far-field series or atan2, which series tier) compare the high 32 bits (sign,
// exponent, 20 mantissa bits): one integer compare instead of two.  A value above the threshold
// by less than 2^-20 of it may take the series tier meant for the threshold, whose truncation
// bound then grows by less than 2e-5 of itself (still below 1.2e-17).  The cut-off test stays
// exact (lt_nn).  pos_hi(x): x > +0 with at least one bit in the high word (a smaller positive
// x takes the atan2 form; a +NaN counts as positive and then fails the far-field test).
__device__ __forceinline__ int hi32(double a) { return (int)(__double_as_longlong(a) >> 32); }
__device__ __forceinline__ bool le_hi(double a, double b) { return hi32(a) <= hi32(b); }
__device__ __forceinline__ bool pos_hi(double x) { return hi32(x) > 0; }
__device__ __forceinline__ bool le_hi(float a, float b) { return a <= b; }
__device__ __forceinline__ bool pos_hi(float x) { return x > 0.0f; }
__device__ __forceinline__ bool lt_nn(float a, float b) { return a < b; }

template <typename T> struct FarSeries;
template <> struct FarSeries<double> {
    static constexpr double kW = 0.1;
    // 1/x from the hardware's approximate reciprocal r (rcp.approx.ftz.f64: 20 significant
    // bits, relative error d below 2^-19) by one third-order step of the geometric series
    // 1/x = r / (1 - e), e = 1 - x r = d:  r <- r + r (e + e^2) = (1/x)(1 - d^3), so the
    // error drops to d^3 < 2^-57 before the final rounding (within an ulp of the rounded
    // quotient, like two Newton steps, with three FMAs instead of four).  Used only where x is
    // a positive normal number; a zero, negative, huge or NaN x gives a value that the
    // far-field test rejects, after which the atan2 form is taken.
    static __device__ __forceinline__ double rcp(double x)
    {
        double r;
        asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
        const double e = fma(-x, r, 1.0);
        return fma(r, fma(e, e, e), r);
    }
    static __device__ __forceinline__ double sum(double w)
    {
        double s;
        if (le_hi(w, 1e-4)) {  // most pairs of a wake sweep: four terms, 1e-4^4 / 9 < 1.2e-17
            s = -1.0 / 7.0;
            s = fma(s, w, 1.0 / 5.0);
            s = fma(s, w, -1.0 / 3.0);
            return fma(s, w, 1.0);
        } else if (le_hi(w, 0.01)) {  // eight terms: 0.01^8 / 17 < 1e-17
            s = -1.0 / 15.0;
            s = fma(s, w, 1.0 / 13.0);
            s = fma(s, w, -1.0 / 11.0);
            s = fma(s, w, 1.0 / 9.0);
        } else {  // sixteen terms for w <= 0.1: 0.1^16 / 33 < 4e-18 (pairs 3 to 10 lengths away)
            s = -1.0 / 31.0;
            s = fma(s, w, 1.0 / 29.0);
            s = fma(s, w, -1.0 / 27.0);
            s = fma(s, w, 1.0 / 25.0);
            s = fma(s, w, -1.0 / 23.0);
            s = fma(s, w, 1.0 / 21.0);
            s = fma(s, w, -1.0 / 19.0);
            s = fma(s, w, 1.0 / 17.0);
            s = fma(s, w, -1.0 / 15.0);
            s = fma(s, w, 1.0 / 13.0);
            s = fma(s, w, -1.0 / 11.0);
            s = fma(s, w, 1.0 / 9.0);
        }
        s = fma(s, w, -1.0 / 7.0);
        s = fma(s, w, 1.0 / 5.0);
        s = fma(s, w, -1.0 / 3.0);
        return fma(s, w, 1.0);
    }
    // The same series with the tier voted over the lanes that call it together: each lane
    // gets at least the terms it needs, and the warp runs one tier instead of up to three
    // (kernels whose lanes hold different segments at one point, at spread-out distances).
    static __device__ __forceinline__ double sum_uniform(double w)
    {
        const unsigned m = __activemask();
        if (__any_sync(m, !le_hi(w, 0.01)))
            return sum_tier<16>(w);
        if (__any_sync(m, !le_hi(w, 1e-4)))
            return sum_tier<8>(w);
        return sum_tier<4>(w);
    }
    // sum_{k < N} (-w)^k / (2k + 1) by Horner's rule (the tiers of sum(), without the branches)
    template <int N> static __device__ __forceinline__ double sum_tier(double w)
    {
        double s = ((N - 1) % 2 ? -1.0 : 1.0) / (2 * N - 1);
#pragma unroll
        for (int k = N - 2; k >= 0; --k)
            s = fma(s, w, (k % 2 ? -1.0 : 1.0) / (2 * k + 1));
        return s;
    }
};
template <> struct FarSeries<float> {
    static constexpr float kW = 0.04f;
    // CUDA's fast division (about 2 ulp): the FP32 path's own rounding is of that order
    static __device__ __forceinline__ float rcp(float x) { return __fdividef(1.0f, x); }
    static __device__ __forceinline__ float sum(float w)  // five terms: 0.04^5 / 11 < 1e-8
    {
        float s = 1.0f / 9.0f;
        s = fmaf(s, w, -1.0f / 7.0f);
        s = fmaf(s, w, 1.0f / 5.0f);
        s = fmaf(s, w, -1.0f / 3.0f);
        return fmaf(s, w, 1.0f);
    }
    static __device__ __forceinline__ float sum_uniform(float w) { return sum(w); }
};

// Induction of one straight segment at point p, scaled by `scale`, added to `acc`.
//
// Follows the reference kernel (compute_line_induction, src/core/flow_solver.c:113-135):
//   dr_k = p - r_k, t_k = d.dr_k, h^2 = ((|dr1|^2 - t1^2) + (|dr2|^2 - t2^2)) / 2,
//   zero if h^2 < tol^2, else u = (dr1 x d) * (atan2(t2, h) - atan2(t1, h)) / h.
// Three exact identities of that formula are used:
//   * dr2 = dr1 - len d, so t2 = t1 - len, and both perpendicular distances equal
//     |dr1 x d|: h^2 = |c|^2 with c = dr1 x d, the vector the result points along anyway
//     (no cancellation of |dr|^2 - t^2 for points near the segment's line);
//   * for h > 0, atan2(t2, h) - atan2(t1, h) = atan2(h (t2 - t1), h^2 + t1 t2)
//     = atan2(-h len, h^2 + t1 t2), one atan2 without the far-field cancellation of two;
//   * far pairs evaluate ang / h by the arctangent series of FarSeries (no sqrt, no atan2).
// GAMMA: the scale is the segment's own circulation (sweeps), so that gamma * len comes
// precomputed from the table; otherwise `scale` (ring sums: +-1).
// UNIFORM: the series tier is voted over the warp (FarSeries::sum_uniform).
template <typename T, bool GAMMA = false, bool UNIFORM = false>
__device__ __forceinline__ void segment_induction(const Segment<T>& s, T px, T py, T pz, T tol2, T scale,
                                                  Vec3<T>& acc)
{
    const T ax = px - s.r1x, ay = py - s.r1y, az = pz - s.r1z;
    const T t1 = s.dx * ax + s.dy * ay + s.dz * az;
    const T cx = ay * s.dz - az * s.dy, cy = az * s.dx - ax * s.dz, cz = ax * s.dy - ay * s.dx;
    const T hsq = cx * cx + cy * cy + cz * cz;  // >= +0
    if (lt_nn(hsq, tol2))
        return;
    const T x = hsq + t1 * (t1 - s.len);
    const T r = FarSeries<T>::rcp(x);  // wasted only on the rare near pairs
    const T w = hsq * s.len2 * (r * r);  // >= +0, or +NaN
    T mag;
    if (pos_hi(x) && le_hi(w, FarSeries<T>::kW)) {
        const T S = UNIFORM ? FarSeries<T>::sum_uniform(w) : FarSeries<T>::sum(w);
        mag = (GAMMA ? -s.glen : -scale * s.len) * r * S;
    } else {
        // one reciprocal square root gives both h and 1/h (no separate sqrt and division)
        const T rh = rsqrt(hsq);
        const T h = hsq * rh;
        const T ang = atan2(-h * s.len, x);
        mag = (GAMMA ? s.gamma : scale) * ang * rh;
    }
    acc.x += cx * mag;
    acc.y += cy * mag;
    acc.z += cz * mag;
}

// The segments of one ring (its entries k0 .. k1 of the ring -> line CSR) held in registers,
// so that a thread evaluating the ring at many control points loads them once.  Rings of up
// to kMax lines are cached (quads and triangles); larger rings fall back to loading per point.
template <typename T>
struct RingSegments {
    static constexpr int kMax = 4;
    Segment<T> s[kMax];
    T sign[kMax];
    uint32_t k0, k1;
    bool cached;

    __device__ __forceinline__ void load(const uint32_t* __restrict__ sl, uint32_t k0_, uint32_t k1_,
                                         uint32_t n_lines, const Segment<T>* __restrict__ seg)
    {
        k0 = k0_;
        k1 = k1_;
        cached = k1 - k0 <= (uint32_t)kMax;
#pragma unroll
        for (int q = 0; q < kMax; ++q) {
            const uint32_t k = k0 + q;
            bool ok = cached && k < k1;
            uint32_t g = ok ? sl[k] : 0u;
            const uint32_t l = PVL_IDX(g);
            ok = ok && l < n_lines;
            if (ok) {
                s[q] = seg[l];
            } else {  // an empty slot: d = 0 gives h^2 = 0, below any cut-off
                s[q].r1x = s[q].r1y = s[q].r1z = s[q].dx = s[q].dy = s[q].dz = T(0);
                s[q].len = s[q].len2 = s[q].gamma = s[q].glen = T(0);
                s[q].pad0 = s[q].pad1 = T(0);
            }
            sign[q] = PVL_REV(g) ? T(-1) : T(1);
        }
    }

    // sum over the ring's lines of +-u_k(p), in CSR order (the reference's order)
    __device__ __forceinline__ Vec3<T> sum(const uint32_t* __restrict__ sl, uint32_t n_lines,
                                           const Segment<T>* __restrict__ seg, T px, T py, T pz, T tol2) const
    {
        Vec3<T> acc{T(0), T(0), T(0)};
        if (cached) {
#pragma unroll
            for (int q = 0; q < kMax; ++q)
                segment_induction(s[q], px, py, pz, tol2, sign[q], acc);
        } else {
            for (uint32_t k = k0; k < k1; ++k) {
                const uint32_t g = sl[k];
                const uint32_t l = PVL_IDX(g);
                if (l >= n_lines)
                    continue;
                segment_induction(seg[l], px, py, pz, tol2, PVL_REV(g) ? T(-1) : T(1), acc);
            }
        }
        return acc;
    }
};

// The signed entries of one ring in its tile's line list (tiled ring kernels), held in
// registers for rings of up to kMax lines (quads and triangles), so that summing the ring at
// every control point of a CTA reads its CSR entries once; larger rings read them per point.
// sum() adds +-row[e] in CSR order (the reference's order); an entry at or past `stride` adds 0.
struct RingEntries {
    static constexpr int kMax = 4;
    uint32_t e[kMax];
    bool neg[kMax];
    uint32_t k0, k1;

    __device__ __forceinline__ void load(const uint32_t* __restrict__ sl, const uint32_t* __restrict__ sl_local,
                                         uint32_t k0_, uint32_t k1_)
    {
        k0 = k0_;
        k1 = k1_;
#pragma unroll
        for (int u = 0; u < kMax; ++u) {
            const bool ok = k1 - k0 <= (uint32_t)kMax && k0 + u < k1;
            e[u] = ok ? sl_local[k0 + u] : 0u;
            neg[u] = ok ? PVL_REV(sl[k0 + u]) != 0 : false;
        }
    }

    __device__ __forceinline__ double sum(const double* __restrict__ row, uint32_t stride,
                                          const uint32_t* __restrict__ sl, const uint32_t* __restrict__ sl_local) const
    {
        double v = 0.0;
        if (k1 - k0 <= (uint32_t)kMax) {
#pragma unroll
            for (int u = 0; u < kMax; ++u) {
                if (k0 + u < k1) {
                    const double x = e[u] < stride ? row[e[u]] : 0.0;
                    v += neg[u] ? -x : x;
                }
            }
        } else {
            for (uint32_t k = k0; k < k1; ++k) {
                const uint32_t ek = sl_local[k];
                const double x = ek < stride ? row[ek] : 0.0;
                v += PVL_REV(sl[k]) ? -x : x;
            }
        }
        return v;
    }
};

}  // namespace pvl

#define PVL_CUDA_CHECK(expr)                                                                   \
    do {                                                                                       \
        cudaError_t _e = (expr);                                                               \
        if (_e != cudaSuccess)                                                                 \
            return pvl_fail(PVL_ERR_CUDA, "%s:%d %s: %s", __FILE__, __LINE__, #expr,           \
                            cudaGetErrorString(_e));                                           \
    } while (0)

// Every kernel launch site is followed by PVL_LAUNCH_CHECK(), which also counts the launch.
void pvl_count_launch();
#define PVL_LAUNCH_CHECK()                   \
    do {                                     \
        pvl_count_launch();                  \
        PVL_CUDA_CHECK(cudaGetLastError());  \
    } while (0)
