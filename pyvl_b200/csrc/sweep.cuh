// Pair arithmetic of the FP64 N-body sweep (line_sum_f64_kernel), sm_100a.
//
// The quantities of segment_induction (pvl_common.cuh) in Pluecker form about an origin o
// that the CTA chooses (the centroid of its points): a segment is staged once per CTA as
//   d (unit direction), m = (r1 - o) x d, e = d . (r1 - o), len, gamma len, gamma
// (80 bytes, five 16-byte shared loads per pair; gamma is read only by the near pairs), and
// for a point p' = p - o
//   t1 = d . p' - e = d . (p - r1),   c = p' x d - m = (p - r1) x d
// from 9 FMAs instead of 3 differences and 9 products per pair.  Rounding is relative to
// |p - o| + |r1 - o| instead of |p - r1|; the points of one CTA are neighbours (ring or
// wake-node order, or one case of a batch), so |p - o| stays of the order of the body.
// Everything after c and t1 -- h^2, x = h^2 + t1 t2, the far-field series with the Newton
// reciprocal, the atan2 form for near pairs, the cut-off -- is segment_induction<double, true>,
// with w = h^2 len^2 / x^2 formed as h^2 (len / x)^2.
#pragma once

#include <cstdint>

#include "pvl_common.cuh"

namespace pvl {

struct __align__(16) SweepSeg {
    double dx, dy, dz, mx, my, mz, e, len, glen, gamma;
};

struct SweepGeo {
    double cx, cy, cz, hsq, x, r, w;
};

// The segment g about origin o (o[0..2], usually in shared memory).
__device__ __forceinline__ SweepSeg sweep_seg(const Segment<double>& g, const double* o)
{
    const double rx = g.r1x - o[0], ry = g.r1y - o[1], rz = g.r1z - o[2];
    SweepSeg t;
    t.dx = g.dx;
    t.dy = g.dy;
    t.dz = g.dz;
    t.mx = ry * g.dz - rz * g.dy;
    t.my = rz * g.dx - rx * g.dz;
    t.mz = rx * g.dy - ry * g.dx;
    t.e = g.dx * rx + g.dy * ry + g.dz * rz;
    t.len = g.len;
    t.glen = g.glen;
    t.gamma = g.gamma;
    return t;
}

__device__ __forceinline__ SweepGeo sweep_geo(const SweepSeg& s, double px, double py, double pz)
{
    SweepGeo g;
    const double t1 = fma(s.dz, pz, fma(s.dy, py, fma(s.dx, px, -s.e)));
    g.cx = fma(py, s.dz, -fma(pz, s.dy, s.mx));
    g.cy = fma(pz, s.dx, -fma(px, s.dz, s.my));
    g.cz = fma(px, s.dy, -fma(py, s.dx, s.mz));
    g.hsq = g.cx * g.cx + g.cy * g.cy + g.cz * g.cz;
    g.x = g.hsq + t1 * (t1 - s.len);
    g.r = FarSeries<double>::rcp(g.x);
    const double a = s.len * g.r;
    g.w = g.hsq * (a * a);
    return g;
}

// Far pairs by the arctangent series (selected, no branch), the rare near pairs by atan2 in a
// branch, pairs inside the cut-off skipped; gamma_k u_k(p) added to acc.
__device__ __forceinline__ void sweep_add(const SweepSeg& s, const SweepGeo& g, double tol2, Vec3<double>& acc)
{
    const bool ok = !lt_nn(g.hsq, tol2);
    const bool far = ok && pos_hi(g.x) && le_hi(g.w, FarSeries<double>::kW);
    double mag = far ? -s.glen * g.r * FarSeries<double>::sum(g.w) : 0.0;
    if (ok && !far) {
        const double rh = rsqrt(g.hsq);
        const double h = g.hsq * rh;
        mag = s.gamma * atan2(-h * s.len, g.x) * rh;
    }
    acc.x += g.cx * mag;
    acc.y += g.cy * mag;
    acc.z += g.cz * mag;
}

// o = centroid of the CTA's valid points (0 if none), in fixed summation order, from each
// thread's sum of its valid points (sx, sy, sz) and their count n; every thread of the CTA
// must call it.  red: THREADS / 32 x 4 doubles of shared memory, o: 3.
template <int THREADS>
__device__ __forceinline__ void cta_centroid(double sx, double sy, double sz, double n, double (*red)[4], double* o)
{
    double v[4] = {sx, sy, sz, n};
#pragma unroll
    for (int c = 0; c < 4; ++c)
        for (int k = 16; k > 0; k >>= 1)
            v[c] += __shfl_xor_sync(0xffffffffu, v[c], k);
    if ((threadIdx.x & 31) == 0)
#pragma unroll
        for (int c = 0; c < 4; ++c)
            red[threadIdx.x >> 5][c] = v[c];
    __syncthreads();
    if (threadIdx.x < 3) {
        double t = 0.0, n = 0.0;
        for (int w = 0; w < THREADS / 32; ++w) {
            t += red[w][threadIdx.x];
            n += red[w][3];
        }
        o[threadIdx.x] = n > 0.0 ? t / n : 0.0;
    }
    __syncthreads();
}

}  // namespace pvl
