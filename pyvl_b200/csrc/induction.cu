// Segment -> point induction kernels for sm_100a.
//
// The reference evaluates every (line, point) pair into a 24 B/pair line buffer and then
// reduces it per ring (src/core/flow_solver.c:86-205).  Here no line buffer exists:
//  * ring matrices (normal or vector) evaluate each ring's segments in the thread that
//    owns the (point, ring) entry and store the entry once, coalesced along the row;
//  * contractions with circulations (velocities, the explicit wake term) become an
//    N-body sweep: points live in registers, segments stream through shared memory in
//    tiles, each segment carries its line circulation, and partial sums over segment
//    ranges are reduced deterministically in a second pass.
// All pair arithmetic is pvl::segment_induction (pvl_common.cuh).
#include <algorithm>
#include <cstdint>

#include "pvl_common.cuh"
#include "sweep.cuh"

using pvl::Segment;
using pvl::SweepSeg;
using pvl::Vec3;

namespace {

constexpr int kSegTile = 128;   // segments per shared-memory tile
constexpr int kReducePts = 16;     // points per CTA of the partial-sum reduction (256 CTAs at 4096)
constexpr int kReduceGroups = 16;  // rows of threads (split groups) per CTA
constexpr int kSumThreads = 128;
constexpr int kRingThreads = 128;
constexpr int kRingCPB = 8;     // control points per CTA row-block in ring matrices

inline size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

template <typename T>
__global__ void prep_segments_kernel(uint32_t n_points, uint32_t n_lines, const uint32_t* __restrict__ lines,
                                     const double* __restrict__ pos, const double* __restrict__ line_gamma,
                                     double tol, Segment<T>* __restrict__ seg)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_lines)
        return;
    const uint32_t a = PVL_IDX(lines[2 * i]), b = PVL_IDX(lines[2 * i + 1]);
    Segment<T> s;
    if (a >= n_points || b >= n_points) {
        s.r1x = s.r1y = s.r1z = s.len2 = s.pad0 = s.pad1 = s.dx = s.dy = s.dz = T(0);
        s.len = s.gamma = s.glen = T(0);
        seg[i] = s;
        return;
    }
    const double r1x = pos[3 * (size_t)a], r1y = pos[3 * (size_t)a + 1], r1z = pos[3 * (size_t)a + 2];
    const double r2x = pos[3 * (size_t)b], r2y = pos[3 * (size_t)b + 1], r2z = pos[3 * (size_t)b + 2];
    double dx = r2x - r1x, dy = r2y - r1y, dz = r2z - r1z;
    double len = sqrt(dx * dx + dy * dy + dz * dz);
    if (len < tol) {
        // src/core/flow_solver.c:107-112: a segment shorter than tol induces nothing (d = 0, len = 0:
        // every point then has h^2 = 0, below the cut-off)
        dx = dy = dz = 0.0;
        len = 0.0;
    } else {
        dx /= len;
        dy /= len;
        dz /= len;
    }
    s.r1x = T(r1x);
    s.r1y = T(r1y);
    s.r1z = T(r1z);
    s.len2 = T(len * len);
    s.pad0 = T(0);
    s.pad1 = T(0);
    s.dx = T(dx);
    s.dy = T(dy);
    s.dz = T(dz);
    s.len = T(len);
    const double g = line_gamma ? line_gamma[i] : 1.0;
    s.gamma = T(g);
    s.glen = T(g * len);
    seg[i] = s;
}

template <typename T, typename OutT, int MODE>
__global__ void __launch_bounds__(kRingThreads) ring_matrix_kernel(
    uint32_t n_surfaces, const uint32_t* __restrict__ off, const uint32_t* __restrict__ sl, uint32_t n_lines,
    const Segment<T>* __restrict__ seg, uint32_t n_cp, const double* __restrict__ cps,
    const double* __restrict__ normals, T tol2, OutT* __restrict__ out, uint32_t ld)
{
    __shared__ T s_p[kRingCPB][3];
    __shared__ T s_n[kRingCPB][3];
    const uint32_t i0 = blockIdx.y * kRingCPB;
    if (threadIdx.x < kRingCPB * 3) {
        const uint32_t c = threadIdx.x / 3, e = threadIdx.x % 3;
        const uint32_t i = i0 + c;
        s_p[c][e] = i < n_cp ? T(cps[3 * (size_t)i + e]) : T(0);
        s_n[c][e] = (MODE == 0 && i < n_cp) ? T(normals[3 * (size_t)i + e]) : T(0);
    }
    __syncthreads();
    const uint32_t j = blockIdx.x * kRingThreads + threadIdx.x;
    if (j >= n_surfaces)
        return;
    pvl::RingSegments<T> rs;
    rs.load(sl, off[j], off[j + 1], n_lines, seg);
#pragma unroll 1
    for (int c = 0; c < kRingCPB; ++c) {
        const uint32_t i = i0 + c;
        if (i >= n_cp)
            break;
        const Vec3<T> v = rs.sum(sl, n_lines, seg, s_p[c][0], s_p[c][1], s_p[c][2], tol2);
        if (MODE == 0) {
            out[(size_t)i * ld + j] = OutT(v.x * s_n[c][0] + v.y * s_n[c][1] + v.z * s_n[c][2]);
        } else {
            OutT* o = out + 3 * ((size_t)i * n_surfaces + j);
            o[0] = OutT(v.x);
            o[1] = OutT(v.y);
            o[2] = OutT(v.z);
        }
    }
}

// Ring-matrix rows with each line evaluated once per control point: rings are taken in tiles
// of kRingTile consecutive rings; a CTA evaluates n_i . u_l(cp_i) for the distinct lines of
// its tile (tile_lines[tile_offsets[t] ..]) at its CPB control points into shared memory,
// then each thread sums its ring's signed entries (sl_local: each CSR entry's position in its
// tile's line list) in CSR order.  Adjacent rings share lines, so a structured wing needs
// ~0.57 line evaluations per (point, ring line) instead of one.  The CTA has THREADS >=
// kRingTile threads (chosen per launch from the largest tile's line count, so that the line
// loop's last round is not mostly idle: 292 lines take two rounds of 160 threads instead of
// three of 128); the first kRingTile of them sum the rings.
constexpr int kRingTile = 128;
constexpr int kTileCPB = 8;   // control points per CTA (8: 231 us, 16: 272 us on the 4096-ring body)

template <int THREADS>
__global__ void __launch_bounds__(THREADS) ring_tile_kernel(uint32_t n_surfaces, const uint32_t* __restrict__ off,
                                                              const uint32_t* __restrict__ sl,
                                                              const uint32_t* __restrict__ sl_local,
                                                              const uint32_t* __restrict__ tile_off,
                                                              const uint32_t* __restrict__ tile_lines,
                                                              uint32_t tile_stride, uint32_t n_lines,
                                                              const Segment<double>* __restrict__ seg, uint32_t n_cp,
                                                              const double* __restrict__ cps,
                                                              const double* __restrict__ normals, double tol2,
                                                              double* __restrict__ out, uint32_t ld)
{
    extern __shared__ double sV[];  // [kTileCPB][tile_stride]
    __shared__ double s_p[kTileCPB][3], s_n[kTileCPB][3];
    const uint32_t tile = blockIdx.x, i0 = blockIdx.y * kTileCPB;
    if (threadIdx.x < kTileCPB * 3) {
        const uint32_t c = threadIdx.x / 3, e = threadIdx.x % 3;
        const bool ok = i0 + c < n_cp;
        s_p[c][e] = ok ? cps[3 * (size_t)(i0 + c) + e] : 0.0;
        s_n[c][e] = ok ? normals[3 * (size_t)(i0 + c) + e] : 0.0;
    }
    __syncthreads();
    const uint32_t L0 = tile_off[tile], nl = tile_off[tile + 1] - L0;
    for (uint32_t l = threadIdx.x; l < nl; l += THREADS) {
        const uint32_t g = tile_lines[L0 + l];
        const bool ok = g < n_lines;
        Segment<double> sg;
        if (ok) {
            sg = seg[g];
        } else {
            sg.r1x = sg.r1y = sg.r1z = sg.dx = sg.dy = sg.dz = 0.0;
            sg.len = sg.len2 = sg.gamma = sg.glen = sg.pad0 = sg.pad1 = 0.0;
        }
#pragma unroll  // all 8 control points: 232 vs 236 us for the body (unroll 4), no spills
        for (int q = 0; q < kTileCPB; ++q) {
            Vec3<double> acc{0.0, 0.0, 0.0};
            pvl::segment_induction<double, false, true>(sg, s_p[q][0], s_p[q][1], s_p[q][2], tol2, 1.0, acc);
            sV[q * tile_stride + l] = acc.x * s_n[q][0] + acc.y * s_n[q][1] + acc.z * s_n[q][2];
        }
    }
    __syncthreads();
    const uint32_t j = tile * kRingTile + threadIdx.x;
    if (threadIdx.x >= kRingTile || j >= n_surfaces)
        return;
    pvl::RingEntries re;
    re.load(sl, sl_local, off[j], off[j + 1]);
    for (int q = 0; q < kTileCPB; ++q) {
        if (i0 + q >= n_cp)
            break;
        out[(size_t)(i0 + q) * ld + j] = re.sum(sV + q * tile_stride, tile_stride, sl, sl_local);
    }
}

// out[(i*n_lines + l)*3 + c] = u_l(cp_i)
__global__ void __launch_bounds__(kRingThreads) line_matrix_kernel(uint32_t n_lines,
                                                                   const Segment<double>* __restrict__ seg,
                                                                   uint32_t n_cp, const double* __restrict__ cps,
                                                                   double tol2, double* __restrict__ out)
{
    __shared__ double s_p[kRingCPB][3];
    const uint32_t i0 = blockIdx.y * kRingCPB;
    if (threadIdx.x < kRingCPB * 3) {
        const uint32_t c = threadIdx.x / 3, e = threadIdx.x % 3;
        s_p[c][e] = (i0 + c) < n_cp ? cps[3 * (size_t)(i0 + c) + e] : 0.0;
    }
    __syncthreads();
    const uint32_t l = blockIdx.x * kRingThreads + threadIdx.x;
    if (l >= n_lines)
        return;
    const Segment<double> s = seg[l];
    for (int c = 0; c < kRingCPB; ++c) {
        const uint32_t i = i0 + c;
        if (i >= n_cp)
            break;
        Vec3<double> acc{0.0, 0.0, 0.0};
        pvl::segment_induction(s, s_p[c][0], s_p[c][1], s_p[c][2], tol2, 1.0, acc);
        double* o = out + 3 * ((size_t)i * n_lines + l);
        o[0] = acc.x;
        o[1] = acc.y;
        o[2] = acc.z;
    }
}

// Point p of a sweep is pts[col(p / group) * stride + row(p % group)] with col(c) = cols ? cols[c]
// : c and row(k) = rows ? rows[k] : k * row_step + in_off: group == stride == n_pts, row_step 1
// is a plain array; group = a set of wake rows, stride = rows + 1, in_off = first row, row_step =
// the rows' spacing walks those rows of the listed wake node columns (strip side s * 2 + side);
// a row list walks any rows.  A listed column at or past col_limit, or a listed row at or past
// row_limit, is no point.
__device__ __forceinline__ bool sweep_point(uint32_t p, uint32_t n_pts, uint32_t group, uint32_t stride,
                                            uint32_t in_off, uint32_t row_step, const uint32_t* __restrict__ cols,
                                            uint32_t col_limit, const uint32_t* __restrict__ rows, uint32_t row_limit,
                                            size_t& q)
{
    bool ok = p < n_pts;
    const uint32_t col = ok ? (cols ? cols[p / group] : p / group) : 0;
    const uint32_t row = ok ? (rows ? rows[p % group] : (p % group) * row_step + in_off) : 0;
    if (col >= col_limit || (rows && row >= row_limit))
        ok = false;
    q = ok ? (size_t)col * stride + row : 0;
    return ok;
}

// FP64 N-body sweep: partial[(split*n_pts + p)*3 + c] = sum over this split's segments of
// gamma_k u_k(p).  One point per thread; segments stream through shared memory in tiles of
// kSegTile, converted to the Pluecker form about the CTA's origin as they are staged, and
// are evaluated two at a time (two independent dependency chains per thread).
__global__ void __launch_bounds__(kSumThreads, 8) line_sum_f64_kernel(
    const Segment<double>* __restrict__ seg, uint32_t n_lines, uint32_t lines_per_split,
    const double* __restrict__ pts, uint32_t n_pts, uint32_t group, uint32_t stride, uint32_t in_off,
    uint32_t row_step, const uint32_t* __restrict__ cols, uint32_t col_limit, const uint32_t* __restrict__ rows,
    uint32_t row_limit, double tol2, double* __restrict__ partial)
{
    __shared__ SweepSeg s_seg[kSegTile + 1];
    __shared__ double s_red[kSumThreads / 32][4];
    __shared__ double s_o[3];
    const uint32_t split = blockIdx.y;
    const uint32_t l_begin = split * lines_per_split;
    const uint32_t l_end = min(n_lines, l_begin + lines_per_split);
    const uint32_t p = blockIdx.x * kSumThreads + threadIdx.x;
    size_t q;
    const bool ok = sweep_point(p, n_pts, group, stride, in_off, row_step, cols, col_limit, rows, row_limit, q);
    double px = ok ? pts[3 * q] : 0.0, py = ok ? pts[3 * q + 1] : 0.0, pz = ok ? pts[3 * q + 2] : 0.0;
    pvl::cta_centroid<kSumThreads>(px, py, pz, ok ? 1.0 : 0.0, s_red, s_o);  // px.. are 0 when !ok
    px -= s_o[0];
    py -= s_o[1];
    pz -= s_o[2];
    Vec3<double> acc{0.0, 0.0, 0.0};
    if (threadIdx.x == 0)
        s_seg[kSegTile] = SweepSeg{};  // the partner of an odd last segment: d = 0, nothing induced
    for (uint32_t l0 = l_begin; l0 < l_end; l0 += kSegTile) {
        const uint32_t l = l0 + threadIdx.x;
        const SweepSeg t = threadIdx.x < kSegTile && l < l_end ? pvl::sweep_seg(seg[l], s_o) : SweepSeg{};
        if (threadIdx.x < kSegTile)
            s_seg[threadIdx.x] = t;
        __syncthreads();
        const int cnt = (int)min((uint32_t)kSegTile, l_end - l0);
#pragma unroll 1
        for (int k = 0; k < cnt; k += 2) {
            const SweepSeg a = s_seg[k], b = s_seg[k + 1];
            const pvl::SweepGeo ga = pvl::sweep_geo(a, px, py, pz), gb = pvl::sweep_geo(b, px, py, pz);
            pvl::sweep_add(a, ga, tol2, acc);
            pvl::sweep_add(b, gb, tol2, acc);
        }
        __syncthreads();
    }
    if (p < n_pts) {
        double* o = partial + 3 * ((size_t)split * n_pts + p);
        o[0] = acc.x;
        o[1] = acc.y;
        o[2] = acc.z;
    }
}

// The FP32 sweep with Blackwell's packed FP32x2 arithmetic (__ffma2_rn / __fadd2_rn /
// __fmul2_rn): each thread evaluates every segment at two points held in the two lanes of
// float2 registers, so one instruction serves two pairs.  The pair arithmetic is the Pluecker
// form of sweep.cuh about the CTA's centroid o (t1 = d . p' - e, c = p' x d - m, p' = p - o;
// m and e formed in FP64 when the tile is staged; -d, -m, -e, -len and -gamma len staged too,
// so that no operand is negated in the loop): 26 packed instructions per two pairs on the FMA
// pipe, which bounds this kernel.  (Staging every operand already broadcast to both lanes as
// float2 was slower: 112 instead of 64 bytes of shared loads per segment.)  Both lanes take
// the far-field series of segment_induction; a lane inside the cut-off contributes zero
// (selected, not computed), and a lane that needs the near-field atan2 form takes a scalar
// side path.  Same function and layout as line_sum_f64_kernel; points p and p + 128 of each
// 256-point block.  40 registers, 12 CTAs per SM (541 us; 48 registers, 10 CTAs: 547 us).
__device__ __forceinline__ float2 bc2(float a) { return make_float2(a, a); }

struct __align__(16) SweepSeg2 {
    float dx, dy, dz, ndx, ndy, ndz;  // d and -d
    float nmx, nmy, nmz, ne;          // -m and -e about the CTA's origin
    float nlen, len2, nglen;          // -len, len^2, -gamma len
    float gamma, len;                 // the near-field side path
    float pad;
};

__device__ __forceinline__ SweepSeg2 sweep_seg2(const Segment<float>& g, const double* o)
{
    const double rx = (double)g.r1x - o[0], ry = (double)g.r1y - o[1], rz = (double)g.r1z - o[2];
    const double dx = g.dx, dy = g.dy, dz = g.dz;
    SweepSeg2 t;
    t.dx = g.dx;
    t.dy = g.dy;
    t.dz = g.dz;
    t.ndx = -g.dx;
    t.ndy = -g.dy;
    t.ndz = -g.dz;
    t.nmx = (float)(rz * dy - ry * dz);
    t.nmy = (float)(rx * dz - rz * dx);
    t.nmz = (float)(ry * dx - rx * dy);
    t.ne = (float)-(dx * rx + dy * ry + dz * rz);
    t.nlen = -g.len;
    t.len2 = g.len2;
    t.nglen = -g.glen;
    t.gamma = g.gamma;
    t.len = g.len;
    t.pad = 0.0f;
    return t;
}

__global__ void __launch_bounds__(kSumThreads, 12) line_sum_f32x2_kernel(const Segment<float>* __restrict__ seg,
                                                                     uint32_t n_lines, uint32_t lines_per_split,
                                                                     const double* __restrict__ pts, uint32_t n_pts,
                                                                     uint32_t group, uint32_t stride, uint32_t in_off,
                                                                     uint32_t row_step,
                                                                     const uint32_t* __restrict__ cols,
                                                                     uint32_t col_limit,
                                                                     const uint32_t* __restrict__ rows,
                                                                     uint32_t row_limit, float tol2,
                                                                     float* __restrict__ partial)
{
    __shared__ SweepSeg2 s_seg[kSegTile];
    __shared__ double s_red[kSumThreads / 32][4];
    __shared__ double s_o[3];
    const uint32_t split = blockIdx.y;
    const uint32_t l_begin = split * lines_per_split;
    const uint32_t l_end = min(n_lines, l_begin + lines_per_split);
    double pv[2][3];
    uint32_t pid[2];
    double cs[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int t = 0; t < 2; ++t) {
        const uint32_t p = blockIdx.x * (kSumThreads * 2) + t * kSumThreads + threadIdx.x;
        pid[t] = p;
        size_t q;
        const bool ok = sweep_point(p, n_pts, group, stride, in_off, row_step, cols, col_limit, rows, row_limit, q);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            pv[t][c] = ok ? pts[3 * q + c] : 0.0;
            cs[c] += pv[t][c];
        }
        cs[3] += ok ? 1.0 : 0.0;
    }
    pvl::cta_centroid<kSumThreads>(cs[0], cs[1], cs[2], cs[3], s_red, s_o);
    const float2 px = make_float2((float)(pv[0][0] - s_o[0]), (float)(pv[1][0] - s_o[0])),
                 py = make_float2((float)(pv[0][1] - s_o[1]), (float)(pv[1][1] - s_o[1])),
                 pz = make_float2((float)(pv[0][2] - s_o[2]), (float)(pv[1][2] - s_o[2]));
    float2 accx = bc2(0.0f), accy = bc2(0.0f), accz = bc2(0.0f);
    constexpr float kW = pvl::FarSeries<float>::kW;
    for (uint32_t l0 = l_begin; l0 < l_end; l0 += kSegTile) {
        const uint32_t l = l0 + threadIdx.x;
        if (threadIdx.x < kSegTile && l < l_end)
            s_seg[threadIdx.x] = sweep_seg2(seg[l], s_o);
        __syncthreads();
        const int cnt = (int)min((uint32_t)kSegTile, l_end - l0);
#pragma unroll 1
        for (int k = 0; k < cnt; ++k) {
            const SweepSeg2 s = s_seg[k];
            float2 t1 = __ffma2_rn(bc2(s.dx), px, bc2(s.ne));
            t1 = __ffma2_rn(bc2(s.dy), py, t1);
            t1 = __ffma2_rn(bc2(s.dz), pz, t1);
            const float2 cx = __ffma2_rn(py, bc2(s.dz), __ffma2_rn(pz, bc2(s.ndy), bc2(s.nmx)));
            const float2 cy = __ffma2_rn(pz, bc2(s.dx), __ffma2_rn(px, bc2(s.ndz), bc2(s.nmy)));
            const float2 cz = __ffma2_rn(px, bc2(s.dy), __ffma2_rn(py, bc2(s.ndx), bc2(s.nmz)));
            float2 hsq = __fmul2_rn(cx, cx);
            hsq = __ffma2_rn(cy, cy, hsq);
            hsq = __ffma2_rn(cz, cz, hsq);
            const float2 x = __ffma2_rn(t1, __fadd2_rn(t1, bc2(s.nlen)), hsq);
            const float2 r = make_float2(pvl::FarSeries<float>::rcp(x.x), pvl::FarSeries<float>::rcp(x.y));
            const float2 w = __fmul2_rn(__fmul2_rn(hsq, bc2(s.len2)), __fmul2_rn(r, r));
            float2 S = bc2(1.0f / 9.0f);  // FarSeries<float>::sum, packed
            S = __ffma2_rn(S, w, bc2(-1.0f / 7.0f));
            S = __ffma2_rn(S, w, bc2(1.0f / 5.0f));
            S = __ffma2_rn(S, w, bc2(-1.0f / 3.0f));
            S = __ffma2_rn(S, w, bc2(1.0f));
            float2 mag = __fmul2_rn(__fmul2_rn(bc2(s.nglen), r), S);
            const bool cut0 = hsq.x < tol2, cut1 = hsq.y < tol2;
            const bool far0 = x.x > 0.0f && w.x <= kW, far1 = x.y > 0.0f && w.y <= kW;
            if (!(cut0 || far0) || !(cut1 || far1)) {  // rare: a lane in the near field
                if (!(cut0 || far0)) {
                    const float rh = rsqrtf(hsq.x);
                    mag.x = s.gamma * atan2f(-(hsq.x * rh) * s.len, x.x) * rh;
                }
                if (!(cut1 || far1)) {
                    const float rh = rsqrtf(hsq.y);
                    mag.y = s.gamma * atan2f(-(hsq.y * rh) * s.len, x.y) * rh;
                }
            }
            mag.x = cut0 ? 0.0f : mag.x;
            mag.y = cut1 ? 0.0f : mag.y;
            accx = __ffma2_rn(cx, mag, accx);
            accy = __ffma2_rn(cy, mag, accy);
            accz = __ffma2_rn(cz, mag, accz);
        }
        __syncthreads();
    }
    const float a[2][3] = {{accx.x, accy.x, accz.x}, {accx.y, accy.y, accz.y}};
#pragma unroll
    for (int t = 0; t < 2; ++t) {
        if (pid[t] < n_pts) {
            float* o = partial + 3 * ((size_t)split * n_pts + pid[t]);
            o[0] = a[t][0];
            o[1] = a[t][1];
            o[2] = a[t][2];
        }
    }
}

// out = beta * out + alpha * v (+ (ux, uy, uz) for vector output), v = sum of the partials.
// Point p is written at o = (p / group) * out_stride + p % group + out_off (normals are
// indexed by p: normal output is always a plain array).
template <typename T>
__global__ void __launch_bounds__(kReducePts * kReduceGroups) reduce_partials_kernel(
    uint32_t n_pts, uint32_t n_split, const T* __restrict__ partial, const double* __restrict__ normals, double alpha,
    double beta, double ux, double uy, double uz, uint32_t group, uint32_t row_step, uint32_t out_stride,
    uint32_t out_off, const uint32_t* __restrict__ rows, uint32_t row_limit,
    double* __restrict__ out)
{
    // kReducePts consecutive points per CTA (their partials are contiguous for every split, so a
    // row of threads reads them coalesced); kReduceGroups rows of threads take every
    // kReduceGroups-th split, and the rows' sums are added in row order (deterministic).
    __shared__ double s_v[kReduceGroups][kReducePts][3];
    const uint32_t tx = threadIdx.x % kReducePts, ty = threadIdx.x / kReducePts;
    const uint32_t p = blockIdx.x * kReducePts + tx;
    double vx = 0, vy = 0, vz = 0;
    if (p < n_pts) {
        for (uint32_t s = ty; s < n_split; s += kReduceGroups) {
            const T* q = partial + 3 * ((size_t)s * n_pts + p);
            vx += double(q[0]);
            vy += double(q[1]);
            vz += double(q[2]);
        }
    }
    s_v[ty][tx][0] = vx;
    s_v[ty][tx][1] = vy;
    s_v[ty][tx][2] = vz;
    __syncthreads();
    if (ty != 0 || p >= n_pts)
        return;
    for (int g = 1; g < kReduceGroups; ++g) {
        vx += s_v[g][tx][0];
        vy += s_v[g][tx][1];
        vz += s_v[g][tx][2];
    }
    const uint32_t row = rows ? rows[p % group] : (p % group) * row_step + out_off;
    if (rows && row >= row_limit)
        return;  // no point (the sweep skipped it too)
    const size_t op = (size_t)(p / group) * out_stride + row;
    if (normals) {
        const double v = vx * normals[3 * (size_t)p] + vy * normals[3 * (size_t)p + 1] + vz * normals[3 * (size_t)p + 2];
        out[p] = beta == 0.0 ? alpha * v : beta * out[p] + alpha * v;
    } else {
        double* o = out + 3 * op;
        if (beta == 0.0) {
            o[0] = ux + alpha * vx;
            o[1] = uy + alpha * vy;
            o[2] = uz + alpha * vz;
        } else {
            o[0] = beta * o[0] + (ux + alpha * vx);
            o[1] = beta * o[1] + (uy + alpha * vy);
            o[2] = beta * o[2] + (uz + alpha * vz);
        }
    }
}

__global__ void line_circulation_kernel(uint32_t n_lines, const uint32_t* __restrict__ map_off,
                                        const uint32_t* __restrict__ map_ent, const double* __restrict__ ring_gamma,
                                        uint32_t ring_period, double* __restrict__ out)
{
    const uint32_t l = blockIdx.x * blockDim.x + threadIdx.x;
    if (l >= n_lines)
        return;
    double g = 0.0;
    for (uint32_t k = map_off[l]; k < map_off[l + 1]; ++k) {
        const uint32_t e = map_ent[k];
        const uint32_t r = PVL_IDX(e);
        if (ring_period && (r % ring_period) == 0)
            continue;
        g += PVL_REV(e) ? -ring_gamma[r] : ring_gamma[r];
    }
    out[l] = g;
}

__device__ __forceinline__ void load3(const double* p, uint32_t i, double& x, double& y, double& z)
{
    x = p[3 * (size_t)i];
    y = p[3 * (size_t)i + 1];
    z = p[3 * (size_t)i + 2];
}

// src/core/mesh.c:48-68 (direction of an oriented line: mesh.c:14-22)
__global__ void surface_normal_kernel(uint32_t n_surfaces, const uint32_t* __restrict__ off,
                                      const uint32_t* __restrict__ sl, const uint32_t* __restrict__ lines,
                                      const double* __restrict__ pos, double* __restrict__ out)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_surfaces)
        return;
    const uint32_t k0 = off[s], k1 = off[s + 1];
    auto dir = [&](uint32_t g, double& x, double& y, double& z) {
        double ax, ay, az, bx, by, bz;
        load3(pos, PVL_IDX(lines[2 * PVL_IDX(g)]), ax, ay, az);
        load3(pos, PVL_IDX(lines[2 * PVL_IDX(g) + 1]), bx, by, bz);
        if (PVL_REV(g)) {
            x = bx - ax; y = by - ay; z = bz - az;
        } else {
            x = ax - bx; y = ay - by; z = az - bz;
        }
    };
    double ox = 0, oy = 0, oz = 0, d1x, d1y, d1z;
    dir(sl[k0], d1x, d1y, d1z);
    const double d0x = d1x, d0y = d1y, d0z = d1z;
    for (uint32_t k = k0 + 1; k < k1; ++k) {
        double d2x, d2y, d2z;
        dir(sl[k], d2x, d2y, d2z);
        ox += d2y * d1z - d2z * d1y;
        oy += d2z * d1x - d2x * d1z;
        oz += d2x * d1y - d2y * d1x;
        d1x = d2x; d1y = d2y; d1z = d2z;
    }
    ox += d0y * d1z - d0z * d1y;
    oy += d0z * d1x - d0x * d1z;
    oz += d0x * d1y - d0y * d1x;
    const double inv = 1.0 / sqrt(ox * ox + oy * oy + oz * oz);
    out[3 * (size_t)s] = ox * inv;
    out[3 * (size_t)s + 1] = oy * inv;
    out[3 * (size_t)s + 2] = oz * inv;
}

// src/core/mesh.c:24-46
__global__ void surface_average_kernel(uint32_t n_surfaces, const uint32_t* __restrict__ off,
                                       const uint32_t* __restrict__ sl, const uint32_t* __restrict__ lines,
                                       const double* __restrict__ val, double* __restrict__ out)
{
    const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_surfaces)
        return;
    double ax = 0, ay = 0, az = 0;
    for (uint32_t k = off[s]; k < off[s + 1]; ++k) {
        const uint32_t g = sl[k];
        const uint32_t pt = PVL_REV(g) ? lines[2 * PVL_IDX(g) + 1] : lines[2 * PVL_IDX(g)];
        double x, y, z;
        load3(val, PVL_IDX(pt), x, y, z);
        ax += x; ay += y; az += z;
    }
    const double div = 1.0 / double(off[s + 1] - off[s]);
    out[3 * (size_t)s] = ax * div;
    out[3 * (size_t)s + 1] = ay * div;
    out[3 * (size_t)s + 2] = az * div;
}

// python/pyvl/solver.py:199-206
__global__ void rhs_kernel(uint32_t n, const double* __restrict__ normals, const double* __restrict__ flow, double ux,
                           double uy, double uz, const double* __restrict__ cpv, double* __restrict__ rhs,
                           int32_t* __restrict__ nonfinite)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
        return;
    double ex = flow ? flow[3 * (size_t)i] : ux, ey = flow ? flow[3 * (size_t)i + 1] : uy,
           ez = flow ? flow[3 * (size_t)i + 2] : uz;
    if (cpv) {
        ex -= cpv[3 * (size_t)i];
        ey -= cpv[3 * (size_t)i + 1];
        ez -= cpv[3 * (size_t)i + 2];
    }
    const double b = normals[3 * (size_t)i] * -ex + normals[3 * (size_t)i + 1] * -ey + normals[3 * (size_t)i + 2] * -ez;
    rhs[i] = b;
    if (nonfinite && !isfinite(b))
        atomicExch(nonfinite, 1);
}

// src/meshobject.c:1368-1393
__global__ void line_forces_kernel(uint32_t n_lines, const uint32_t* __restrict__ pl, const uint32_t* __restrict__ dl,
                                   const double* __restrict__ circ, const double* __restrict__ pos,
                                   const double* __restrict__ vel, double* __restrict__ out)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_lines)
        return;
    const uint32_t p1 = PVL_IDX(pl[2 * i]), p2 = PVL_IDX(pl[2 * i + 1]);
    const uint32_t d1 = PVL_IDX(dl[2 * i]), d2 = PVL_IDX(dl[2 * i + 1]);
    double ax, ay, az, bx, by, bz;
    load3(pos, p1, ax, ay, az);
    load3(pos, p2, bx, by, bz);
    const double rx = bx - ax, ry = by - ay, rz = bz - az;
    double c = 0.0;
    if (d1 != PVL_INVALID)
        c += circ[d1];
    if (d2 != PVL_INVALID)
        c -= circ[d2];
    double v1x, v1y, v1z, v2x, v2y, v2z;
    load3(vel, p1, v1x, v1y, v1z);
    load3(vel, p2, v2x, v2y, v2z);
    const double k = 0.5 * c;
    const double wx = (v1x + v2x) * k, wy = (v1y + v2y) * k, wz = (v1z + v2z) * k;
    out[3 * (size_t)i] = ry * wz - rz * wy;
    out[3 * (size_t)i + 1] = rz * wx - rx * wz;
    out[3 * (size_t)i + 2] = rx * wy - ry * wx;
}

inline unsigned blocks_for(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

template <typename T>
int prep_segments(uint32_t n_points, uint32_t n_lines, const uint32_t* lines, const double* positions,
                  const double* line_gamma, double tol, Segment<T>* seg, cudaStream_t st)
{
    if (n_lines == 0)
        return PVL_OK;
    prep_segments_kernel<T><<<blocks_for(n_lines, 256), 256, 0, st>>>(n_points, n_lines, lines, positions, line_gamma,
                                                                       tol, seg);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

// Points per CTA of the sweeps: one per thread in FP64, two per thread (FP32x2) in FP32.
inline uint32_t sweep_points_per_cta(int precision) { return precision == PVL_F32 ? 2 * kSumThreads : kSumThreads; }

// Number of segment ranges a sweep is split into: enough CTAs to fill the 148 SMs many times
// over (32 per SM, so that the last resident wave is short), at least half a tile of segments
// per range in FP64 (small point sets such as the near-row advection then still fill one
// resident wave: 52 instead of 58 us for 1032 points) and two tiles in FP32.
#ifndef PVL_SUM_CTAS_PER_SM
#define PVL_SUM_CTAS_PER_SM 32  // CTAs per SM (148 SMs) the point tiles x line splits aim at
#endif

uint32_t sum_splits(uint32_t n_lines, uint32_t n_pts, int precision)
{
    const uint64_t ctas_x = (n_pts + sweep_points_per_cta(precision) - 1) / sweep_points_per_cta(precision);
    const uint64_t want = 148ull * PVL_SUM_CTAS_PER_SM;
    uint64_t s = (want + ctas_x - 1) / std::max<uint64_t>(ctas_x, 1);
    const uint64_t min_range = precision == PVL_F32 ? 2 * kSegTile : kSegTile / 2;
    const uint64_t max_s = std::max<uint64_t>(1, (n_lines + min_range - 1) / min_range);
    s = std::min(std::max<uint64_t>(s, 1), max_s);
    return (uint32_t)std::min<uint64_t>(s, 65535);
}

int check_stream_args(const void* p, const char* what)
{
    if (!p)
        return pvl_fail(PVL_ERR_ARG, "%s is NULL", what);
    return PVL_OK;
}

}  // namespace

#define PVL_REQUIRE(ptr)                                 \
    do {                                                 \
        int _r = check_stream_args((ptr), #ptr);         \
        if (_r)                                          \
            return _r;                                   \
    } while (0)

extern "C" size_t pvl_segments_workspace(uint32_t n_lines, int precision)
{
    return align256((size_t)n_lines * (precision == PVL_F32 ? sizeof(Segment<float>) : sizeof(Segment<double>)));
}

extern "C" int pvl_prep_segments(int precision, uint32_t n_points, uint32_t n_lines, const uint32_t* lines,
                                 const double* positions, const double* line_gamma, double tol, void* segments,
                                 void* stream)
{
    if (n_lines == 0)
        return PVL_OK;
    PVL_REQUIRE(lines); PVL_REQUIRE(positions); PVL_REQUIRE(segments);
    cudaStream_t st = (cudaStream_t)stream;
    if (precision == PVL_F64)
        return prep_segments<double>(n_points, n_lines, lines, positions, line_gamma, tol,
                                     static_cast<Segment<double>*>(segments), st);
    if (precision == PVL_F32)
        return prep_segments<float>(n_points, n_lines, lines, positions, line_gamma, tol,
                                    static_cast<Segment<float>*>(segments), st);
    return pvl_fail(PVL_ERR_ARG, "pvl_prep_segments: unknown precision %d", precision);
}

extern "C" int pvl_surface_normal(uint32_t n_surfaces, const uint32_t* off, const uint32_t* sl, const uint32_t* lines,
                                  const double* positions, double* out, void* stream)
{
    if (n_surfaces == 0)
        return PVL_OK;
    PVL_REQUIRE(off); PVL_REQUIRE(sl); PVL_REQUIRE(lines); PVL_REQUIRE(positions); PVL_REQUIRE(out);
    surface_normal_kernel<<<blocks_for(n_surfaces, 128), 128, 0, (cudaStream_t)stream>>>(n_surfaces, off, sl, lines,
                                                                                         positions, out);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_surface_average(uint32_t n_surfaces, const uint32_t* off, const uint32_t* sl, const uint32_t* lines,
                                   const double* values, double* out, void* stream)
{
    if (n_surfaces == 0)
        return PVL_OK;
    PVL_REQUIRE(off); PVL_REQUIRE(sl); PVL_REQUIRE(lines); PVL_REQUIRE(values); PVL_REQUIRE(out);
    surface_average_kernel<<<blocks_for(n_surfaces, 128), 128, 0, (cudaStream_t)stream>>>(n_surfaces, off, sl, lines,
                                                                                          values, out);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_rhs(uint32_t n, const double* normals, const double* flow, double ux, double uy, double uz,
                       const double* cp_velocity, double* rhs_out, int32_t* nonfinite, void* stream)
{
    if (n == 0)
        return PVL_OK;
    PVL_REQUIRE(normals); PVL_REQUIRE(rhs_out);
    rhs_kernel<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(n, normals, flow, ux, uy, uz, cp_velocity,
                                                                     rhs_out, nonfinite);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_line_induction(uint32_t n_points, uint32_t n_lines, const uint32_t* lines, const double* positions,
                                  uint32_t n_cp, const double* cps, double tol, double* out, void* ws,
                                  size_t ws_bytes, void* stream)
{
    if (n_lines == 0 || n_cp == 0)
        return PVL_OK;
    PVL_REQUIRE(lines); PVL_REQUIRE(positions); PVL_REQUIRE(cps); PVL_REQUIRE(out); PVL_REQUIRE(ws);
    if (ws_bytes < pvl_segments_workspace(n_lines, PVL_F64))
        return pvl_fail(PVL_ERR_ALLOC, "pvl_line_induction: workspace %zu < %zu", ws_bytes,
                        pvl_segments_workspace(n_lines, PVL_F64));
    cudaStream_t st = (cudaStream_t)stream;
    auto* seg = static_cast<Segment<double>*>(ws);
    if (int r = prep_segments<double>(n_points, n_lines, lines, positions, nullptr, tol, seg, st))
        return r;
    dim3 grid(blocks_for(n_lines, kRingThreads), blocks_for(n_cp, kRingCPB));
    if (grid.y > 65535)
        return pvl_fail(PVL_ERR_ARG, "pvl_line_induction: too many points (%u)", n_cp);
    line_matrix_kernel<<<grid, kRingThreads, 0, st>>>(n_lines, seg, n_cp, cps, pvl::cutoff2<double>(tol), out);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_induction_matrix(uint32_t n_points, uint32_t n_lines, const uint32_t* lines,
                                    const double* positions, uint32_t n_surfaces, const uint32_t* off,
                                    const uint32_t* sl, uint32_t n_cp, const double* cps, double tol, double* out,
                                    void* ws, size_t ws_bytes, void* stream)
{
    if (n_surfaces == 0 || n_cp == 0)
        return PVL_OK;
    PVL_REQUIRE(lines); PVL_REQUIRE(positions); PVL_REQUIRE(off); PVL_REQUIRE(sl); PVL_REQUIRE(cps);
    PVL_REQUIRE(out); PVL_REQUIRE(ws);
    if (ws_bytes < pvl_segments_workspace(n_lines, PVL_F64))
        return pvl_fail(PVL_ERR_ALLOC, "pvl_induction_matrix: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    auto* seg = static_cast<Segment<double>*>(ws);
    if (int r = prep_segments<double>(n_points, n_lines, lines, positions, nullptr, tol, seg, st))
        return r;
    dim3 grid(blocks_for(n_surfaces, kRingThreads), blocks_for(n_cp, kRingCPB));
    if (grid.y > 65535)
        return pvl_fail(PVL_ERR_ARG, "pvl_induction_matrix: too many points (%u)", n_cp);
    ring_matrix_kernel<double, double, 1><<<grid, kRingThreads, 0, st>>>(n_surfaces, off, sl, n_lines, seg, n_cp, cps,
                                                                         nullptr, pvl::cutoff2<double>(tol), out, 0);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_induction_normal(int precision, uint32_t n_points, uint32_t n_lines, const uint32_t* lines,
                                    const double* positions, uint32_t n_surfaces, const uint32_t* off,
                                    const uint32_t* sl, uint32_t n_cp, const double* cps, const double* normals,
                                    double tol, void* out, uint32_t ld, void* ws, size_t ws_bytes, void* stream)
{
    if (n_surfaces == 0 || n_cp == 0)
        return PVL_OK;
    PVL_REQUIRE(lines); PVL_REQUIRE(positions); PVL_REQUIRE(off); PVL_REQUIRE(sl); PVL_REQUIRE(cps);
    PVL_REQUIRE(normals); PVL_REQUIRE(out); PVL_REQUIRE(ws);
    if (precision != PVL_F64 && precision != PVL_F32)
        return pvl_fail(PVL_ERR_ARG, "pvl_induction_normal: unknown precision %d", precision);
    if (ld < n_surfaces)
        return pvl_fail(PVL_ERR_ARG, "pvl_induction_normal: ld %u < n_surfaces %u", ld, n_surfaces);
    if (ws_bytes < pvl_segments_workspace(n_lines, precision))
        return pvl_fail(PVL_ERR_ALLOC, "pvl_induction_normal: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    dim3 grid(blocks_for(n_surfaces, kRingThreads), blocks_for(n_cp, kRingCPB));
    if (grid.y > 65535)
        return pvl_fail(PVL_ERR_ARG, "pvl_induction_normal: too many points (%u)", n_cp);
    if (precision == PVL_F64) {
        auto* seg = static_cast<Segment<double>*>(ws);
        if (int r = prep_segments<double>(n_points, n_lines, lines, positions, nullptr, tol, seg, st))
            return r;
        ring_matrix_kernel<double, double, 0><<<grid, kRingThreads, 0, st>>>(
            n_surfaces, off, sl, n_lines, seg, n_cp, cps, normals, pvl::cutoff2<double>(tol), static_cast<double*>(out), ld);
    } else {
        auto* seg = static_cast<Segment<float>*>(ws);
        if (int r = prep_segments<float>(n_points, n_lines, lines, positions, nullptr, tol, seg, st))
            return r;
        ring_matrix_kernel<float, float, 0><<<grid, kRingThreads, 0, st>>>(
            n_surfaces, off, sl, n_lines, seg, n_cp, cps, normals, pvl::cutoff2<float>(tol), static_cast<float*>(out), ld);
    }
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

namespace {

// Threads of a ring-tile CTA: the candidate with the fewest idle lane-slots in the line loop
// (rounds x threads - lines), ties to fewer threads.
int ring_tile_threads(uint32_t max_tile_lines)
{
    int best = kRingTile;
    uint64_t best_slots = ~0ull;
    for (int t : {128, 160, 192, 256}) {
        const uint64_t slots = (uint64_t)((max_tile_lines + t - 1) / t) * (uint64_t)t;
        if (slots < best_slots) {
            best = t;
            best_slots = slots;
        }
    }
    return best;
}

template <int THREADS>
int launch_ring_tile(dim3 grid, size_t smem, cudaStream_t st, uint32_t n_surfaces, const uint32_t* offsets,
                     const uint32_t* surface_lines, const uint32_t* sl_local, const uint32_t* tile_offsets,
                     const uint32_t* tile_lines, uint32_t max_tile_lines, uint32_t n_lines,
                     const Segment<double>* seg, uint32_t n_cp, const double* cps, const double* normals, double tol,
                     double* out, uint32_t ld)
{
    PVL_SMEM_OPTIN(ring_tile_kernel<THREADS>, smem);
    ring_tile_kernel<THREADS><<<grid, THREADS, smem, st>>>(n_surfaces, offsets, surface_lines, sl_local,
                                                           tile_offsets, tile_lines, max_tile_lines, n_lines, seg,
                                                           n_cp, cps, normals, pvl::cutoff2<double>(tol), out, ld);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

}  // namespace

extern "C" int pvl_induction_normal_tiled(uint32_t n_points, uint32_t n_lines, const uint32_t* lines,
                                          const double* positions, uint32_t n_surfaces, const uint32_t* offsets,
                                          const uint32_t* surface_lines, const uint32_t* tile_offsets,
                                          const uint32_t* tile_lines, const uint32_t* sl_local,
                                          uint32_t max_tile_lines, uint32_t n_cp, const double* cps,
                                          const double* normals, double tol, double* out, uint32_t ld, void* ws,
                                          size_t ws_bytes, void* stream)
{
    if (n_cp == 0 || n_surfaces == 0)
        return PVL_OK;
    PVL_REQUIRE(lines); PVL_REQUIRE(positions); PVL_REQUIRE(offsets); PVL_REQUIRE(surface_lines);
    PVL_REQUIRE(tile_offsets); PVL_REQUIRE(tile_lines); PVL_REQUIRE(sl_local); PVL_REQUIRE(cps);
    PVL_REQUIRE(normals); PVL_REQUIRE(out); PVL_REQUIRE(ws);
    if (ld < n_surfaces)
        return pvl_fail(PVL_ERR_ARG, "pvl_induction_normal_tiled: ld < n_surfaces");
    if (ws_bytes < pvl_segments_workspace(n_lines, PVL_F64))
        return pvl_fail(PVL_ERR_ALLOC, "pvl_induction_normal_tiled: workspace too small");
    const size_t smem = (size_t)kTileCPB * max_tile_lines * sizeof(double);
    if (smem > 200 * 1024)
        return pvl_fail(PVL_ERR_ARG, "pvl_induction_normal_tiled: %u lines in one ring tile exceed shared memory",
                        max_tile_lines);
    cudaStream_t st = (cudaStream_t)stream;
    auto* seg = static_cast<Segment<double>*>(ws);
    if (int r = prep_segments<double>(n_points, n_lines, lines, positions, nullptr, tol, seg, st))
        return r;
    dim3 grid((n_surfaces + kRingTile - 1) / kRingTile, (n_cp + kTileCPB - 1) / kTileCPB);
    switch (ring_tile_threads(max_tile_lines)) {
    case 160:
        return launch_ring_tile<160>(grid, smem, st, n_surfaces, offsets, surface_lines, sl_local, tile_offsets,
                                     tile_lines, max_tile_lines, n_lines, seg, n_cp, cps, normals, tol, out, ld);
    case 192:
        return launch_ring_tile<192>(grid, smem, st, n_surfaces, offsets, surface_lines, sl_local, tile_offsets,
                                     tile_lines, max_tile_lines, n_lines, seg, n_cp, cps, normals, tol, out, ld);
    case 256:
        return launch_ring_tile<256>(grid, smem, st, n_surfaces, offsets, surface_lines, sl_local, tile_offsets,
                                     tile_lines, max_tile_lines, n_lines, seg, n_cp, cps, normals, tol, out, ld);
    default:
        return launch_ring_tile<128>(grid, smem, st, n_surfaces, offsets, surface_lines, sl_local, tile_offsets,
                                     tile_lines, max_tile_lines, n_lines, seg, n_cp, cps, normals, tol, out, ld);
    }
}

extern "C" size_t pvl_line_velocity_workspace(uint32_t n_lines, uint32_t n_pts, int precision)
{
    const size_t el = precision == PVL_F32 ? sizeof(float) : sizeof(double);
    return pvl_segments_workspace(n_lines, precision) +
           align256((size_t)sum_splits(n_lines, n_pts, precision) * n_pts * 3 * el);
}

namespace {

// Shared driver of the N-body sweep: segment table, split sweep, deterministic reduction.
int run_line_sum(int precision, uint32_t n_points, uint32_t n_lines, const uint32_t* lines, const double* positions,
                 const double* line_gamma, uint32_t n_pts, const double* pts, uint32_t group, uint32_t stride,
                 uint32_t in_off, uint32_t row_step, const uint32_t* cols, uint32_t col_limit, uint32_t out_stride,
                 uint32_t out_off, const uint32_t* rows, uint32_t row_limit,
                 const double* normals, double tol,
                 double alpha, double beta, double ux, double uy, double uz, double* out, void* ws, size_t ws_bytes,
                 cudaStream_t st, const char* who)
{
    if (precision != PVL_F64 && precision != PVL_F32)
        return pvl_fail(PVL_ERR_ARG, "%s: unknown precision %d", who, precision);
    if (n_lines == 0) {
        reduce_partials_kernel<double><<<blocks_for(n_pts, kReducePts), kReducePts * kReduceGroups, 0, st>>>(
            n_pts, 0, nullptr, normals, alpha, beta, ux, uy, uz, group, row_step, out_stride, out_off, rows, row_limit,
            out);
        PVL_LAUNCH_CHECK();
        return PVL_OK;
    }
    if (!lines || !positions || !ws)
        return pvl_fail(PVL_ERR_ARG, "%s: null pointer argument", who);
    if (ws_bytes < pvl_line_velocity_workspace(n_lines, n_pts, precision))
        return pvl_fail(PVL_ERR_ALLOC, "%s: workspace %zu < %zu", who, ws_bytes,
                        pvl_line_velocity_workspace(n_lines, n_pts, precision));
    const uint32_t n_split = sum_splits(n_lines, n_pts, precision);
    const uint32_t per = (n_lines + n_split - 1) / n_split;
    const uint32_t n_split_used = (n_lines + per - 1) / per;
    dim3 grid(blocks_for(n_pts, sweep_points_per_cta(precision)), n_split_used);
    char* base = static_cast<char*>(ws);
    if (precision == PVL_F64) {
        auto* seg = reinterpret_cast<Segment<double>*>(base);
        auto* part = reinterpret_cast<double*>(base + pvl_segments_workspace(n_lines, PVL_F64));
        if (int r = prep_segments<double>(n_points, n_lines, lines, positions, line_gamma, tol, seg, st))
            return r;
        line_sum_f64_kernel<<<grid, kSumThreads, 0, st>>>(seg, n_lines, per, pts, n_pts, group, stride, in_off,
                                                          row_step, cols, col_limit, rows, row_limit,
                                                          pvl::cutoff2<double>(tol), part);
        PVL_LAUNCH_CHECK();
        reduce_partials_kernel<double><<<blocks_for(n_pts, kReducePts), kReducePts * kReduceGroups, 0, st>>>(
            n_pts, n_split_used, part, normals, alpha, beta, ux, uy, uz, group, row_step, out_stride, out_off, rows,
            row_limit, out);
    } else {
        auto* seg = reinterpret_cast<Segment<float>*>(base);
        auto* part = reinterpret_cast<float*>(base + pvl_segments_workspace(n_lines, PVL_F32));
        if (int r = prep_segments<float>(n_points, n_lines, lines, positions, line_gamma, tol, seg, st))
            return r;
        line_sum_f32x2_kernel<<<grid, kSumThreads, 0, st>>>(seg, n_lines, per, pts, n_pts, group, stride, in_off,
                                                               row_step, cols, col_limit, rows, row_limit,
                                                               pvl::cutoff2<float>(tol), part);
        PVL_LAUNCH_CHECK();
        reduce_partials_kernel<float><<<blocks_for(n_pts, kReducePts), kReducePts * kReduceGroups, 0, st>>>(
            n_pts, n_split_used, part, normals, alpha, beta, ux, uy, uz, group, row_step, out_stride, out_off, rows,
            row_limit, out);
    }
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

}  // namespace

extern "C" int pvl_line_velocity(int precision, uint32_t n_points, uint32_t n_lines, const uint32_t* lines,
                                 const double* positions, const double* line_gamma, uint32_t n_pts, const double* pts,
                                 const double* normals, double tol, double alpha, double beta, double* out, void* ws,
                                 size_t ws_bytes, void* stream)
{
    if (n_pts == 0)
        return PVL_OK;
    PVL_REQUIRE(pts); PVL_REQUIRE(out);
    return run_line_sum(precision, n_points, n_lines, lines, positions, line_gamma, n_pts, pts, n_pts, n_pts, 0, 1,
                        nullptr, 0xFFFFFFFFu, n_pts, 0, nullptr, 0, normals, tol, alpha, beta, 0.0, 0.0, 0.0, out, ws, ws_bytes, (cudaStream_t)stream,
                        "pvl_line_velocity");
}

extern "C" size_t pvl_wake_node_velocity_workspace(uint32_t n_lines, uint32_t n_shed, uint32_t complete_rows,
                                                   int precision)
{
    return pvl_line_velocity_workspace(n_lines, 2 * n_shed * complete_rows, precision);
}

namespace {

// Sweep of the body's (or any) segments at wake nodes: rows row_begin + k * row_step (k < row_count)
// or, with a row list, rows[k] (k < row_count; entries at or past complete_rows skipped) of the
// n_cols listed node columns; node_vel (n_cols, complete_rows, 3) at the same rows.
int node_velocity(int precision, uint32_t n_points, uint32_t n_lines, const uint32_t* lines, const double* positions,
                  const double* line_gamma, uint32_t n_shed, uint32_t line_rows, uint32_t complete_rows,
                  uint32_t row_begin, uint32_t row_count, uint32_t row_step, const uint32_t* rows, uint32_t n_cols,
                  const uint32_t* cols, const double* wake_pos, double ux, double uy, double uz, double tol,
                  double* node_vel, void* ws, size_t ws_bytes, void* stream, const char* who)
{
    if (complete_rows > line_rows)
        return pvl_fail(PVL_ERR_ARG, "%s: complete_rows %u > line_rows %u", who, complete_rows, line_rows);
    if (!rows && row_count > 0 &&
        (row_step == 0 || (uint64_t)row_begin + (uint64_t)(row_count - 1) * row_step >= (uint64_t)complete_rows))
        return pvl_fail(PVL_ERR_ARG, "%s: rows %u + k * %u (k < %u) outside [0, %u)", who, row_begin, row_step,
                        row_count, complete_rows);
    if (!cols && n_cols != 2 * n_shed)
        return pvl_fail(PVL_ERR_ARG, "%s: without a column list n_cols must be 2 n_shed", who);
    if (n_cols == 0 || row_count == 0)
        return PVL_OK;
    PVL_REQUIRE(wake_pos); PVL_REQUIRE(node_vel);
    const uint64_t n_pts = (uint64_t)n_cols * row_count;
    if (n_pts > 0xFFFFFFFFull)
        return pvl_fail(PVL_ERR_ARG, "%s: too many nodes", who);
    return run_line_sum(precision, n_points, n_lines, lines, positions, line_gamma, (uint32_t)n_pts, wake_pos,
                        row_count, line_rows + 1, row_begin, row_step, cols, 2 * n_shed, complete_rows, row_begin,
                        rows, complete_rows, nullptr, tol, 1.0, 0.0, ux, uy, uz, node_vel, ws, ws_bytes,
                        (cudaStream_t)stream, who);
}

}  // namespace

extern "C" int pvl_wake_node_velocity_rows(int precision, uint32_t n_points, uint32_t n_lines,
                                           const uint32_t* lines, const double* positions, const double* line_gamma,
                                           uint32_t n_shed, uint32_t line_rows, uint32_t complete_rows,
                                           uint32_t row_begin, uint32_t row_count, uint32_t row_step, uint32_t n_cols,
                                           const uint32_t* cols, const double* wake_pos, double ux, double uy,
                                           double uz, double tol, double* node_vel, void* ws, size_t ws_bytes,
                                           void* stream)
{
    return node_velocity(precision, n_points, n_lines, lines, positions, line_gamma, n_shed, line_rows, complete_rows,
                         row_begin, row_count, row_step, nullptr, n_cols, cols, wake_pos, ux, uy, uz, tol, node_vel,
                         ws, ws_bytes, stream, "pvl_wake_node_velocity_rows");
}

extern "C" int pvl_wake_node_velocity_list(int precision, uint32_t n_points, uint32_t n_lines,
                                           const uint32_t* lines, const double* positions, const double* line_gamma,
                                           uint32_t n_shed, uint32_t line_rows, uint32_t complete_rows,
                                           uint32_t n_rows, const uint32_t* rows, uint32_t n_cols,
                                           const uint32_t* cols, const double* wake_pos, double ux, double uy,
                                           double uz, double tol, double* node_vel, void* ws, size_t ws_bytes,
                                           void* stream)
{
    if (n_rows && !rows)
        return pvl_fail(PVL_ERR_ARG, "pvl_wake_node_velocity_list: rows is NULL");
    return node_velocity(precision, n_points, n_lines, lines, positions, line_gamma, n_shed, line_rows, complete_rows,
                         0, n_rows, 1, rows, n_cols, cols, wake_pos, ux, uy, uz, tol, node_vel, ws, ws_bytes, stream,
                         "pvl_wake_node_velocity_list");
}

extern "C" int pvl_wake_node_velocity_cols(int precision, uint32_t n_points, uint32_t n_lines,
                                           const uint32_t* lines, const double* positions, const double* line_gamma,
                                           uint32_t n_shed, uint32_t line_rows, uint32_t complete_rows,
                                           uint32_t row_begin, uint32_t row_end, uint32_t n_cols,
                                           const uint32_t* cols, const double* wake_pos, double ux, double uy,
                                           double uz, double tol, double* node_vel, void* ws, size_t ws_bytes,
                                           void* stream)
{
    if (row_begin > row_end || row_end > complete_rows)
        return pvl_fail(PVL_ERR_ARG, "pvl_wake_node_velocity_cols: rows [%u, %u) outside [0, %u)", row_begin, row_end,
                        complete_rows);
    return pvl_wake_node_velocity_rows(precision, n_points, n_lines, lines, positions, line_gamma, n_shed, line_rows,
                                       complete_rows, row_begin, row_end - row_begin, 1, n_cols, cols, wake_pos, ux,
                                       uy, uz, tol, node_vel, ws, ws_bytes, stream);
}

extern "C" int pvl_wake_node_velocity(int precision, uint32_t n_points, uint32_t n_lines, const uint32_t* lines,
                                      const double* positions, const double* line_gamma, uint32_t n_shed,
                                      uint32_t line_rows, uint32_t complete_rows, const double* wake_pos, double ux,
                                      double uy, double uz, double tol, double* node_vel, void* ws, size_t ws_bytes,
                                      void* stream)
{
    return pvl_wake_node_velocity_cols(precision, n_points, n_lines, lines, positions, line_gamma, n_shed, line_rows,
                                       complete_rows, 0, complete_rows, 2 * n_shed, nullptr, wake_pos, ux, uy, uz,
                                       tol, node_vel, ws, ws_bytes, stream);
}

extern "C" int pvl_line_circulation(uint32_t n_lines, const uint32_t* map_offsets, const uint32_t* map_entries,
                                    const double* ring_gamma, uint32_t ring_period, double* line_gamma_out,
                                    void* stream)
{
    if (n_lines == 0)
        return PVL_OK;
    PVL_REQUIRE(map_offsets); PVL_REQUIRE(map_entries); PVL_REQUIRE(ring_gamma); PVL_REQUIRE(line_gamma_out);
    line_circulation_kernel<<<blocks_for(n_lines, 256), 256, 0, (cudaStream_t)stream>>>(
        n_lines, map_offsets, map_entries, ring_gamma, ring_period, line_gamma_out);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_line_forces(uint32_t n_lines, const uint32_t* primal_lines, const uint32_t* dual_lines,
                               const double* circ, const double* positions, const double* velocity, double* out,
                               void* stream)
{
    if (n_lines == 0)
        return PVL_OK;
    PVL_REQUIRE(primal_lines); PVL_REQUIRE(dual_lines); PVL_REQUIRE(circ); PVL_REQUIRE(positions);
    PVL_REQUIRE(velocity); PVL_REQUIRE(out);
    line_forces_kernel<<<blocks_for(n_lines, 256), 256, 0, (cudaStream_t)stream>>>(n_lines, primal_lines, dual_lines,
                                                                                   circ, positions, velocity, out);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}
