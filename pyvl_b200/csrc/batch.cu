// Batched UVLM steps: many independent cases of uneven size, each kernel one launch over the
// whole batch.  No reference counterpart (the reference runs one geometry per solver loop,
// python/pyvl/solver.py:145-265); every case's arithmetic is the single-case path's.
//
// The batch is laid out as one concatenated mesh (global point / line / ring indices, so the
// single-case geometry, segment-table and line-circulation kernels run over it unchanged)
// plus job tables that keep each case's pairs inside the case:
//   * ring jobs   -- a block of a case's ring matrix: its control points x a set of rings
//                    (body rings -> the case's system matrix; first-row wake rings -> its
//                    implicit wake block);
//   * sweep jobs  -- an N-body sum of a case's segments (body or wake) at a list of points
//                    (control points: the explicit wake term; wake nodes: the advection).
// Both job kinds run as persistent kernels: CTAs take work items (job, point block, segment
// range) from an atomic counter, find the job by binary search over the jobs' item offsets,
// and process it; so one launch covers every case regardless of how uneven they are.  The
// tile shape (points per thread, threads per CTA; control points per CTA for ring jobs) is a
// template parameter chosen by the host-side autotuner.
//
// The solve is a device-resident, Jacobi right-preconditioned GMRES per case with FP64
// residuals: per-case Hessenberg matrices, Givens rotations and convergence masks live on the
// device, a fixed number of iterations is launched (converged cases skip their work), so a
// whole step contains no host synchronisation and can be captured in a CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "pvl_common.cuh"
#include "sweep.cuh"

using pvl::Segment;
using pvl::Vec3;

namespace {

inline unsigned blocks_for(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

constexpr int kSegTile = 128;

// ------------------------------------------------------------------ job tables
struct RingJob {
    uint32_t cp_begin, n_cp;      // control points (global index into cps / normals)
    uint32_t ring_begin, n_rings; // rings (global CSR rows: offsets[ring_begin ..])
    uint64_t out_begin;           // out[out_begin + i * ld + j]
    uint32_t ld;
    uint32_t item_begin;          // first work item of this job
};

struct SweepJob {
    uint32_t seg_begin, seg_count;   // segments of the job (global segment table)
    uint32_t pt_begin, pt_max;       // point list: pidx[pt_begin ..] (or points pts[pt_begin ..] when pidx == NULL)
    uint32_t pt_per_row;             // > 0: pt_count = pt_per_row * min(*rows, pt_max / pt_per_row)
    uint32_t out_begin;              // output slot of the job's first point
    uint32_t n_split, per;           // segment ranges and segments per range
    uint32_t part_begin;             // partials of the job: part[(part_begin + split * pt_max + p) * 3 + c]
    uint32_t item_begin;             // first work item; items = ceil(pt_max / pts_per_cta) * n_split
    uint32_t mode;                   // 0: normal output (out[o] += n . v); 1: vector output (out = U + v)
    uint32_t case_id;
    uint32_t seg_rows;               // != kNoRows: the job's segments are in row order and only the first
                                     // seg_upto[seg_rows + min(*rows, rows_max)] of them (the rows shed so
                                     // far) are swept; the other ranges write zero partials
};

constexpr uint32_t kNoRows = 0xFFFFFFFFu;

__device__ __forceinline__ uint32_t find_job(const uint32_t* __restrict__ item_begin, uint32_t n_jobs, uint32_t item)
{
    uint32_t lo = 0, hi = n_jobs;  // largest j with item_begin[j] <= item
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (item_begin[mid] <= item)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// ------------------------------------------------------------------ ring jobs
template <int CPB>
__global__ void __launch_bounds__(128) batched_ring_kernel(const RingJob* __restrict__ jobs,
                                                           const uint32_t* __restrict__ job_item, uint32_t n_jobs,
                                                           uint32_t n_items, uint32_t* __restrict__ counter,
                                                           const uint32_t* __restrict__ off,
                                                           const uint32_t* __restrict__ sl, uint32_t n_lines,
                                                           const Segment<double>* __restrict__ seg,
                                                           const double* __restrict__ cps,
                                                           const double* __restrict__ nrm, double tol2,
                                                           double* __restrict__ out)
{
    __shared__ uint32_t s_item;
    __shared__ double s_p[CPB][3], s_n[CPB][3];
    for (;;) {
        if (threadIdx.x == 0)
            s_item = atomicAdd(counter, 1u);
        __syncthreads();
        const uint32_t item = s_item;
        if (item >= n_items)
            return;
        const uint32_t jb = find_job(job_item, n_jobs, item);
        const RingJob J = jobs[jb];
        const uint32_t col_tiles = (J.n_rings + 127) / 128;
        const uint32_t local = item - J.item_begin;
        const uint32_t rb = local / col_tiles, ct = local % col_tiles;
        const uint32_t i0 = rb * CPB;
        if (threadIdx.x < CPB * 3) {
            const uint32_t q = threadIdx.x / 3, c = threadIdx.x % 3;
            const bool ok = i0 + q < J.n_cp;
            s_p[q][c] = ok ? cps[3 * (size_t)(J.cp_begin + i0 + q) + c] : 0.0;
            s_n[q][c] = ok ? nrm[3 * (size_t)(J.cp_begin + i0 + q) + c] : 0.0;
        }
        __syncthreads();
        const uint32_t j = ct * 128 + threadIdx.x;
        if (j < J.n_rings) {
            const uint32_t r = J.ring_begin + j;
            pvl::RingSegments<double> rs;
            rs.load(sl, off[r], off[r + 1], n_lines, seg);
#pragma unroll 1
            for (int q = 0; q < CPB; ++q) {
                if (i0 + q >= J.n_cp)
                    break;
                const Vec3<double> acc = rs.sum(sl, n_lines, seg, s_p[q][0], s_p[q][1], s_p[q][2], tol2);
                out[J.out_begin + (size_t)(i0 + q) * J.ld + j] =
                    acc.x * s_n[q][0] + acc.y * s_n[q][1] + acc.z * s_n[q][2];
            }
        }
        __syncthreads();
    }
}

// The same blocks with each line of a tile evaluated once per control point (as
// pvl_induction_normal_tiled does for one mesh): work item (job, CPB control points, 128
// rings); the tile's distinct lines (tile_lines[tile_off[t] ..], t = job_tile[job] + column
// tile) are evaluated at the CTA's control points into shared memory, n_i . u_l(cp_i), and
// each thread sums its ring's signed entries (sl_local: each CSR entry's position in its
// tile's list), in CSR order.  Adjacent rings share lines, so a quad mesh needs ~0.57 line
// evaluations per (point, ring line) instead of one.
// FOLD (implicit wake blocks): the block is not stored; the value of control point i and
// first-row ring j (shedding line shed = J.ring_begin + j) is folded straight into the case's
// system matrix, A[i, adj[2 shed + 1]] -= v and A[i, adj[2 shed]] += v (out_begin / ld = the
// matrix), the arithmetic of the fold kernel.  Only for cases in which every body ring is
// adjacent to at most one shedding-line side, so that no two threads touch one entry.
template <int CPB, bool FOLD>
__global__ void __launch_bounds__(128) batched_ring_tile_kernel(
    const RingJob* __restrict__ jobs, const uint32_t* __restrict__ job_item, uint32_t n_jobs, uint32_t n_items,
    uint32_t* __restrict__ counter, const uint32_t* __restrict__ off, const uint32_t* __restrict__ sl,
    const uint32_t* __restrict__ sl_local, const uint32_t* __restrict__ job_tile,
    const uint32_t* __restrict__ tile_off, const uint32_t* __restrict__ tile_lines, uint32_t tile_stride,
    uint32_t n_lines, const Segment<double>* __restrict__ seg, const double* __restrict__ cps,
    const double* __restrict__ nrm, double tol2, const uint32_t* __restrict__ fold_adj, double* __restrict__ out)
{
    extern __shared__ double sV[];  // [CPB][tile_stride]
    __shared__ uint32_t s_item;
    __shared__ double s_p[CPB][3], s_n[CPB][3];
    for (;;) {
        if (threadIdx.x == 0)
            s_item = atomicAdd(counter, 1u);
        __syncthreads();
        const uint32_t item = s_item;
        if (item >= n_items)
            return;
        const uint32_t jb = find_job(job_item, n_jobs, item);
        const RingJob J = jobs[jb];
        const uint32_t col_tiles = (J.n_rings + 127) / 128;
        const uint32_t local = item - J.item_begin;
        const uint32_t rb = local / col_tiles, ct = local % col_tiles;
        const uint32_t i0 = rb * CPB;
        const int nq = (int)min((uint32_t)CPB, J.n_cp - i0);  // CTA-uniform, >= 1
        if (threadIdx.x < CPB * 3) {
            const uint32_t q = threadIdx.x / 3, c = threadIdx.x % 3;
            const bool ok = (int)q < nq;
            s_p[q][c] = ok ? cps[3 * (size_t)(J.cp_begin + i0 + q) + c] : 0.0;
            s_n[q][c] = ok ? nrm[3 * (size_t)(J.cp_begin + i0 + q) + c] : 0.0;
        }
        __syncthreads();
        const uint32_t t = job_tile[jb] + ct;
        const uint32_t L0 = tile_off[t], nl = min(tile_off[t + 1] - L0, tile_stride);
        for (uint32_t l = threadIdx.x; l < nl; l += 128) {
            const uint32_t g = tile_lines[L0 + l];
            Segment<double> sg;
            if (g < n_lines) {
                sg = seg[g];
            } else {  // d = 0: nothing induced
                sg.r1x = sg.r1y = sg.r1z = sg.dx = sg.dy = sg.dz = 0.0;
                sg.len = sg.len2 = sg.gamma = sg.glen = sg.pad0 = sg.pad1 = 0.0;
            }
#pragma unroll 4
            for (int q = 0; q < nq; ++q) {
                Vec3<double> acc{0.0, 0.0, 0.0};
                pvl::segment_induction<double, false, true>(sg, s_p[q][0], s_p[q][1], s_p[q][2], tol2, 1.0, acc);
                sV[q * tile_stride + l] = acc.x * s_n[q][0] + acc.y * s_n[q][1] + acc.z * s_n[q][2];
            }
        }
        __syncthreads();
        const uint32_t j = ct * 128 + threadIdx.x;
        if (j < J.n_rings) {
            const uint32_t r = J.ring_begin + j;
            pvl::RingEntries re;
            re.load(sl, sl_local, off[r], off[r + 1]);
            for (int q = 0; q < nq; ++q) {
                const double v = re.sum(sV + q * tile_stride, tile_stride, sl, sl_local);
                if (FOLD) {
                    double* arow = out + J.out_begin + (size_t)(i0 + q) * J.ld;
                    const uint32_t a1 = fold_adj[2 * (size_t)r + 1], a0 = fold_adj[2 * (size_t)r];
                    if (a1 != PVL_INVALID && a1 < J.ld)
                        arow[a1] -= v;
                    if (a0 != PVL_INVALID && a0 < J.ld)
                        arow[a0] += v;
                } else {
                    out[J.out_begin + (size_t)(i0 + q) * J.ld + j] = v;
                }
            }
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------ sweep jobs
// The single-case sweep's pair arithmetic (sweep.cuh): each work item's segments are staged in
// Pluecker form about the centroid of the item's points (one case's points, so neighbours),
// and a thread evaluates them at its PPT points -- two segments per iteration when it holds
// one point, one segment at PPT points otherwise (PPT independent chains).
template <int THREADS, int PPT>
__global__ void __launch_bounds__(THREADS) batched_sweep_kernel(const SweepJob* __restrict__ jobs,
                                                                const uint32_t* __restrict__ job_item,
                                                                uint32_t n_jobs, uint32_t n_items,
                                                                uint32_t* __restrict__ counter,
                                                                const uint32_t* __restrict__ rows,
                                                                const uint32_t* __restrict__ seg_upto,
                                                                uint32_t rows_max,
                                                                const Segment<double>* __restrict__ seg,
                                                                const double* __restrict__ pts,
                                                                const uint32_t* __restrict__ pidx, double tol2,
                                                                double* __restrict__ part)
{
    constexpr uint32_t kPts = THREADS * PPT;
    __shared__ pvl::SweepSeg s_seg[kSegTile + 1];
    __shared__ double s_red[THREADS / 32][4];
    __shared__ double s_o[3];
    __shared__ uint32_t s_item;
    if (threadIdx.x == 0)
        s_seg[kSegTile] = pvl::SweepSeg{};  // the partner of an odd last segment: d = 0, nothing induced
    for (;;) {
        if (threadIdx.x == 0)
            s_item = atomicAdd(counter, 1u);
        __syncthreads();
        const uint32_t item = s_item;
        if (item >= n_items)
            return;
        const uint32_t jb = find_job(job_item, n_jobs, item);
        const SweepJob J = jobs[jb];
        uint32_t n_pts = J.pt_max;
        if (J.pt_per_row)
            n_pts = J.pt_per_row * min(rows[0], J.pt_max / J.pt_per_row);
        const uint32_t blocks = (J.pt_max + kPts - 1) / kPts;
        const uint32_t local = item - J.item_begin;
        const uint32_t split = local / blocks, pb = local % blocks;
        const uint32_t p0 = pb * kPts;
        if (p0 >= n_pts) {  // CTA-uniform: this step has fewer points than the job's maximum
            __syncthreads();
            continue;
        }
        uint32_t seg_count = J.seg_count;
        if (J.seg_rows != kNoRows && seg_upto)
            seg_count = min(seg_count, seg_upto[J.seg_rows + min(rows[0], rows_max)]);
        const uint32_t l_begin = J.seg_begin + split * J.per;
        const uint32_t l_end = J.seg_begin + min(seg_count, (split + 1) * J.per);  // may be <= l_begin: zeros
        double px[PPT], py[PPT], pz[PPT];
        Vec3<double> acc[PPT];
        double cx = 0.0, cy = 0.0, cz = 0.0, cn = 0.0;
#pragma unroll
        for (int t = 0; t < PPT; ++t) {
            const uint32_t p = p0 + t * THREADS + threadIdx.x;
            const bool ok = p < n_pts;
            const size_t q = ok ? (pidx ? pidx[J.pt_begin + p] : J.pt_begin + p) : 0;
            px[t] = ok ? pts[3 * q] : 0.0;
            py[t] = ok ? pts[3 * q + 1] : 0.0;
            pz[t] = ok ? pts[3 * q + 2] : 0.0;
            cx += px[t];
            cy += py[t];
            cz += pz[t];
            cn += ok ? 1.0 : 0.0;
            acc[t] = Vec3<double>{0.0, 0.0, 0.0};
        }
        pvl::cta_centroid<THREADS>(cx, cy, cz, cn, s_red, s_o);  // px.. are 0 for absent points
#pragma unroll
        for (int t = 0; t < PPT; ++t) {
            px[t] -= s_o[0];
            py[t] -= s_o[1];
            pz[t] -= s_o[2];
        }
        for (uint32_t l0 = l_begin; l0 < l_end; l0 += kSegTile) {
            for (uint32_t e = threadIdx.x; e < kSegTile; e += THREADS)
                if (l0 + e < l_end)
                    s_seg[e] = pvl::sweep_seg(seg[l0 + e], s_o);
            __syncthreads();
            const int cnt = (int)min((uint32_t)kSegTile, l_end - l0);
            if (PPT == 1) {
#pragma unroll 1
                for (int k = 0; k < cnt; k += 2) {  // k + 1 <= cnt: a segment, or the zero one at the tile end
                    const pvl::SweepSeg a = s_seg[k], b = s_seg[k + 1 < cnt ? k + 1 : kSegTile];
                    const pvl::SweepGeo ga = pvl::sweep_geo(a, px[0], py[0], pz[0]);
                    const pvl::SweepGeo gb = pvl::sweep_geo(b, px[0], py[0], pz[0]);
                    pvl::sweep_add(a, ga, tol2, acc[0]);
                    pvl::sweep_add(b, gb, tol2, acc[0]);
                }
            } else {
#pragma unroll 1
                for (int k = 0; k < cnt; ++k) {
                    const pvl::SweepSeg a = s_seg[k];
#pragma unroll
                    for (int t = 0; t < PPT; ++t) {
                        const pvl::SweepGeo ga = pvl::sweep_geo(a, px[t], py[t], pz[t]);
                        pvl::sweep_add(a, ga, tol2, acc[t]);
                    }
                }
            }
            __syncthreads();
        }
#pragma unroll
        for (int t = 0; t < PPT; ++t) {
            const uint32_t p = p0 + t * THREADS + threadIdx.x;
            if (p < n_pts) {
                double* o = part + 3 * ((size_t)J.part_begin + (size_t)split * J.pt_max + p);
                o[0] = acc[t].x;
                o[1] = acc[t].y;
                o[2] = acc[t].z;
            }
        }
        __syncthreads();
    }
}

// out for every job point: mode 0: rhs[out] += n . sum_split; mode 1: vel[out] = U_case + sum_split.
// One thread per (job, point) over the maximal point count; threads beyond this step's count idle.
__global__ void batched_sweep_reduce_kernel(const SweepJob* __restrict__ jobs, const uint32_t* __restrict__ pt_item,
                                            uint32_t n_jobs, uint32_t n_total, const uint32_t* __restrict__ rows,
                                            const double* __restrict__ part, const double* __restrict__ nrm,
                                            const double* __restrict__ uinf, double* __restrict__ out)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_total)
        return;
    const uint32_t jb = find_job(pt_item, n_jobs, t);
    const SweepJob J = jobs[jb];
    const uint32_t p = t - pt_item[jb];
    uint32_t n_pts = J.pt_max;
    if (J.pt_per_row)
        n_pts = J.pt_per_row * min(rows[0], J.pt_max / J.pt_per_row);
    if (p >= n_pts)
        return;
    double vx = 0.0, vy = 0.0, vz = 0.0;
    for (uint32_t s = 0; s < J.n_split; ++s) {
        const double* q = part + 3 * ((size_t)J.part_begin + (size_t)s * J.pt_max + p);
        vx += q[0];
        vy += q[1];
        vz += q[2];
    }
    const size_t o = (size_t)J.out_begin + p;
    if (J.mode == 0) {
        const size_t cp = (size_t)J.pt_begin + p;  // normal output: points are control points in order
        out[o] += vx * nrm[3 * cp] + vy * nrm[3 * cp + 1] + vz * nrm[3 * cp + 2];
    } else {
        out[3 * o] = uinf[3 * J.case_id] + vx;
        out[3 * o + 1] = uinf[3 * J.case_id + 1] + vy;
        out[3 * o + 2] = uinf[3 * J.case_id + 2] + vz;
    }
}

// ------------------------------------------------------------------ per-case wake bookkeeping
struct WakeCase {
    uint32_t P, S, n_cols;         // rings, shedding lines, distinct node columns
    uint32_t ring_begin;           // global index of the case's first body ring (control point)
    uint64_t mat_begin;            // system matrix block (P x P, ld = P)
    uint32_t imp_begin;            // implicit block (P x S, ld = S)
    uint32_t shed_begin;           // shedding-line tables: adj / bn / col_slot at shed_begin * 2
    uint32_t pos_begin;            // wake node positions: (S, 2, R + 1, 3) at pos_begin * 3
    uint32_t circ_begin;           // wake circulations (S, R) at circ_begin
    uint32_t vel_begin;            // node velocities (R rows x n_cols) at vel_begin * 3
    double dt;
};

// A[i][adj1] -= implicit[i][s], A[i][adj0] += implicit[i][s] for every case
// (wake_models.py:204-216); thread per (case row).
__global__ void batched_fold_kernel(const WakeCase* __restrict__ cases, const uint32_t* __restrict__ row_case,
                                   uint32_t n_rows, const double* __restrict__ implicit,
                                   const uint32_t* __restrict__ adj, double* __restrict__ A)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_rows)
        return;
    const WakeCase C = cases[row_case[t]];
    const uint32_t i = t - C.ring_begin;
    double* arow = A + C.mat_begin + (size_t)i * C.P;
    const double* irow = implicit + C.imp_begin + (size_t)i * C.S;
    for (uint32_t s = 0; s < C.S; ++s) {  // same order and signs as the single-case fold
        const double v = irow[s];
        const uint32_t a1 = adj[2 * (size_t)(C.shed_begin + s) + 1], a0 = adj[2 * (size_t)(C.shed_begin + s)];
        if (a1 != PVL_INVALID && a1 < C.P)
            arow[a1] -= v;
        if (a0 != PVL_INVALID && a0 < C.P)
            arow[a0] += v;
    }
}

// new positions of every wake node (wake_models.py:113-137): row 0 pinned to the bordering body
// node, rows 1..complete advected from the old row above, rows beyond collapsed.  Thread per node.
__global__ void batched_advect_kernel(const WakeCase* __restrict__ cases, const uint32_t* __restrict__ node_case,
                                      uint32_t n_nodes, uint32_t R, const uint32_t* __restrict__ rows,
                                      const double* __restrict__ old_pos, const double* __restrict__ vel,
                                      const uint32_t* __restrict__ col_slot, const double* __restrict__ body,
                                      const uint32_t* __restrict__ bnodes, double* __restrict__ new_pos)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_nodes)
        return;
    const WakeCase C = cases[node_case[t]];
    const uint32_t complete = min(rows[0], R);
    const uint32_t local = t - C.pos_begin;
    const uint32_t npr = R + 1;
    const uint32_t row = local % npr, col = local / npr;  // col = s * 2 + side
    const uint32_t src = row <= complete ? row : complete;
    double x, y, z;
    if (src == 0) {
        const uint32_t b = bnodes[2 * (size_t)C.shed_begin + col];
        x = body[3 * (size_t)b];
        y = body[3 * (size_t)b + 1];
        z = body[3 * (size_t)b + 2];
    } else {
        const uint32_t i = src - 1;
        const double* o = old_pos + 3 * ((size_t)C.pos_begin + (size_t)col * npr + i);
        const uint32_t slot = col_slot[2 * (size_t)C.shed_begin + col];
        const double* v = vel + 3 * ((size_t)C.vel_begin + (size_t)i * C.n_cols + slot);
        x = o[0] + v[0] * C.dt;
        y = o[1] + v[1] * C.dt;
        z = o[2] + v[2] * C.dt;
    }
    double* out = new_pos + 3 * (size_t)t;
    out[0] = x;
    out[1] = y;
    out[2] = z;
}

// wake circulation shift + shed (wake_models.py:139-151): new[s][0] = gamma[adj1] - gamma[adj0],
// new[s][r] = old[s][r-1].
__global__ void batched_shed_kernel(const WakeCase* __restrict__ cases, const uint32_t* __restrict__ circ_case,
                                    uint32_t n_circ, uint32_t R, const double* __restrict__ old_circ,
                                    const uint32_t* __restrict__ adj, const double* __restrict__ gamma,
                                    double* __restrict__ new_circ)
{
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n_circ)
        return;
    const WakeCase C = cases[circ_case[t]];
    const uint32_t local = t - C.circ_begin;
    const uint32_t s = local / R, r = local % R;
    if (r > 0) {
        new_circ[t] = old_circ[t - 1];
        return;
    }
    double g = 0.0;  // same order and signs as the single-case shed
    const uint32_t a1 = adj[2 * (size_t)(C.shed_begin + s) + 1], a0 = adj[2 * (size_t)(C.shed_begin + s)];
    if (a1 != PVL_INVALID && a1 < C.P)
        g += gamma[C.ring_begin + a1];
    if (a0 != PVL_INVALID && a0 < C.P)
        g -= gamma[C.ring_begin + a0];
    new_circ[t] = g;
}

__global__ void increment_kernel(uint32_t* __restrict__ v)
{
    if (threadIdx.x == 0 && blockIdx.x == 0)
        v[0] += 1u;
}

// ------------------------------------------------------------------ batched GMRES (Jacobi, FP64)
struct SolveCase {
    uint32_t row_begin, n;   // rows of the case in the concatenated vectors
    uint64_t mat_begin;      // A block (n x n, ld = n)
};

// y[row] = alpha * (A_c (D^-1 v))[row] + beta * y[row] (jacobi != 0) or alpha * (A_c v)[row] + ...,
// one warp per row; rows of inactive cases are skipped.
__global__ void __launch_bounds__(256) bgemv_kernel(const SolveCase* __restrict__ cases,
                                                    const uint32_t* __restrict__ row_case, uint32_t n_rows,
                                                    const double* __restrict__ A, const double* __restrict__ v,
                                                    const double* __restrict__ dinv, double alpha, double beta,
                                                    double* __restrict__ y, const uint8_t* __restrict__ active)
{
    const uint32_t r = blockIdx.x * 8 + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (r >= n_rows)
        return;
    const uint32_t c = row_case[r];
    if (active && !active[c])
        return;
    const SolveCase C = cases[c];
    const double* arow = A + C.mat_begin + (size_t)(r - C.row_begin) * C.n;
    const double* x = v + C.row_begin;
    const double* di = dinv ? dinv + C.row_begin : nullptr;
    double s = 0.0;
    for (uint32_t j = lane; j < C.n; j += 32)
        s += arow[j] * (di ? x[j] * di[j] : x[j]);
    for (int o = 16; o > 0; o >>= 1)
        s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0)
        y[r] = beta == 0.0 ? alpha * s : alpha * s + beta * y[r];
}

// out[c * stride + i] = V_i . w over case c's rows (i < k), or ||w||^2 when V == NULL; block per (case, i).
__global__ void __launch_bounds__(256) bdot_kernel(const SolveCase* __restrict__ cases, uint32_t k,
                                                   const double* __restrict__ V, uint64_t ldv,
                                                   const double* __restrict__ w, double* __restrict__ out,
                                                   uint32_t stride, const uint8_t* __restrict__ active)
{
    __shared__ double red[8];
    const uint32_t c = blockIdx.x, i = blockIdx.y;
    if (i >= k || (active && !active[c]))
        return;
    const SolveCase C = cases[c];
    const double* a = V ? V + (size_t)i * ldv + C.row_begin : w + C.row_begin;
    const double* b = w + C.row_begin;
    double s = 0.0;
    for (uint32_t j = threadIdx.x; j < C.n; j += 256)
        s += a[j] * b[j];
    for (int o = 16; o > 0; o >>= 1)
        s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0)
        red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < 8; ++q)
            t += red[q];
        out[(size_t)c * stride + i] = t;
    }
}

// w[row] -= sum_{i<k} c[case][i] V_i[row]; with acc != NULL also acc[case][i] += c[case][i] (thread 0 of row 0).
__global__ void baxpy_kernel(const uint32_t* __restrict__ row_case, uint32_t n_rows, uint32_t k,
                             const double* __restrict__ V, uint64_t ldv, const double* __restrict__ coef,
                             uint32_t stride, double sign, double* __restrict__ w,
                             const uint8_t* __restrict__ active)
{
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_rows)
        return;
    const uint32_t c = row_case[r];
    if (active && !active[c])
        return;
    double s = 0.0;
    for (uint32_t i = 0; i < k; ++i)
        s += coef[(size_t)c * stride + i] * V[(size_t)i * ldv + r];
    w[r] += sign * s;
}

// v[row] = w[row] / sqrt(nsq[case]) (0 when the norm is 0).
__global__ void bscale_kernel(const uint32_t* __restrict__ row_case, uint32_t n_rows, const double* __restrict__ w,
                              const double* __restrict__ nsq, uint32_t stride, double* __restrict__ v,
                              const uint8_t* __restrict__ active)
{
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_rows)
        return;
    const uint32_t c = row_case[r];
    if (active && !active[c])
        return;
    const double n2 = nsq[(size_t)c * stride];
    v[r] = n2 > 0.0 ? w[r] / sqrt(n2) : 0.0;
}

// Per-case GMRES state, one thread per case.
struct GmresState {
    double H[16][17];   // H[j][i]: column j (i <= j + 1), rotated in place
    double cs[16], sn[16], g[17];
    double bnorm, target;
    uint32_t k;          // columns accepted
    uint32_t done;
};

// Start: nsq0 = ||b||^2 (slot 0), nsq1 = ||r0||^2 (slot 1).
__global__ void bgmres_init_kernel(uint32_t n_cases, const double* __restrict__ nsq, uint32_t stride, double tol,
                                   GmresState* __restrict__ st, uint8_t* __restrict__ active)
{
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cases)
        return;
    GmresState& S = st[c];
    S.bnorm = sqrt(nsq[(size_t)c * stride]);
    const double beta = sqrt(nsq[(size_t)c * stride + 1]);
    S.target = tol * S.bnorm;
    S.g[0] = beta;
    S.k = 0;
    S.done = beta <= S.target ? 1u : 0u;
    active[c] = S.done ? 0 : 1;
}

// Column j: h (first j+1 entries, two CGS passes summed) and ||w||^2 at hn[c*stride]; apply the
// previous rotations, form the new one, update g; mark converged cases inactive.
__global__ void bgmres_column_kernel(uint32_t n_cases, uint32_t j, const double* __restrict__ h1,
                                     const double* __restrict__ h2, uint32_t stride, const double* __restrict__ hn,
                                     GmresState* __restrict__ st, uint8_t* __restrict__ active)
{
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cases || !active[c])
        return;
    GmresState& S = st[c];
    double col[17];
    for (uint32_t i = 0; i <= j; ++i)
        col[i] = h1[(size_t)c * stride + i] + h2[(size_t)c * stride + i];
    const double hnext = sqrt(hn[(size_t)c * stride]);
    col[j + 1] = hnext;
    for (uint32_t i = 0; i < j; ++i) {
        const double t = S.cs[i] * col[i] + S.sn[i] * col[i + 1];
        col[i + 1] = -S.sn[i] * col[i] + S.cs[i] * col[i + 1];
        col[i] = t;
    }
    const double den = hypot(col[j], col[j + 1]);
    const double cj = den == 0.0 ? 1.0 : col[j] / den, sj = den == 0.0 ? 0.0 : col[j + 1] / den;
    S.cs[j] = cj;
    S.sn[j] = sj;
    col[j] = cj * col[j] + sj * col[j + 1];
    col[j + 1] = 0.0;
    S.g[j + 1] = -sj * S.g[j];
    S.g[j] = cj * S.g[j];
    for (uint32_t i = 0; i <= j; ++i)
        S.H[j][i] = col[i];
    S.k = j + 1;
    if (fabs(S.g[j + 1]) <= S.target || hnext == 0.0) {
        S.done = 1;
        active[c] = 0;
    }
}

// y = R^-1 g (back substitution, k columns), written to y[c * stride + i].
__global__ void bgmres_solve_kernel(uint32_t n_cases, const GmresState* __restrict__ st, double* __restrict__ y,
                                    uint32_t stride)
{
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cases)
        return;
    const GmresState& S = st[c];
    const uint32_t k = S.k;
    for (uint32_t i = 0; i < stride; ++i)
        y[(size_t)c * stride + i] = 0.0;
    for (int i = (int)k - 1; i >= 0; --i) {
        double t = S.g[i];
        for (uint32_t q = (uint32_t)i + 1; q < k; ++q)
            t -= S.H[q][i] * y[(size_t)c * stride + q];
        y[(size_t)c * stride + i] = S.H[i][i] != 0.0 ? t / S.H[i][i] : 0.0;
    }
}

// x[row] += dinv[row] * sum_{i < k_case} y[case][i] V_i[row]  (columns a case never built are not read)
__global__ void bgmres_update_kernel(const uint32_t* __restrict__ row_case, uint32_t n_rows,
                                     const GmresState* __restrict__ st, const double* __restrict__ V, uint64_t ldv,
                                     const double* __restrict__ y, uint32_t stride, const double* __restrict__ dinv,
                                     double* __restrict__ x)
{
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_rows)
        return;
    const uint32_t c = row_case[r];
    const uint32_t k = st[c].k;
    double s = 0.0;
    for (uint32_t i = 0; i < k; ++i)
        s += y[(size_t)c * stride + i] * V[(size_t)i * ldv + r];
    x[r] += dinv[r] * s;
}

// dinv[row] = 1 / A_c[i][i]
__global__ void bdiag_inverse_kernel(const SolveCase* __restrict__ cases, const uint32_t* __restrict__ row_case,
                                     uint32_t n_rows, const double* __restrict__ A, double* __restrict__ dinv)
{
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_rows)
        return;
    const SolveCase C = cases[row_case[r]];
    const uint32_t i = r - C.row_begin;
    const double d = A[C.mat_begin + (size_t)i * C.n + i];
    dinv[r] = d != 0.0 ? 1.0 / d : 1.0;
}

// flag[c] = 1 if ||b - A x||_c > tol ||b||_c (nsq slot 0: ||r||^2, GmresState::bnorm), else 0; and
// the batch's count of failed cases in fail[0].
__global__ void bcheck_kernel(uint32_t n_cases, const double* __restrict__ nsq, uint32_t stride,
                              const GmresState* __restrict__ st, double tol, uint8_t* __restrict__ flag,
                              uint32_t* __restrict__ fail)
{
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cases)
        return;
    const double r = sqrt(nsq[(size_t)c * stride]);
    const bool bad = !(r <= tol * st[c].bnorm);
    flag[c] = bad ? 1 : 0;
    if (bad)
        atomicAdd(fail, 1u);
}

// Persistent grid: every SM filled with as many CTAs as fit (occupancy of the kernel).
uint32_t persistent_ctas(const void* fn, int threads)
{
    int dev = 0, sms = 0, per = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, threads, 0) != cudaSuccess)
        return 148u * 4u;
    return (uint32_t)std::max(1, sms * std::max(1, per));
}

template <int CPB>
int launch_ring(const void* jobs, const uint32_t* job_item, uint32_t n_jobs, uint32_t n_items, uint32_t* counter,
                const uint32_t* off, const uint32_t* sl, uint32_t n_lines, const void* seg, const double* cps,
                const double* nrm, double tol, double* out, uint32_t n_ctas, cudaStream_t st)
{
    if (n_ctas == 0)
        n_ctas = persistent_ctas((const void*)batched_ring_kernel<CPB>, 128);
    batched_ring_kernel<CPB><<<n_ctas, 128, 0, st>>>(static_cast<const RingJob*>(jobs), job_item, n_jobs, n_items,
                                                      counter, off, sl, n_lines,
                                                      static_cast<const Segment<double>*>(seg), cps, nrm, pvl::cutoff2<double>(tol),
                                                      out);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

template <int CPB>
int launch_ring_tiled(const void* jobs, const uint32_t* job_item, uint32_t n_jobs, uint32_t n_items,
                      uint32_t* counter, const uint32_t* off, const uint32_t* sl, const uint32_t* sl_local,
                      const uint32_t* job_tile, const uint32_t* tile_off, const uint32_t* tile_lines,
                      uint32_t tile_stride, uint32_t n_lines, const void* seg, const double* cps, const double* nrm,
                      double tol, const uint32_t* fold_adj, double* out, uint32_t n_ctas, cudaStream_t st)
{
    const size_t smem = (size_t)CPB * tile_stride * sizeof(double);
    if (smem > 200 * 1024)
        return pvl_fail(PVL_ERR_ARG, "pvl_batch_ring_matrix_tiled: %u lines in one tile x %d control points exceed "
                        "shared memory", tile_stride, CPB);
    const void* fn = fold_adj ? (const void*)batched_ring_tile_kernel<CPB, true>
                              : (const void*)batched_ring_tile_kernel<CPB, false>;
    PVL_SMEM_OPTIN(fn, smem);
    if (n_ctas == 0) {
        int dev = 0, sms = 0, per = 0;
        if (cudaGetDevice(&dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, 128, smem) != cudaSuccess)
            return pvl_fail(PVL_ERR_CUDA, "pvl_batch_ring_matrix_tiled: occupancy query failed");
        n_ctas = (uint32_t)std::max(1, sms * std::max(1, per));
    }
    auto* J = static_cast<const RingJob*>(jobs);
    auto* sg = static_cast<const Segment<double>*>(seg);
    if (fold_adj)
        batched_ring_tile_kernel<CPB, true><<<n_ctas, 128, smem, st>>>(J, job_item, n_jobs, n_items, counter, off, sl,
                                                                        sl_local, job_tile, tile_off, tile_lines,
                                                                        tile_stride, n_lines, sg, cps, nrm,
                                                                        pvl::cutoff2<double>(tol), fold_adj, out);
    else
        batched_ring_tile_kernel<CPB, false><<<n_ctas, 128, smem, st>>>(J, job_item, n_jobs, n_items, counter, off,
                                                                         sl, sl_local, job_tile, tile_off, tile_lines,
                                                                         tile_stride, n_lines, sg, cps, nrm,
                                                                         pvl::cutoff2<double>(tol), nullptr, out);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

template <int THREADS, int PPT>
int launch_sweep(const void* jobs, const uint32_t* job_item, uint32_t n_jobs, uint32_t n_items, uint32_t* counter,
                 const uint32_t* rows, const uint32_t* seg_upto, uint32_t rows_max, const void* seg, const double* pts,
                 const uint32_t* pidx, double tol, double* part, uint32_t n_ctas, cudaStream_t st)
{
    if (n_ctas == 0)
        n_ctas = persistent_ctas((const void*)batched_sweep_kernel<THREADS, PPT>, THREADS);
    batched_sweep_kernel<THREADS, PPT><<<n_ctas, THREADS, 0, st>>>(
        static_cast<const SweepJob*>(jobs), job_item, n_jobs, n_items, counter, rows, seg_upto, rows_max,
        static_cast<const Segment<double>*>(seg), pts, pidx, pvl::cutoff2<double>(tol), part);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

}  // namespace

// ------------------------------------------------------------------ C ABI
extern "C" size_t pvl_batch_ring_job_bytes(void) { return sizeof(RingJob); }
extern "C" size_t pvl_batch_sweep_job_bytes(void) { return sizeof(SweepJob); }
extern "C" size_t pvl_batch_wake_case_bytes(void) { return sizeof(WakeCase); }
extern "C" size_t pvl_batch_solve_case_bytes(void) { return sizeof(SolveCase); }
extern "C" size_t pvl_batch_gmres_state_bytes(void) { return sizeof(GmresState); }
extern "C" uint32_t pvl_batch_gmres_max_iter(void) { return 16; }

extern "C" int pvl_batch_ring_matrix(int cpb, const void* jobs, const uint32_t* job_item, uint32_t n_jobs,
                                     uint32_t n_items, uint32_t* counter, const uint32_t* offsets,
                                     const uint32_t* surface_lines, uint32_t n_lines, const void* segments,
                                     const double* cps, const double* normals, double tol, double* out,
                                     uint32_t n_ctas, void* stream)
{
    if (n_items == 0)
        return PVL_OK;
    if (!jobs || !job_item || !counter || !offsets || !surface_lines || !segments || !cps || !normals || !out)
        return pvl_fail(PVL_ERR_ARG, "pvl_batch_ring_matrix: null pointer argument");
    cudaStream_t st = (cudaStream_t)stream;
    PVL_CUDA_CHECK(cudaMemsetAsync(counter, 0, sizeof(uint32_t), st));
    switch (cpb) {
    case 4: return launch_ring<4>(jobs, job_item, n_jobs, n_items, counter, offsets, surface_lines, n_lines, segments,
                                  cps, normals, tol, out, n_ctas, st);
    case 8: return launch_ring<8>(jobs, job_item, n_jobs, n_items, counter, offsets, surface_lines, n_lines, segments,
                                  cps, normals, tol, out, n_ctas, st);
    case 16: return launch_ring<16>(jobs, job_item, n_jobs, n_items, counter, offsets, surface_lines, n_lines,
                                    segments, cps, normals, tol, out, n_ctas, st);
    default: return pvl_fail(PVL_ERR_ARG, "pvl_batch_ring_matrix: control points per CTA must be 4, 8 or 16");
    }
}

extern "C" int pvl_batch_ring_matrix_tiled(int cpb, const void* jobs, const uint32_t* job_item, uint32_t n_jobs,
                                           uint32_t n_items, uint32_t* counter, const uint32_t* offsets,
                                           const uint32_t* surface_lines, const uint32_t* sl_local,
                                           const uint32_t* job_tile, const uint32_t* tile_offsets,
                                           const uint32_t* tile_lines, uint32_t max_tile_lines, uint32_t n_lines,
                                           const void* segments, const double* cps, const double* normals, double tol,
                                           const uint32_t* fold_adj, double* out, uint32_t n_ctas, void* stream)
{
    if (n_items == 0)
        return PVL_OK;
    if (!jobs || !job_item || !counter || !offsets || !surface_lines || !sl_local || !job_tile || !tile_offsets ||
        !tile_lines || !segments || !cps || !normals || !out)
        return pvl_fail(PVL_ERR_ARG, "pvl_batch_ring_matrix_tiled: null pointer argument");
    if (max_tile_lines == 0)
        return pvl_fail(PVL_ERR_ARG, "pvl_batch_ring_matrix_tiled: max_tile_lines is 0");
    cudaStream_t st = (cudaStream_t)stream;
    PVL_CUDA_CHECK(cudaMemsetAsync(counter, 0, sizeof(uint32_t), st));
    switch (cpb) {
#define PVL_RING_TILED(C)                                                                                           \
    case C:                                                                                                         \
        return launch_ring_tiled<C>(jobs, job_item, n_jobs, n_items, counter, offsets, surface_lines, sl_local,     \
                                    job_tile, tile_offsets, tile_lines, max_tile_lines, n_lines, segments, cps,     \
                                    normals, tol, fold_adj, out, n_ctas, st);
        PVL_RING_TILED(8)
        PVL_RING_TILED(16)
        PVL_RING_TILED(32)
#undef PVL_RING_TILED
    default: return pvl_fail(PVL_ERR_ARG, "pvl_batch_ring_matrix_tiled: control points per CTA must be 8, 16 or 32");
    }
}

extern "C" int pvl_batch_sweep(int threads, int ppt, const void* jobs, const uint32_t* job_item, uint32_t n_jobs,
                               uint32_t n_items, uint32_t* counter, const uint32_t* rows, const uint32_t* seg_upto,
                               uint32_t rows_max, const void* segments, const double* pts, const uint32_t* pidx,
                               double tol, double* partials, uint32_t n_ctas, void* stream)
{
    if (n_items == 0)
        return PVL_OK;
    if (!jobs || !job_item || !counter || !rows || !segments || !pts || !partials)
        return pvl_fail(PVL_ERR_ARG, "pvl_batch_sweep: null pointer argument");
    cudaStream_t st = (cudaStream_t)stream;
    PVL_CUDA_CHECK(cudaMemsetAsync(counter, 0, sizeof(uint32_t), st));
    const int key = threads * 10 + ppt;
    switch (key) {
    case 1281: return launch_sweep<128, 1>(jobs, job_item, n_jobs, n_items, counter, rows, seg_upto, rows_max,
                                           segments, pts, pidx, tol, partials, n_ctas, st);
    case 1282: return launch_sweep<128, 2>(jobs, job_item, n_jobs, n_items, counter, rows, seg_upto, rows_max,
                                           segments, pts, pidx, tol, partials, n_ctas, st);
    case 1284: return launch_sweep<128, 4>(jobs, job_item, n_jobs, n_items, counter, rows, seg_upto, rows_max,
                                           segments, pts, pidx, tol, partials, n_ctas, st);
    case 2561: return launch_sweep<256, 1>(jobs, job_item, n_jobs, n_items, counter, rows, seg_upto, rows_max,
                                           segments, pts, pidx, tol, partials, n_ctas, st);
    case 2562: return launch_sweep<256, 2>(jobs, job_item, n_jobs, n_items, counter, rows, seg_upto, rows_max,
                                           segments, pts, pidx, tol, partials, n_ctas, st);
    default: return pvl_fail(PVL_ERR_ARG, "pvl_batch_sweep: unsupported tile (threads %d, points/thread %d)", threads,
                             ppt);
    }
}

extern "C" int pvl_batch_sweep_reduce(const void* jobs, const uint32_t* pt_item, uint32_t n_jobs, uint32_t n_total,
                                      const uint32_t* rows, const double* partials, const double* normals,
                                      const double* uinf, double* out, void* stream)
{
    if (n_total == 0)
        return PVL_OK;
    if (!jobs || !pt_item || !rows || !partials || !out)
        return pvl_fail(PVL_ERR_ARG, "pvl_batch_sweep_reduce: null pointer argument");
    batched_sweep_reduce_kernel<<<blocks_for(n_total, 256), 256, 0, (cudaStream_t)stream>>>(
        static_cast<const SweepJob*>(jobs), pt_item, n_jobs, n_total, rows, partials, normals, uinf, out);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_batch_fold_implicit(const void* cases, const uint32_t* row_case, uint32_t n_rows,
                                       const double* implicit, const uint32_t* adjacent, double* A, void* stream)
{
    if (n_rows == 0)
        return PVL_OK;
    if (!cases || !row_case || !implicit || !adjacent || !A)
        return pvl_fail(PVL_ERR_ARG, "pvl_batch_fold_implicit: null pointer argument");
    batched_fold_kernel<<<blocks_for(n_rows, 128), 128, 0, (cudaStream_t)stream>>>(
        static_cast<const WakeCase*>(cases), row_case, n_rows, implicit, adjacent, A);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_batch_wake_advect(const void* cases, const uint32_t* node_case, uint32_t n_nodes, uint32_t R,
                                     const uint32_t* rows, const double* old_pos, const double* node_vel,
                                     const uint32_t* col_slot, const double* body, const uint32_t* bordering_nodes,
                                     double* new_pos, void* stream)
{
    if (n_nodes == 0)
        return PVL_OK;
    if (!cases || !node_case || !rows || !old_pos || !node_vel || !col_slot || !body || !bordering_nodes || !new_pos)
        return pvl_fail(PVL_ERR_ARG, "pvl_batch_wake_advect: null pointer argument");
    if (old_pos == new_pos)
        return pvl_fail(PVL_ERR_ARG, "pvl_batch_wake_advect: old_pos and new_pos must not alias");
    batched_advect_kernel<<<blocks_for(n_nodes, 256), 256, 0, (cudaStream_t)stream>>>(
        static_cast<const WakeCase*>(cases), node_case, n_nodes, R, rows, old_pos, node_vel, col_slot, body,
        bordering_nodes, new_pos);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_batch_wake_shed(const void* cases, const uint32_t* circ_case, uint32_t n_circ, uint32_t R,
                                   const double* old_circ, const uint32_t* adjacent, const double* gamma,
                                   double* new_circ, void* stream)
{
    if (n_circ == 0)
        return PVL_OK;
    if (!cases || !circ_case || !old_circ || !adjacent || !gamma || !new_circ || R == 0)
        return pvl_fail(PVL_ERR_ARG, "pvl_batch_wake_shed: null pointer argument");
    if (old_circ == new_circ)
        return pvl_fail(PVL_ERR_ARG, "pvl_batch_wake_shed: old_circ and new_circ must not alias");
    batched_shed_kernel<<<blocks_for(n_circ, 256), 256, 0, (cudaStream_t)stream>>>(
        static_cast<const WakeCase*>(cases), circ_case, n_circ, R, old_circ, adjacent, gamma, new_circ);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_batch_increment(uint32_t* value, void* stream)
{
    if (!value)
        return pvl_fail(PVL_ERR_ARG, "pvl_batch_increment: null pointer");
    increment_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(value);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

// Batched GMRES: x (rows of every case) updated in place so that ||b - A x||_c <= tol ||b||_c;
// fail_flags[c] = 1 for cases that missed 10 tol, and fail_count (not reset here) counts them.
// ws layout (doubles unless noted), sized by pvl_batch_gmres_workspace:
//   V (m + 1) x n_rows | w n_rows | dinv n_rows | coef: 3 blocks of n_cases x stride |
//   GmresState n_cases | active bytes n_cases.
extern "C" size_t pvl_batch_gmres_workspace(uint32_t n_rows, uint32_t n_cases, uint32_t max_iter)
{
    const size_t stride = 32;
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    return al(sizeof(double) * (size_t)(max_iter + 1) * n_rows) + 2 * al(sizeof(double) * n_rows) +
           3 * al(sizeof(double) * n_cases * stride) + al(sizeof(GmresState) * n_cases) + al(n_cases);
}

extern "C" int pvl_batch_gmres(const void* cases, const uint32_t* row_case, uint32_t n_rows, uint32_t n_cases,
                               const double* A, const double* b, double* x, uint32_t max_iter, double tol,
                               uint8_t* fail_flags, uint32_t* fail_count, void* ws, size_t ws_bytes, void* stream)
{
    if (n_rows == 0 || n_cases == 0)
        return PVL_OK;
    if (!cases || !row_case || !A || !b || !x || !fail_flags || !fail_count || !ws)
        return pvl_fail(PVL_ERR_ARG, "pvl_batch_gmres: null pointer argument");
    if (max_iter == 0 || max_iter > 16)
        return pvl_fail(PVL_ERR_ARG, "pvl_batch_gmres: max_iter must be in [1, 16]");
    if (ws_bytes < pvl_batch_gmres_workspace(n_rows, n_cases, max_iter))
        return pvl_fail(PVL_ERR_ALLOC, "pvl_batch_gmres: workspace too small");
    cudaStream_t st = (cudaStream_t)stream;
    const uint32_t stride = 32;
    auto al = [](size_t x) { return (x + 255) & ~size_t(255); };
    char* p = static_cast<char*>(ws);
    double* V = reinterpret_cast<double*>(p);
    p += al(sizeof(double) * (size_t)(max_iter + 1) * n_rows);
    double* w = reinterpret_cast<double*>(p);
    p += al(sizeof(double) * n_rows);
    double* dinv = reinterpret_cast<double*>(p);
    p += al(sizeof(double) * n_rows);
    double* h1 = reinterpret_cast<double*>(p);
    p += al(sizeof(double) * n_cases * stride);
    double* h2 = reinterpret_cast<double*>(p);
    p += al(sizeof(double) * n_cases * stride);
    double* nsq = reinterpret_cast<double*>(p);
    p += al(sizeof(double) * n_cases * stride);
    GmresState* gs = reinterpret_cast<GmresState*>(p);
    p += al(sizeof(GmresState) * n_cases);
    uint8_t* active = reinterpret_cast<uint8_t*>(p);
    const SolveCase* C = static_cast<const SolveCase*>(cases);
    const uint64_t ldv = n_rows;
    const unsigned gr = blocks_for(n_rows, 8), g1 = blocks_for(n_rows, 256), gc = blocks_for(n_cases, 128);

    bdiag_inverse_kernel<<<g1, 256, 0, st>>>(C, row_case, n_rows, A, dinv);
    PVL_LAUNCH_CHECK();
    // r0 = b - A x ; ||b||^2 -> nsq[c][0], ||r0||^2 -> nsq[c][1]; V0 = r0 / ||r0||
    PVL_CUDA_CHECK(cudaMemcpyAsync(w, b, sizeof(double) * n_rows, cudaMemcpyDeviceToDevice, st));
    bgemv_kernel<<<gr, 256, 0, st>>>(C, row_case, n_rows, A, x, nullptr, -1.0, 1.0, w, nullptr);
    PVL_LAUNCH_CHECK();
    bdot_kernel<<<dim3(n_cases, 1), 256, 0, st>>>(C, 1, nullptr, 0, b, nsq, stride, nullptr);
    PVL_LAUNCH_CHECK();
    bdot_kernel<<<dim3(n_cases, 1), 256, 0, st>>>(C, 1, nullptr, 0, w, nsq + 1, stride, nullptr);
    PVL_LAUNCH_CHECK();
    bgmres_init_kernel<<<gc, 128, 0, st>>>(n_cases, nsq, stride, tol, gs, active);
    PVL_LAUNCH_CHECK();
    bscale_kernel<<<g1, 256, 0, st>>>(row_case, n_rows, w, nsq + 1, stride, V, nullptr);
    PVL_LAUNCH_CHECK();
    for (uint32_t j = 0; j < max_iter; ++j) {
        double* Vj = V + (size_t)j * ldv;
        // w = A D^-1 V_j
        bgemv_kernel<<<gr, 256, 0, st>>>(C, row_case, n_rows, A, Vj, dinv, 1.0, 0.0, w, active);
        PVL_LAUNCH_CHECK();
        // two classical Gram-Schmidt passes
        double* hp[2] = {h1, h2};
        for (int pass = 0; pass < 2; ++pass) {
            bdot_kernel<<<dim3(n_cases, j + 1), 256, 0, st>>>(C, j + 1, V, ldv, w, hp[pass], stride, active);
            PVL_LAUNCH_CHECK();
            baxpy_kernel<<<g1, 256, 0, st>>>(row_case, n_rows, j + 1, V, ldv, hp[pass], stride, -1.0, w, active);
            PVL_LAUNCH_CHECK();
        }
        bdot_kernel<<<dim3(n_cases, 1), 256, 0, st>>>(C, 1, nullptr, 0, w, nsq, stride, active);
        PVL_LAUNCH_CHECK();
        bscale_kernel<<<g1, 256, 0, st>>>(row_case, n_rows, w, nsq, stride, V + (size_t)(j + 1) * ldv, active);
        PVL_LAUNCH_CHECK();
        bgmres_column_kernel<<<gc, 128, 0, st>>>(n_cases, j, h1, h2, stride, nsq, gs, active);
        PVL_LAUNCH_CHECK();
    }
    bgmres_solve_kernel<<<gc, 128, 0, st>>>(n_cases, gs, h1, stride);
    PVL_LAUNCH_CHECK();
    bgmres_update_kernel<<<g1, 256, 0, st>>>(row_case, n_rows, gs, V, ldv, h1, stride, dinv, x);
    PVL_LAUNCH_CHECK();
    // the true FP64 residual decides
    PVL_CUDA_CHECK(cudaMemcpyAsync(w, b, sizeof(double) * n_rows, cudaMemcpyDeviceToDevice, st));
    bgemv_kernel<<<gr, 256, 0, st>>>(C, row_case, n_rows, A, x, nullptr, -1.0, 1.0, w, nullptr);
    PVL_LAUNCH_CHECK();
    bdot_kernel<<<dim3(n_cases, 1), 256, 0, st>>>(C, 1, nullptr, 0, w, nsq, stride, nullptr);
    PVL_LAUNCH_CHECK();
    bcheck_kernel<<<gc, 128, 0, st>>>(n_cases, nsq, stride, gs, tol * 10.0, fail_flags, fail_count);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}
