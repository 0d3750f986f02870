// Free-wake state kernels and the closed-body constraint helpers.
//
// Wake node layout is the reference's wake_positions (n_shed, 2, line_rows + 1, 3)
// (python/pyvl/wake_models.py:66-68); wake circulations are (n_shed, line_rows)
// (wake_models.py:74-75); node (s, side, row) = s*2*(R+1) + side*(R+1) + row.
#include <cstdint>

#include "pvl_common.cuh"

namespace {

inline unsigned blocks_for(size_t n, unsigned t) { return (unsigned)((n + t - 1) / t); }

// One thread per system row: apply the shed lines' implicit columns in line order,
// the same order (and so the same rounding) as wake_models.py:209-216.
__global__ void fold_implicit_kernel(uint32_t n_cp, uint32_t n_shed, const double* __restrict__ implicit,
                                     const uint32_t* __restrict__ adj, double* __restrict__ A, uint32_t lda)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_cp)
        return;
    double* row = A + (size_t)i * lda;
    const double* imp = implicit + (size_t)i * n_shed;
    for (uint32_t s = 0; s < n_shed; ++s) {
        const double c = imp[s];
        const uint32_t s1 = adj[2 * s + 1], s0 = adj[2 * s];
        if (s1 != PVL_INVALID)
            row[s1] -= c;
        if (s0 != PVL_INVALID)
            row[s0] += c;
    }
}

// The same fold with one thread per (row, shedding line), for adjacency tables in which no ring
// appears twice (then no two threads touch the same entry, and each entry receives exactly the
// one update the sequential fold gives it).
__global__ void fold_implicit_parallel_kernel(uint32_t n_cp, uint32_t n_shed, const double* __restrict__ implicit,
                                              const uint32_t* __restrict__ adj, double* __restrict__ A, uint32_t lda)
{
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (uint64_t)n_cp * n_shed)
        return;
    const uint32_t i = (uint32_t)(t / n_shed), s = (uint32_t)(t % n_shed);
    const double c = implicit[t];
    const uint32_t s1 = adj[2 * s + 1], s0 = adj[2 * s];
    double* row = A + (size_t)i * lda;
    if (s1 != PVL_INVALID)
        row[s1] -= c;
    if (s0 != PVL_INVALID)
        row[s0] += c;
}

// new[s, side, row]: row 0 = body node; row i+1 = old[i] + v[i] dt (i < complete); rows
// beyond complete collapse onto row `complete` (wake_models.py:113-137).
__global__ void advect_kernel(uint32_t n_shed, uint32_t R, uint32_t complete, const double* __restrict__ old_pos,
                              const double* __restrict__ vel, const uint32_t* __restrict__ col_slot,
                              uint32_t n_slots, double dt,
                              const double* __restrict__ body,
                              const uint32_t* __restrict__ bnodes, double* __restrict__ new_pos)
{
    const uint32_t npr = R + 1;
    const uint64_t n = (uint64_t)n_shed * 2 * npr;
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n)
        return;
    const uint32_t row = (uint32_t)(t % npr);
    const uint64_t col = t / npr;  // s*2 + side
    const uint32_t s = (uint32_t)(col / 2), side = (uint32_t)(col % 2);
    // the source row for this output row
    const uint32_t src = row <= complete ? row : complete;
    double x, y, z;
    if (src == 0) {
        const uint32_t b = bnodes[2 * s + side];
        x = body[3 * (size_t)b];
        y = body[3 * (size_t)b + 1];
        z = body[3 * (size_t)b + 2];
    } else {
        const uint32_t i = src - 1;  // new[i+1] = old[i] + v[i] dt
        const double* o = old_pos + 3 * (col * npr + i);
        const uint64_t slot = col_slot ? col_slot[col] : col;  // node columns may share one velocity row
        if (slot < n_slots) {
            const double* v = vel + 3 * (slot * complete + i);
            x = o[0] + v[0] * dt;
            y = o[1] + v[1] * dt;
            z = o[2] + v[2] * dt;
        } else {  // a slot outside node_vel (broken column map): the node is not moved
            x = o[0];
            y = o[1];
            z = o[2];
        }
    }
    double* out = new_pos + 3 * t;
    out[0] = x;
    out[1] = y;
    out[2] = z;
}

// wake_models.py:139-151
__global__ void shed_kernel(uint32_t n_shed, uint32_t R, const double* __restrict__ old_circ,
                            const uint32_t* __restrict__ adj, const double* __restrict__ gamma,
                            double* __restrict__ new_circ)
{
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (uint64_t)n_shed * R)
        return;
    const uint32_t s = (uint32_t)(t / R), r = (uint32_t)(t % R);
    if (r > 0) {
        new_circ[t] = old_circ[(size_t)s * R + r - 1];
        return;
    }
    double c = 0.0;
    const uint32_t a1 = adj[2 * s + 1], a0 = adj[2 * s];
    if (a1 != PVL_INVALID)
        c += gamma[a1];
    if (a0 != PVL_INVALID)
        c -= gamma[a0];
    new_circ[t] = c;
}

// One CTA per group: mean by a block reduction, then subtract (solver.py:229-233).
__global__ void group_mean_kernel(const uint32_t* __restrict__ goff, double* __restrict__ x)
{
    __shared__ double red[256];
    const uint32_t g = blockIdx.x;
    const uint32_t b = goff[g], e = goff[g + 1];
    double s = 0.0;
    for (uint32_t i = b + threadIdx.x; i < e; i += blockDim.x)
        s += x[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (unsigned w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w)
            red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    const double mean = e > b ? red[0] / double(e - b) : 0.0;
    for (uint32_t i = b + threadIdx.x; i < e; i += blockDim.x)
        x[i] -= mean;
}

__global__ void border_kernel(uint32_t n, uint32_t m, const uint32_t* __restrict__ goff, double* __restrict__ A,
                              uint32_t lda, double* __restrict__ rhs)
{
    // thread t < n + m fills border column entries of row t and border row entries of column t
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t N = n + m;
    if (t >= N)
        return;
    for (uint32_t g = 0; g < m; ++g) {
        const bool in = t < n && t >= goff[g] && t < goff[g + 1];
        A[(size_t)t * lda + n + g] = in ? 1.0 : 0.0;  // column n+g
        A[(size_t)(n + g) * lda + t] = in ? 1.0 : 0.0;  // row n+g
    }
    if (t >= n)
        rhs[t] = 0.0;
}

int require(const void* p, const char* what)
{
    return p ? PVL_OK : pvl_fail(PVL_ERR_ARG, "%s is NULL", what);
}

}  // namespace

#define PVL_REQUIRE(p)                   \
    do {                                 \
        if (int _r = require((p), #p))   \
            return _r;                   \
    } while (0)

// node_vel (n_cols, complete, 3): rows row_first, row_first + 2h, ... <= row_last of every column
// from their neighbours at -3h, -h, +h, +3h rows by the cubic that passes through the four
// (v = (-v[-3h] + 9 v[-h] + 9 v[+h] - v[+3h]) / 16, the midpoint value of the interpolating cubic
// of equally spaced samples).
__global__ void interp_rows_kernel(uint32_t n_cols, uint32_t complete, uint32_t row_first, uint32_t n_rows,
                                   uint32_t h, double* __restrict__ node_vel)
{
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (uint64_t)n_cols * n_rows * 3)
        return;
    const uint32_t k = (uint32_t)(e % 3), r = (uint32_t)((e / 3) % n_rows), c = (uint32_t)(e / (3 * (uint64_t)n_rows));
    const uint32_t i = row_first + 2 * h * r;
    double* col = node_vel + (size_t)c * complete * 3 + k;
    const double a = col[(size_t)(i - 3 * h) * 3], b = col[(size_t)(i - h) * 3];
    const double d = col[(size_t)(i + h) * 3], f = col[(size_t)(i + 3 * h) * 3];
    col[(size_t)i * 3] = (9.0 * (b + d) - (a + f)) * 0.0625;
}

// out[k] = pts[index[k]] (3 doubles); an index outside [0, n_pts) gives NaN.
__global__ void gather_points_kernel(uint32_t n, const uint32_t* __restrict__ index, uint32_t n_pts,
                                     const double* __restrict__ pts, double* __restrict__ out)
{
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (uint64_t)n * 3)
        return;
    const uint32_t k = (uint32_t)(e / 3), c = (uint32_t)(e % 3);
    const uint32_t i = index[k];
    out[e] = i < n_pts ? pts[(size_t)i * 3 + c] : __longlong_as_double(0x7FF8000000000000ll);
}

// out[p] += n_p . sum_k weights[k] values[entries[k]] over k in [offsets[p], offsets[p+1]);
// kStencilLanes lanes per point, each summing every kStencilLanes-th term, then a butterfly
// over the lanes (a fixed order: the result does not depend on the launch).  A range outside
// [0, n_entries) or an entry outside [0, n_values) makes the point's sum NaN (nothing outside
// the arrays is read).  Threads past the last point run the shuffles with no terms.
constexpr unsigned kStencilLanes = 8;

__global__ void stencil_normal_add_kernel(uint32_t n_cp, const uint32_t* __restrict__ offsets, uint32_t n_entries,
                                          const uint32_t* __restrict__ entries, const double* __restrict__ weights,
                                          uint32_t n_values, const double* __restrict__ values,
                                          const double* __restrict__ normals, double* __restrict__ out)
{
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t lane = (uint32_t)(t % kStencilLanes);
    const uint64_t p = t / kStencilLanes;
    const bool live = p < n_cp;
    uint32_t k0 = 0, k1 = 0;
    bool bad = false;
    if (live) {
        k0 = offsets[p];
        k1 = offsets[p + 1];
        bad = k0 > k1 || k1 > n_entries;
        if (bad)
            k1 = k0;
    }
    double vx = 0.0, vy = 0.0, vz = 0.0;
    for (uint32_t k = k0 + lane; k < k1; k += kStencilLanes) {
        const uint32_t j = entries[k];
        if (j >= n_values) {
            bad = true;
            continue;
        }
        const double w = weights[k];
        const double* v = values + (size_t)j * 3;
        vx = fma(w, v[0], vx);
        vy = fma(w, v[1], vy);
        vz = fma(w, v[2], vz);
    }
    int any_bad = bad;
#pragma unroll
    for (unsigned o = kStencilLanes / 2; o > 0; o >>= 1) {
        vx += __shfl_xor_sync(0xffffffffu, vx, o, kStencilLanes);
        vy += __shfl_xor_sync(0xffffffffu, vy, o, kStencilLanes);
        vz += __shfl_xor_sync(0xffffffffu, vz, o, kStencilLanes);
        any_bad |= __shfl_xor_sync(0xffffffffu, any_bad, o, kStencilLanes);
    }
    if (!live || lane != 0)
        return;
    if (any_bad) {
        out[p] = __longlong_as_double(0x7FF8000000000000ll);
        return;
    }
    const double* n = normals + (size_t)p * 3;
    out[p] += n[0] * vx + n[1] * vy + n[2] * vz;
}

// node_vel[c, r] = sum_k weights[k] sub_vel[entries[k], r] over k in [offsets[c], offsets[c+1])
// for rows r in [row_begin, row_end) of every column c; both arrays (columns, complete, 3).  A
// range outside [0, n_entries) or an entry outside [0, n_sub) gives NaN.
__global__ void interp_cols_kernel(uint32_t n_cols, uint32_t complete, uint32_t row_begin, uint32_t n_rows,
                                   const uint32_t* __restrict__ offsets, uint32_t n_entries,
                                   const uint32_t* __restrict__ entries, const double* __restrict__ weights,
                                   uint32_t n_sub, const double* __restrict__ sub_vel, double* __restrict__ node_vel)
{
    const uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (uint64_t)n_cols * n_rows * 3)
        return;
    const uint32_t k = (uint32_t)(e % 3), r = row_begin + (uint32_t)((e / 3) % n_rows);
    const uint32_t c = (uint32_t)(e / (3 * (uint64_t)n_rows));
    const uint32_t k0 = offsets[c], k1 = offsets[c + 1];
    double v = 0.0;
    if (k0 > k1 || k1 > n_entries) {
        v = __longlong_as_double(0x7FF8000000000000ll);
    } else {
        for (uint32_t q = k0; q < k1; ++q) {
            const uint32_t j = entries[q];
            if (j >= n_sub) {
                v = __longlong_as_double(0x7FF8000000000000ll);
                break;
            }
            v = fma(weights[q], sub_vel[((size_t)j * complete + r) * 3 + k], v);
        }
    }
    node_vel[((size_t)c * complete + r) * 3 + k] = v;
}

extern "C" int pvl_gather_points(uint32_t n, const uint32_t* index, uint32_t n_pts, const double* pts, double* out,
                                 void* stream)
{
    if (n == 0)
        return PVL_OK;
    PVL_REQUIRE(index); PVL_REQUIRE(pts); PVL_REQUIRE(out);
    gather_points_kernel<<<blocks_for((uint64_t)n * 3, 256), 256, 0, (cudaStream_t)stream>>>(n, index, n_pts, pts,
                                                                                             out);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_stencil_normal_add(uint32_t n_cp, const uint32_t* offsets, uint32_t n_entries,
                                      const uint32_t* entries, const double* weights, uint32_t n_values,
                                      const double* values, const double* normals, double* out, void* stream)
{
    if (n_cp == 0)
        return PVL_OK;
    PVL_REQUIRE(offsets); PVL_REQUIRE(normals); PVL_REQUIRE(out);
    if (n_entries) {
        PVL_REQUIRE(entries); PVL_REQUIRE(weights); PVL_REQUIRE(values);
    }
    stencil_normal_add_kernel<<<blocks_for((uint64_t)n_cp * kStencilLanes, 128), 128, 0, (cudaStream_t)stream>>>(
        n_cp, offsets, n_entries, entries, weights, n_values, values, normals, out);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_wake_interp_cols(uint32_t n_cols, uint32_t complete_rows, uint32_t row_begin, uint32_t row_end,
                                    const uint32_t* offsets, uint32_t n_entries, const uint32_t* entries,
                                    const double* weights, uint32_t n_sub, const double* sub_vel, double* node_vel,
                                    void* stream)
{
    if (row_end > complete_rows || row_begin > row_end)
        return pvl_fail(PVL_ERR_ARG, "pvl_wake_interp_cols: rows [%u, %u) outside [0, %u)", row_begin, row_end,
                        complete_rows);
    if (n_cols == 0 || row_end == row_begin)
        return PVL_OK;
    PVL_REQUIRE(offsets); PVL_REQUIRE(node_vel);
    if (n_entries) {
        PVL_REQUIRE(entries); PVL_REQUIRE(weights); PVL_REQUIRE(sub_vel);
    }
    const uint32_t n_rows = row_end - row_begin;
    interp_cols_kernel<<<blocks_for((uint64_t)n_cols * n_rows * 3, 256), 256, 0, (cudaStream_t)stream>>>(
        n_cols, complete_rows, row_begin, n_rows, offsets, n_entries, entries, weights, n_sub, sub_vel, node_vel);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_wake_fold_implicit(uint32_t n_cp, uint32_t n_shed, const double* implicit, const uint32_t* adjacent,
                                      double* A, uint32_t lda, void* stream)
{
    if (n_cp == 0 || n_shed == 0)
        return PVL_OK;
    PVL_REQUIRE(implicit); PVL_REQUIRE(adjacent); PVL_REQUIRE(A);
    fold_implicit_kernel<<<blocks_for(n_cp, 128), 128, 0, (cudaStream_t)stream>>>(n_cp, n_shed, implicit, adjacent, A,
                                                                                   lda);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_wake_fold_implicit_distinct(uint32_t n_cp, uint32_t n_shed, const double* implicit,
                                               const uint32_t* adjacent, double* A, uint32_t lda, void* stream)
{
    if (n_cp == 0 || n_shed == 0)
        return PVL_OK;
    PVL_REQUIRE(implicit); PVL_REQUIRE(adjacent); PVL_REQUIRE(A);
    if (lda < n_cp)
        return pvl_fail(PVL_ERR_ARG, "pvl_wake_fold_implicit_distinct: lda < n_cp");
    fold_implicit_parallel_kernel<<<blocks_for((uint64_t)n_cp * n_shed, 256), 256, 0, (cudaStream_t)stream>>>(
        n_cp, n_shed, implicit, adjacent, A, lda);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_wake_advect_cols(uint32_t n_shed, uint32_t line_rows, uint32_t complete_rows,
                                    const double* old_pos, const double* node_vel, const uint32_t* col_slot,
                                    uint32_t n_slots, double dt,
                                    const double* body_positions, const uint32_t* bordering_nodes, double* new_pos,
                                    void* stream)
{
    if (n_shed == 0)
        return PVL_OK;
    if (complete_rows > line_rows)
        return pvl_fail(PVL_ERR_ARG, "pvl_wake_advect: complete_rows %u > line_rows %u", complete_rows, line_rows);
    PVL_REQUIRE(old_pos); PVL_REQUIRE(body_positions); PVL_REQUIRE(bordering_nodes); PVL_REQUIRE(new_pos);
    if (complete_rows > 0)
        PVL_REQUIRE(node_vel);
    if (old_pos == new_pos)
        return pvl_fail(PVL_ERR_ARG, "pvl_wake_advect: old_pos and new_pos must not alias");
    const uint64_t n = (uint64_t)n_shed * 2 * (line_rows + 1);
    advect_kernel<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(
        n_shed, line_rows, complete_rows, old_pos, node_vel, col_slot, col_slot ? n_slots : 2 * n_shed, dt,
        body_positions, bordering_nodes, new_pos);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_wake_advect(uint32_t n_shed, uint32_t line_rows, uint32_t complete_rows, const double* old_pos,
                               const double* node_vel, double dt, const double* body_positions,
                               const uint32_t* bordering_nodes, double* new_pos, void* stream)
{
    return pvl_wake_advect_cols(n_shed, line_rows, complete_rows, old_pos, node_vel, nullptr, 2 * n_shed, dt,
                                body_positions, bordering_nodes, new_pos, stream);
}

extern "C" int pvl_wake_shed(uint32_t n_shed, uint32_t line_rows, const double* old_circ, const uint32_t* adjacent,
                             const double* gamma, double* new_circ, void* stream)
{
    if (n_shed == 0 || line_rows == 0)
        return PVL_OK;
    PVL_REQUIRE(old_circ); PVL_REQUIRE(adjacent); PVL_REQUIRE(gamma); PVL_REQUIRE(new_circ);
    if (old_circ == new_circ)
        return pvl_fail(PVL_ERR_ARG, "pvl_wake_shed: old_circ and new_circ must not alias");
    shed_kernel<<<blocks_for((uint64_t)n_shed * line_rows, 256), 256, 0, (cudaStream_t)stream>>>(
        n_shed, line_rows, old_circ, adjacent, gamma, new_circ);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_group_mean_remove(uint32_t n_groups, const uint32_t* group_offsets, double* x, void* stream)
{
    if (n_groups == 0)
        return PVL_OK;
    PVL_REQUIRE(group_offsets); PVL_REQUIRE(x);
    group_mean_kernel<<<n_groups, 256, 0, (cudaStream_t)stream>>>(group_offsets, x);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_border_groups(uint32_t n, uint32_t m, const uint32_t* group_offsets, double* A, uint32_t lda,
                                 double* rhs, void* stream)
{
    if (m == 0)
        return PVL_OK;
    PVL_REQUIRE(group_offsets); PVL_REQUIRE(A); PVL_REQUIRE(rhs);
    if (lda < n + m)
        return pvl_fail(PVL_ERR_ARG, "pvl_border_groups: lda %u < n + m = %u", lda, n + m);
    border_kernel<<<blocks_for(n + m, 256), 256, 0, (cudaStream_t)stream>>>(n, m, group_offsets, A, lda, rhs);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_wake_interp_rows_spaced(uint32_t n_cols, uint32_t complete_rows, uint32_t row_first,
                                           uint32_t row_last, uint32_t half, double* node_vel, void* stream)
{
    if (half == 0)
        return pvl_fail(PVL_ERR_ARG, "pvl_wake_interp_rows_spaced: half spacing 0");
    if (n_cols == 0 || row_last < row_first)
        return PVL_OK;
    PVL_REQUIRE(node_vel);
    if ((uint64_t)row_first < 3ull * half || (uint64_t)row_last + 3ull * half >= complete_rows)
        return pvl_fail(PVL_ERR_ARG,
                        "pvl_wake_interp_rows: rows %u..%u need rows %u below and above within [0, %u)", row_first,
                        row_last, 3 * half, complete_rows);
    const uint32_t n_rows = (row_last - row_first) / (2 * half) + 1;
    interp_rows_kernel<<<blocks_for((uint64_t)n_cols * n_rows * 3, 256), 256, 0, (cudaStream_t)stream>>>(
        n_cols, complete_rows, row_first, n_rows, half, node_vel);
    PVL_LAUNCH_CHECK();
    return PVL_OK;
}

extern "C" int pvl_wake_interp_rows(uint32_t n_cols, uint32_t complete_rows, uint32_t row_first, uint32_t row_last,
                                    double* node_vel, void* stream)
{
    return pvl_wake_interp_rows_spaced(n_cols, complete_rows, row_first, row_last, 1, node_vel, stream);
}
