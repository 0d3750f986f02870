/*
 * CPU ORACLE — test infrastructure only.
 *
 * A plain-C restatement of the reference's induction, reduction, topology and
 * line-force routines, used by tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py as the CHECKER of the CUDA path.  Nothing in the
 * product (pyvl_b200/, include/) links, loads or calls this file.
 *
 * Every function restates one reference function and cites it (paths relative to
 * the reference project root).  The arithmetic follows the reference operation by
 * operation so that results agree to the last few ulps; the parity of this file
 * with the reference itself is pinned by tests/test_oracle_pins.py against golden
 * vectors generated from the compiled reference (tests/golden/make_golden.py).
 *
 * Index convention: a "geo id" is a uint32 whose low 31 bits are an index and
 * whose bit 31 marks reversed orientation (src/core/common.h:46-56;
 * INVALID_ID = 0x7FFFFFFF).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_IDX(g) ((g) & 0x7FFFFFFFu)
#define ORC_REV(g) ((g) >> 31)
#define ORC_INVALID 0x7FFFFFFFu

typedef struct { double x, y, z; } v3;

static inline v3 v3_sub(v3 a, v3 b) { return (v3){a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline v3 v3_add(v3 a, v3 b) { return (v3){a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline double v3_dot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 v3_cross(v3 a, v3 b)
{
    return (v3){a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
static inline v3 v3_scale(v3 a, double k) { return (v3){a.x * k, a.y * k, a.z * k}; }
static inline v3 v3_load(const double *p) { return (v3){p[0], p[1], p[2]}; }
static inline void v3_store(double *p, v3 a) { p[0] = a.x; p[1] = a.y; p[2] = a.z; }

/*
 * Segment -> point induction for every (line, point) pair.
 * Restates compute_line_induction, src/core/flow_solver.c:86-139:
 *   d = (r2 - r1)/|r2 - r1|; zero if |r2 - r1| < tol (:107-112)
 *   t_k = d.(p - r_k); h^2 = ((|dr1|^2 - t1^2) + (|dr2|^2 - t2^2))/2 (:117-123)
 *   zero if h^2 < tol^2 (:125-130)
 *   u = (dr1 x d) * (atan2(t2, h) - atan2(t1, h)) / h (:131-135)
 * Output layout out[(icp * n_lines + iln) * 3 + c] (:136).
 */
void orc_line_induction(unsigned n_lines, const uint32_t *lines, const double *positions,
                        unsigned n_cpts, const double *cpts, double *out, double tol)
{
    long iln;
#pragma omp parallel for schedule(static)
    for (iln = 0; iln < (long)n_lines; ++iln)
    {
        const v3 r1 = v3_load(positions + 3 * (size_t)ORC_IDX(lines[2 * iln + 0]));
        const v3 r2 = v3_load(positions + 3 * (size_t)ORC_IDX(lines[2 * iln + 1]));
        v3 d = v3_sub(r2, r1);
        const double len = sqrt(v3_dot(d, d));
        d.x /= len;
        d.y /= len;
        d.z /= len;
        for (unsigned icp = 0; icp < n_cpts; ++icp)
        {
            double *const o = out + 3 * ((size_t)icp * n_lines + (size_t)iln);
            if (len < tol)
            {
                v3_store(o, (v3){0, 0, 0});
                continue;
            }
            const v3 p = v3_load(cpts + 3 * (size_t)icp);
            const v3 dr1 = v3_sub(p, r1);
            const v3 dr2 = v3_sub(p, r2);
            const double t1 = v3_dot(d, dr1);
            const double t2 = v3_dot(d, dr2);
            const double h1 = v3_dot(dr1, dr1) - t1 * t1;
            const double h2 = v3_dot(dr2, dr2) - t2 * t2;
            const double hsq = (h1 + h2) / 2.0;
            if (hsq < tol * tol)
            {
                v3_store(o, (v3){0, 0, 0});
                continue;
            }
            const double h = sqrt(hsq);
            const double mag = (atan2(t2, h) - atan2(t1, h)) / h;
            v3_store(o, v3_scale(v3_cross(dr1, d), mag));
        }
    }
}

/*
 * Signed ring sum of line inductions, optionally projected on the point normal.
 * Restates line_induction_to_surface_induction (src/core/flow_solver.c:141-172)
 * when normals == NULL (out is (n_cpts, n_surfaces, 3)), and
 * line_induction_to_normal_surface_induction (:174-205) otherwise (out is
 * (n_cpts, n_surfaces)).  Reversed lines are subtracted (:159-166, :192-199).
 */
void orc_ring_reduce(unsigned n_surfaces, const uint32_t *surface_offsets,
                     const uint32_t *surface_lines, unsigned n_lines, unsigned n_cpts,
                     const double *normals, const double *line_ind, double *out)
{
    long is;
#pragma omp parallel for schedule(static)
    for (is = 0; is < (long)n_surfaces; ++is)
    {
        for (unsigned icp = 0; icp < n_cpts; ++icp)
        {
            v3 res = {0, 0, 0};
            for (uint32_t k = surface_offsets[is]; k < surface_offsets[is + 1]; ++k)
            {
                const uint32_t g = surface_lines[k];
                const v3 u = v3_load(line_ind + 3 * ((size_t)icp * n_lines + ORC_IDX(g)));
                res = ORC_REV(g) ? v3_sub(res, u) : v3_add(res, u);
            }
            if (normals)
                out[(size_t)icp * n_surfaces + (size_t)is] = v3_dot(res, v3_load(normals + 3 * (size_t)icp));
            else
                v3_store(out + 3 * ((size_t)icp * n_surfaces + (size_t)is), res);
        }
    }
}

/* Ring centroid = mean of the ring's vertices, each taken as the start point of the
 * oriented line.  Restates surface_center, src/core/mesh.c:24-46. */
void orc_surface_center(unsigned n_surfaces, const uint32_t *surface_offsets,
                        const uint32_t *surface_lines, const uint32_t *lines,
                        const double *positions, double *out)
{
    for (unsigned is = 0; is < n_surfaces; ++is)
    {
        v3 acc = {0, 0, 0};
        for (uint32_t k = surface_offsets[is]; k < surface_offsets[is + 1]; ++k)
        {
            const uint32_t g = surface_lines[k];
            const uint32_t pt = ORC_REV(g) ? lines[2 * ORC_IDX(g) + 1] : lines[2 * ORC_IDX(g) + 0];
            acc = v3_add(acc, v3_load(positions + 3 * (size_t)ORC_IDX(pt)));
        }
        const double div = 1.0 / (double)(surface_offsets[is + 1] - surface_offsets[is]);
        v3_store(out + 3 * (size_t)is, (v3){acc.x * div, acc.y * div, acc.z * div});
    }
}

/* Oriented line direction p1 - p2 (reversed: p2 - p1), src/core/mesh.c:14-22. */
static v3 orc_line_direction(const double *positions, const uint32_t *lines, uint32_t g)
{
    const v3 a = v3_load(positions + 3 * (size_t)ORC_IDX(lines[2 * ORC_IDX(g) + 0]));
    const v3 b = v3_load(positions + 3 * (size_t)ORC_IDX(lines[2 * ORC_IDX(g) + 1]));
    return ORC_REV(g) ? v3_sub(b, a) : v3_sub(a, b);
}

/* Unit ring normal = normalise(sum_k d_k x d_{k-1} + d_0 x d_last).
 * Restates surface_normal, src/core/mesh.c:48-68 (real3_unit at common.h:122-126). */
void orc_surface_normal(unsigned n_surfaces, const uint32_t *surface_offsets,
                        const uint32_t *surface_lines, const uint32_t *lines,
                        const double *positions, double *out)
{
    for (unsigned is = 0; is < n_surfaces; ++is)
    {
        const uint32_t i0 = surface_offsets[is], i1 = surface_offsets[is + 1];
        v3 acc = {0, 0, 0};
        v3 d1 = orc_line_direction(positions, lines, surface_lines[i0]);
        const v3 d0 = d1;
        for (uint32_t k = i0 + 1; k < i1; ++k)
        {
            const v3 d2 = orc_line_direction(positions, lines, surface_lines[k]);
            acc = v3_add(acc, v3_cross(d2, d1));
            d1 = d2;
        }
        acc = v3_add(acc, v3_cross(d0, d1));
        const double inv = 1.0 / sqrt(v3_dot(acc, acc));
        v3_store(out + 3 * (size_t)is, v3_scale(acc, inv));
    }
}

/*
 * Element connectivity -> unique lines + signed ring->line CSR.
 * Restates mesh_from_elements, src/core/mesh.c:175-247: the k-th line of an element
 * runs from its vertex k-1 to vertex k; a line equal to an existing one in the same
 * direction gets orientation 0, in the opposite direction orientation 1, else a new
 * line is appended.  lines_out needs room for sum(counts) pairs,
 * surface_lines_out for sum(counts) entries, offsets_out for n_elements+1.
 * Returns the number of unique lines.
 */
unsigned orc_mesh_from_elements(unsigned n_elements, const uint32_t *counts,
                                const uint32_t *flat, uint32_t *lines_out,
                                uint32_t *surface_lines_out, uint32_t *offsets_out)
{
    /* The reference scans every existing line for a match (O(E*L)); a line can
     * match at most one existing line, so an open-addressing table keyed on the
     * unordered node pair gives the same line numbering and orientations. */
    unsigned total = 0;
    for (unsigned ie = 0; ie < n_elements; ++ie)
        total += counts[ie];
    unsigned cap = 16;
    while (cap < 2 * total + 16)
        cap <<= 1;
    uint32_t *table = malloc(sizeof(uint32_t) * cap);
    if (!table)
        return 0xFFFFFFFFu;
    memset(table, 0xFF, sizeof(uint32_t) * cap);
    unsigned n_lines = 0, offset = 0;
    offsets_out[0] = 0;
    for (unsigned ie = 0; ie < n_elements; ++ie)
    {
        const unsigned n = counts[ie];
        uint32_t left = flat[offset + n - 1];
        for (unsigned ip = 0; ip < n; ++ip)
        {
            const uint32_t right = flat[offset + ip];
            const uint64_t lo = left < right ? left : right, hi = left < right ? right : left;
            uint64_t hsh = (lo * 0x9E3779B97F4A7C15ull) ^ (hi * 0xC2B2AE3D27D4EB4Full);
            unsigned slot = (unsigned)(hsh >> 17) & (cap - 1);
            uint32_t il = 0xFFFFFFFFu, orient = 0;
            while (table[slot] != 0xFFFFFFFFu)
            {
                const uint32_t c = table[slot];
                if (lines_out[2 * c] == left && lines_out[2 * c + 1] == right)
                {
                    il = c;
                    orient = 0;
                    break;
                }
                if (lines_out[2 * c + 1] == left && lines_out[2 * c] == right)
                {
                    il = c;
                    orient = 1;
                    break;
                }
                slot = (slot + 1) & (cap - 1);
            }
            if (il == 0xFFFFFFFFu)
            {
                il = n_lines;
                lines_out[2 * n_lines] = left;
                lines_out[2 * n_lines + 1] = right;
                table[slot] = n_lines;
                n_lines += 1;
            }
            surface_lines_out[offset + ip] = (orient << 31) | il;
            left = right;
        }
        offset += n;
        offsets_out[ie + 1] = offset;
    }
    free(table);
    return n_lines;
}

/*
 * Dual lines: for each primal line, the rings on either side.  Restates the first
 * half of mesh_dual_from_primal, src/core/mesh.c:88-111: the ring holding the line
 * reversed goes to slot 0, the ring holding it forward to slot 1
 * (surf_ids[!orientation]); at most two rings are recorded, scanning rings in order;
 * a missing side is INVALID_ID.  dual_lines_out is (n_lines, 2).
 */
void orc_dual_lines(unsigned n_lines, unsigned n_surfaces, const uint32_t *surface_offsets,
                    const uint32_t *surface_lines, uint32_t *dual_lines_out)
{
    for (unsigned il = 0; il < n_lines; ++il)
    {
        uint32_t ids[2] = {ORC_INVALID, ORC_INVALID};
        unsigned cnt = 0;
        for (unsigned is = 0; is < n_surfaces && cnt < 2; ++is)
        {
            for (uint32_t k = surface_offsets[is]; k < surface_offsets[is + 1]; ++k)
            {
                const uint32_t g = surface_lines[k];
                if (ORC_IDX(g) == il)
                {
                    ids[!ORC_REV(g)] = is;
                    cnt += 1;
                    break;
                }
            }
        }
        dual_lines_out[2 * il + 0] = ids[0];
        dual_lines_out[2 * il + 1] = ids[1];
    }
}

/*
 * Kutta-Joukowski line forces.  Restates Mesh.line_forces, src/meshobject.c:1368-1393:
 *   c = circ[dual.p1] - circ[dual.p2] (INVALID sides skipped)
 *   F = (r_end - r_begin) x (0.5 * c * (v[p1] + v[p2]))
 * circ is the ring circulation already divided by 2*pi by the caller.
 */
void orc_line_forces(unsigned n_lines, const uint32_t *primal_lines, const uint32_t *dual_lines,
                     const double *circ, const double *positions, const double *velocity,
                     double *out)
{
    for (unsigned il = 0; il < n_lines; ++il)
    {
        const uint32_t p1 = ORC_IDX(primal_lines[2 * il]), p2 = ORC_IDX(primal_lines[2 * il + 1]);
        const uint32_t d1 = ORC_IDX(dual_lines[2 * il]), d2 = ORC_IDX(dual_lines[2 * il + 1]);
        const v3 dr = v3_sub(v3_load(positions + 3 * (size_t)p2), v3_load(positions + 3 * (size_t)p1));
        double c = 0;
        if (d1 != ORC_INVALID)
            c += circ[d1];
        if (d2 != ORC_INVALID)
            c -= circ[d2];
        const v3 avg = v3_scale(v3_add(v3_load(velocity + 3 * (size_t)p1), v3_load(velocity + 3 * (size_t)p2)),
                                0.5 * c);
        v3_store(out + 3 * (size_t)il, v3_cross(dr, avg));
    }
}
