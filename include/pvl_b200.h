/*
 * pyvl_b200 -- C ABI of the B200-native UVLM hot path (libpvl_b200.so).
 *
 * Plain pointers and sizes only.  Every entry point returns an int status (PVL_OK = 0,
 * negative on failure; pvl_last_error() gives the message of the calling thread's last
 * failure).  "Device" arguments are CUDA device pointers; `stream` is a cudaStream_t
 * passed as void* (NULL = legacy default stream).  Device entry points only enqueue
 * work: they never synchronise and never allocate; scratch memory comes from the
 * caller through (ws, ws_bytes) pairs sized by the matching *_workspace() query.
 *
 * Geometry ids follow the reference's geo_id_t (src/core/common.h:46-56): bits 0-30
 * index, bit 31 = reversed orientation; PVL_INVALID_ID = 0x7FFFFFFF.  A mesh is the
 * reference's mesh_t CSR (src/core/mesh.h:130-139): lines (n_lines x 2 uint32, point
 * ids), surface_offsets (n_surfaces + 1 uint32), surface_lines (geo ids of lines).
 * Point arrays are (n, 3) float64 row-major like the reference's real3_t arrays.
 *
 * Each declaration names the reference routine it replaces (file:line within the
 * reference project).
 */
#ifndef PVL_B200_H
#define PVL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    PVL_OK = 0,
    PVL_ERR_ARG = -1,           /* invalid argument (the reference raises ValueError/TypeError) */
    PVL_ERR_CUDA = -2,          /* CUDA runtime error */
    PVL_ERR_ALLOC = -3,         /* workspace too small / host allocation failed */
    PVL_ERR_SINGULAR = -4,      /* exactly zero pivot met by the LU factorisation */
    PVL_ERR_NOT_CONVERGED = -5, /* an iterative solve missed its tolerance */
    PVL_ERR_TOPOLOGY = -6,      /* topology construction failed (RuntimeError in the reference) */
    PVL_ERR_TIMEOUT = -7,       /* a device-side wait gave up (bounded spin) */
    PVL_ERR_NONFINITE = -8      /* a NaN or infinity reached the system (set by pvl_rhs through its status word) */
};

enum { PVL_F64 = 0, PVL_F32 = 1 };

#define PVL_INVALID_ID 0x7FFFFFFFu

/* Message of the calling thread's most recent failure ("" if none). */
const char* pvl_last_error(void);
/* ABI version (major * 100 + minor). */
int pvl_version(void);

/* ------------------------------------------------------------------ host topology */

/* Element connectivity -> unique lines + signed ring->line CSR.
 * Replaces mesh_from_elements (src/core/mesh.c:175-247) and the validation of
 * Mesh.__new__ (src/meshobject.c:41-116): every element needs >= 3 points and point ids
 * may not exceed n_points (the reference's own bound, meshobject.c:90).  Line numbering
 * and orientation bits are identical to the reference's (first appearance order).
 * lines_out: 2 * sum(counts) uint32; surface_lines_out: sum(counts); offsets_out:
 * n_elements + 1.  Runs in O(sum(counts)) with a hash of unordered node pairs. */
int pvl_mesh_from_elements(uint32_t n_points, uint32_t n_elements, const uint32_t* counts,
                           const uint32_t* flat_points, uint32_t* lines_out,
                           uint32_t* surface_lines_out, uint32_t* offsets_out,
                           uint32_t* n_lines_out);

/* Dual mesh: dual line i = the rings on either side of primal line i (slot 0: ring holding
 * it reversed, slot 1: ring holding it forward; INVALID_ID where missing); dual surface p =
 * the lines touching primal point p (orientation 0 where p is the line's first point).
 * Replaces mesh_dual_from_primal (src/core/mesh.c:70-173), O(total) instead of O(L*S).
 * dual_lines_out: 2 * n_lines; dual_offsets_out: n_points + 1;
 * dual_surface_lines_out: 2 * n_lines. */
int pvl_mesh_dual(uint32_t n_points, uint32_t n_lines, const uint32_t* lines,
                  uint32_t n_surfaces, const uint32_t* surface_offsets,
                  const uint32_t* surface_lines, uint32_t* dual_lines_out,
                  uint32_t* dual_offsets_out, uint32_t* dual_surface_lines_out);

/* Mesh -> element connectivity (point counts and flattened loops).
 * Replaces mesh_to_elements (src/core/mesh.c:249-301).  counts_out: n_surfaces;
 * flat_out: surface_offsets[n_surfaces]. */
int pvl_mesh_to_elements(uint32_t n_surfaces, const uint32_t* surface_offsets,
                         const uint32_t* surface_lines, const uint32_t* lines,
                         uint32_t* counts_out, uint32_t* flat_out);

/* Inverse of the ring->line CSR: for each line the signed ids of the rings that hold it
 * (bit 31 set where the ring holds the line reversed), rings in ascending order.  Used to
 * turn ring circulations into line circulations.  No reference counterpart; it is the
 * transpose of the CSR the reference reduces over (src/core/flow_solver.c:141-205).
 * map_offsets_out: n_lines + 1; map_entries_out: surface_offsets[n_surfaces]. */
int pvl_line_ring_map(uint32_t n_lines, uint32_t n_surfaces, const uint32_t* surface_offsets,
                      const uint32_t* surface_lines, uint32_t* map_offsets_out,
                      uint32_t* map_entries_out);

/* ------------------------------------------------------------------ device geometry */

/* Unit ring normals (n_surfaces, 3).  Replaces surface_normal (src/core/mesh.c:48-68) as
 * called by Mesh.surface_normal (src/meshobject.c:956-1008). */
int pvl_surface_normal(uint32_t n_surfaces, const uint32_t* surface_offsets,
                       const uint32_t* surface_lines, const uint32_t* lines,
                       const double* positions, double* out, void* stream);

/* Per-ring mean of a per-point vec3 (n_surfaces, 3).  Replaces surface_center
 * (src/core/mesh.c:24-46) as called by Mesh.surface_average_vec3 (src/meshobject.c:1010-1062). */
int pvl_surface_average(uint32_t n_surfaces, const uint32_t* surface_offsets,
                        const uint32_t* surface_lines, const uint32_t* lines,
                        const double* values, double* out, void* stream);

/* No-penetration right-hand side b_i = n_i . (-(U_i - v_i)) with U_i = flow[i] when
 * flow != NULL else (ux, uy, uz); cp_velocity may be NULL (zero).  When `nonfinite` is not
 * NULL, any b_i that is a NaN or an infinity (a NaN or infinity in a position, a velocity or the
 * stream of an element) sets *nonfinite = 1; the word is never cleared here, so it holds the
 * error until the caller reads and resets it.
 * Replaces python/pyvl/solver.py:199-206 (where a NaN propagates silently). */
int pvl_rhs(uint32_t n, const double* normals, const double* flow, double ux, double uy,
            double uz, const double* cp_velocity, double* rhs_out, int32_t* nonfinite, void* stream);

/* ------------------------------------------------------------------ induction */

/* Scratch for the segment table of n_lines segments at `precision`. */
size_t pvl_segments_workspace(uint32_t n_lines, int precision);

/* Line induction matrix (n_cp, n_lines, 3) float64: every (segment, point) pair.
 * Replaces compute_line_induction (src/core/flow_solver.c:86-139) as called by
 * Mesh.line_induction_matrix (src/meshobject.c:1232-1286). */
int pvl_line_induction(uint32_t n_points, uint32_t n_lines, const uint32_t* lines,
                       const double* positions, uint32_t n_cp, const double* cps, double tol,
                       double* out, void* ws, size_t ws_bytes, void* stream);

/* Ring induction matrix (n_cp, n_surfaces, 3) float64, fused pair + signed ring sum (no
 * line buffer).  Replaces Mesh.induction_matrix (src/meshobject.c:475-556):
 * compute_line_induction + line_induction_to_surface_induction (flow_solver.c:141-172). */
int pvl_induction_matrix(uint32_t n_points, uint32_t n_lines, const uint32_t* lines,
                         const double* positions, uint32_t n_surfaces,
                         const uint32_t* surface_offsets, const uint32_t* surface_lines,
                         uint32_t n_cp, const double* cps, double tol, double* out, void* ws,
                         size_t ws_bytes, void* stream);

/* Normal ring induction matrix out[i * ld + j] = n_i . sum_{k in ring j} +-u_k(cp_i),
 * fused (no line buffer); `out_precision` selects float64 or float32 output and
 * arithmetic.  Replaces Mesh.induction_matrix3 (src/meshobject.c:384-473):
 * compute_line_induction + line_induction_to_normal_surface_induction
 * (flow_solver.c:174-205). */
int pvl_induction_normal(int precision, uint32_t n_points, uint32_t n_lines, const uint32_t* lines,
                         const double* positions, uint32_t n_surfaces,
                         const uint32_t* surface_offsets, const uint32_t* surface_lines,
                         uint32_t n_cp, const double* cps, const double* normals, double tol,
                         void* out, uint32_t ld, void* ws, size_t ws_bytes, void* stream);

/* Scratch for pvl_line_velocity. */
/* pvl_induction_normal (FP64) with each line evaluated once per control point: rings in
 * tiles of 128 consecutive rings; tile t's distinct lines are tile_lines[tile_offsets[t] ..
 * tile_offsets[t+1]), sl_local[k] is the position of CSR entry k (surface_lines[k]) in its
 * tile's list, max_tile_lines the largest list (Mesh.ring_tiles builds the three).  Same
 * matrix as pvl_induction_normal to rounding (per-line dot products summed per ring).
 * ws: pvl_segments_workspace(n_lines, PVL_F64) bytes. */
int pvl_induction_normal_tiled(uint32_t n_points, uint32_t n_lines, const uint32_t* lines, const double* positions,
                               uint32_t n_surfaces, const uint32_t* offsets, const uint32_t* surface_lines,
                               const uint32_t* tile_offsets, const uint32_t* tile_lines, const uint32_t* sl_local,
                               uint32_t max_tile_lines, uint32_t n_cp, const double* cps, const double* normals,
                               double tol, double* out, uint32_t ld, void* ws, size_t ws_bytes, void* stream);

size_t pvl_line_velocity_workspace(uint32_t n_lines, uint32_t n_pts, int precision);

/* Velocity induced at points by segments carrying circulations:
 *   v(p) = sum_k gamma_k u_k(p)   (line_gamma == NULL: gamma_k = 1)
 * and, with normals != NULL, the projection n_p . v(p).  out is (n_pts, 3) or (n_pts,);
 * out = beta * out + alpha * v.  This is the contraction sum_j K_ij Gamma_j the reference
 * forms from a materialised (n_pts, n_surfaces, 3) matrix and numpy's vecdot
 * (python/pyvl/wake_models.py:125-126, 170-175, 219-223; solver.py:274-279), evaluated
 * per segment with gamma_k = sum of the signed ring circulations of the rings holding k. */
int pvl_line_velocity(int precision, uint32_t n_points, uint32_t n_lines, const uint32_t* lines,
                      const double* positions, const double* line_gamma, uint32_t n_pts,
                      const double* pts, const double* normals, double tol, double alpha,
                      double beta, double* out, void* ws, size_t ws_bytes, void* stream);

/* Size of the static device array behind pvl_line_velocity_noalloc (32 MiB). */
#define PVL_NOALLOC_SCRATCH_BYTES (32u << 20)

/* pvl_line_velocity without a workspace, for callers that cannot allocate device memory
 * (hosts that own all device memory through their own pool, or loops where an allocation
 * and the synchronisation of a cudaFree are not acceptable).  No counterpart in the
 * reference.  Same arguments and result as pvl_line_velocity minus (ws, ws_bytes): the
 * scratch is a file-scope device array of PVL_NOALLOC_SCRATCH_BYTES that every GPU loading
 * the library keeps until exit.  Calls needing more scratch than that are rejected with
 * PVL_ERR_ARG.  All calls share the array, so calls whose kernels overlap on the GPU race;
 * calls ordered on one stream are safe.  The first call on a device looks up the array's
 * address (cudaGetSymbolAddress); make it before any stream capture.  Allocates nothing. */
int pvl_line_velocity_noalloc(int precision, uint32_t n_points, uint32_t n_lines,
                              const uint32_t* lines, const double* positions,
                              const double* line_gamma, uint32_t n_pts, const double* pts,
                              const double* normals, double tol, double alpha, double beta,
                              double* out, void* stream);

/* Line circulations gamma_line[k] = sum over the rings holding line k of +-gamma_ring
 * (sign from the orientation bit).  With ring_period > 0, rings whose index is a multiple
 * of ring_period are skipped (the implicit first wake row).  Uses pvl_line_ring_map. */
int pvl_line_circulation(uint32_t n_lines, const uint32_t* map_offsets,
                         const uint32_t* map_entries, const double* ring_gamma,
                         uint32_t ring_period, double* line_gamma_out, void* stream);

/* ------------------------------------------------------------------ free wake */

/* Fold the implicit wake row into the system matrix:
 *   A[:, adj[s,1]] -= implicit[:, s];  A[:, adj[s,0]] += implicit[:, s]
 * for s = 0..n_shed-1 in order, INVALID_ID sides skipped.  implicit is (n_cp, n_shed).
 * Replaces python/pyvl/wake_models.py:204-216. */
int pvl_wake_fold_implicit(uint32_t n_cp, uint32_t n_shed, const double* implicit,
                           const uint32_t* adjacent, double* A, uint32_t lda, void* stream);

/* pvl_wake_fold_implicit in parallel over (row, shedding line), for adjacency tables in which
 * every ring appears at most once over all shedding lines and sides (the caller checks; true
 * for wings, where each trailing-edge ring has one shedding edge).  Same result. */
int pvl_wake_fold_implicit_distinct(uint32_t n_cp, uint32_t n_shed, const double* implicit,
                                    const uint32_t* adjacent, double* A, uint32_t lda, void* stream);

/* Velocity of the wake nodes that advect this step: for every (s, side) and row
 * i < complete_rows, node_vel[(s*2 + side)*complete_rows + i] = U_inf + sum_k gamma_k u_k(node)
 * with the body segments (lines, positions, line_gamma).  wake_pos is (n_shed, 2,
 * line_rows + 1, 3).  Replaces the per-row loop of python/pyvl/wake_models.py:120-126
 * (FlowConditions.get_velocity + induction_matrix @ circulation) for a uniform U_inf. */
size_t pvl_wake_node_velocity_workspace(uint32_t n_lines, uint32_t n_shed, uint32_t complete_rows,
                                        int precision);
int pvl_wake_node_velocity(int precision, uint32_t n_points, uint32_t n_lines, const uint32_t* lines,
                           const double* positions, const double* line_gamma, uint32_t n_shed,
                           uint32_t line_rows, uint32_t complete_rows, const double* wake_pos,
                           double ux, double uy, double uz, double tol, double* node_vel, void* ws,
                           size_t ws_bytes, void* stream);

/* pvl_wake_node_velocity restricted to rows [row_begin, row_end) of n_cols node columns:
 * column c is wake node column cols[c] (strip side s * 2 + side, < 2 n_shed; cols == NULL
 * means all 2 n_shed columns in order).  Output node_vel[(c * complete_rows + i) * 3 + k] for
 * the listed rows; other rows untouched.  Lets co-located node columns (adjacent strips share
 * their trailing-edge node, and identical positions advect identically) be evaluated once,
 * and near and far rows run in different precisions.  Workspace:
 * pvl_line_velocity_workspace(n_lines, n_cols (row_end - row_begin), precision).  No
 * reference counterpart (the reference evaluates every node of every row). */
int pvl_wake_node_velocity_cols(int precision, uint32_t n_points, uint32_t n_lines, const uint32_t* lines,
                                const double* positions, const double* line_gamma, uint32_t n_shed,
                                uint32_t line_rows, uint32_t complete_rows, uint32_t row_begin,
                                uint32_t row_end, uint32_t n_cols, const uint32_t* cols, const double* wake_pos,
                                double ux, double uy, double uz, double tol, double* node_vel, void* ws,
                                size_t ws_bytes, void* stream);

/* pvl_wake_node_velocity_cols for rows row_begin + k * row_step, k < row_count (each < complete_rows)
 * of the n_cols node columns; output at the same rows of node_vel.  Workspace:
 * pvl_line_velocity_workspace(n_lines, n_cols row_count, precision).  Used with
 * pvl_wake_interp_rows for the far wake rows, whose body-induced velocity varies slowly along a
 * node column.  No reference counterpart. */
int pvl_wake_node_velocity_rows(int precision, uint32_t n_points, uint32_t n_lines, const uint32_t* lines,
                                const double* positions, const double* line_gamma, uint32_t n_shed,
                                uint32_t line_rows, uint32_t complete_rows, uint32_t row_begin,
                                uint32_t row_count, uint32_t row_step, uint32_t n_cols, const uint32_t* cols,
                                const double* wake_pos, double ux, double uy, double uz, double tol,
                                double* node_vel, void* ws, size_t ws_bytes, void* stream);

/* pvl_wake_node_velocity_rows for the rows listed in `rows` (device array of n_rows row
 * indices; an entry at or past complete_rows is skipped, its nodes left as they are) of the n_cols
 * listed node columns; output at the same rows of node_vel (n_cols, complete_rows, 3).
 * Workspace: pvl_line_velocity_workspace(n_lines, n_cols n_rows, precision).  One sweep for rows
 * that no single stride covers (the mixed path's far rows).  No reference counterpart. */
int pvl_wake_node_velocity_list(int precision, uint32_t n_points, uint32_t n_lines, const uint32_t* lines,
                                const double* positions, const double* line_gamma, uint32_t n_shed,
                                uint32_t line_rows, uint32_t complete_rows, uint32_t n_rows, const uint32_t* rows,
                                uint32_t n_cols, const uint32_t* cols, const double* wake_pos, double ux, double uy,
                                double uz, double tol, double* node_vel, void* ws, size_t ws_bytes, void* stream);

/* node_vel (n_cols, complete_rows, 3): rows row_first, row_first + 2, ... <= row_last of every
 * column set to the midpoint value of the cubic through the same column's rows -3, -1, +1 and +3
 * away ((9 (v[-1] + v[+1]) - (v[-3] + v[+3])) / 16); needs row_first >= 3 and
 * row_last + 3 < complete_rows.  The mixed path's far-row advection (no reference
 * counterpart: the reference evaluates every node). */
int pvl_wake_interp_rows(uint32_t n_cols, uint32_t complete_rows, uint32_t row_first, uint32_t row_last,
                         double* node_vel, void* stream);

/* pvl_wake_interp_rows at spacing `half` (> 0): rows row_first, row_first + 2 half, ... <= row_last
 * from the same column's rows -3 half, -half, +half, +3 half away; needs row_first >= 3 half and
 * row_last + 3 half < complete_rows.  With half = 2 it fills the rows midway between rows
 * evaluated every fourth row, before the odd rows are filled with half = 1. */
int pvl_wake_interp_rows_spaced(uint32_t n_cols, uint32_t complete_rows, uint32_t row_first, uint32_t row_last,
                                uint32_t half, double* node_vel, void* stream);

/* node_vel[c, r] = sum_{k in [offsets[c], offsets[c+1])} weights[k] sub_vel[entries[k], r] for the
 * rows r in [row_begin, row_end) of every column c < n_cols; node_vel is (n_cols, complete_rows, 3)
 * and sub_vel (n_sub, complete_rows, 3), the velocities of the wake nodes of some columns (from
 * pvl_wake_node_velocity_rows with those columns' list).  offsets has n_cols + 1 entries, entries
 * and weights n_entries; a range outside [0, n_entries) or an entry outside [0, n_sub) writes NaN.
 * The mixed path's advection of far rows at every other node column (no reference counterpart:
 * the reference evaluates every node). */
int pvl_wake_interp_cols(uint32_t n_cols, uint32_t complete_rows, uint32_t row_begin, uint32_t row_end,
                         const uint32_t* offsets, uint32_t n_entries, const uint32_t* entries,
                         const double* weights, uint32_t n_sub, const double* sub_vel, double* node_vel,
                         void* stream);

/* out[k] = pts[index[k]] (3 doubles each) for k < n; an index outside [0, n_pts) writes NaN.
 * Gathers the control points at which the mixed path evaluates the far wake term.  No
 * reference counterpart. */
int pvl_gather_points(uint32_t n, const uint32_t* index, uint32_t n_pts, const double* pts, double* out,
                      void* stream);

/* out[p] += n_p . sum_{k in [offsets[p], offsets[p+1])} weights[k] values[entries[k]] for p < n_cp:
 * velocities (values, (n_values, 3)) known at some points, interpolated to every control point
 * by a stencil and projected on its normal (normals (n_cp, 3)), terms summed in stored order.
 * offsets has n_cp + 1 entries, entries and weights n_entries; a range outside [0, n_entries)
 * or an entry outside [0, n_values) makes the point's result NaN.  The mixed path's far wake
 * term (the reference evaluates the wake at every control point,
 * python/pyvl/wake_models.py:219-223). */
int pvl_stencil_normal_add(uint32_t n_cp, const uint32_t* offsets, uint32_t n_entries, const uint32_t* entries,
                           const double* weights, uint32_t n_values, const double* values, const double* normals,
                           double* out, void* stream);

/* Advance wake node rows (explicit Euler) from `old_pos` into `new_pos` (both
 * (n_shed, 2, line_rows + 1, 3)): new[:, :, i+1] = old[:, :, i] + node_vel[:, :, i] * dt for
 * i < complete_rows; row 0 pinned to the bordering body nodes; rows beyond complete_rows
 * collapsed onto row complete_rows.  node_vel is (n_shed, 2, complete_rows, 3) and already
 * holds U_inf + body induction.  Replaces python/pyvl/wake_models.py:113-137. */
int pvl_wake_advect(uint32_t n_shed, uint32_t line_rows, uint32_t complete_rows,
                    const double* old_pos, const double* node_vel, double dt,
                    const double* body_positions, const uint32_t* bordering_nodes,
                    double* new_pos, void* stream);

/* pvl_wake_advect with node column s * 2 + side reading its velocity row from slot
 * col_slot[s * 2 + side] of node_vel ((n_slots, complete_rows, 3)), as written by
 * pvl_wake_node_velocity_cols for a de-duplicated column list. */
int pvl_wake_advect_cols(uint32_t n_shed, uint32_t line_rows, uint32_t complete_rows,
                         const double* old_pos, const double* node_vel, const uint32_t* col_slot,
                         uint32_t n_slots, double dt, const double* body_positions,
                         const uint32_t* bordering_nodes, double* new_pos, void* stream);

/* Shift wake circulations one row back and shed the new first row
 *   circ[:, 0] = gamma[adj[:,1]] - gamma[adj[:,0]]   (INVALID_ID sides skipped)
 * into new_circ (n_shed, line_rows) from old_circ.  Replaces wake_models.py:139-151. */
int pvl_wake_shed(uint32_t n_shed, uint32_t line_rows, const double* old_circ,
                  const uint32_t* adjacent, const double* gamma, double* new_circ, void* stream);

/* ------------------------------------------------------------------ dense solve */

/* Scratch for pvl_lu_factor / pvl_lu_solve. */
size_t pvl_lu_workspace(uint32_t n);
size_t pvl_lu_solve_workspace(uint32_t n);

/* In-place LU with partial pivoting of the row-major n x n matrix A (leading dimension
 * lda): P A = L U with unit-lower L.  ipiv (device int32, 2n entries) receives in its first
 * n entries the LAPACK interchange sequence (ipiv[k] = row swapped with row k, 0-based) and
 * in the next n the resulting row permutation (row i of P A is row perm[i] of A).  info
 * (device int32) receives 0, or k+1 when U[k,k] == 0 (getrf convention).  FP64 throughout;
 * the pivots are exactly those of partial pivoting (first maximal |entry| per column).
 * Replaces scipy.linalg.lu_factor (python/pyvl/solver.py:223). */
int pvl_lu_factor(uint32_t n, double* A, uint32_t lda, int32_t* ipiv, int32_t* info, void* ws,
                  size_t ws_bytes, void* stream);

/* Solve A x = b in place in b (device, n) with the factors and ipiv of pvl_lu_factor.  ws
 * must be the workspace the factorisation ran with, unchanged since: it holds the inverted
 * 64 x 64 diagonal blocks of L and U.  err (device int32) receives 0, or 1 if a wait between
 * row blocks timed out.
 * Replaces scipy.linalg.lu_solve (python/pyvl/solver.py:227). */
int pvl_lu_solve(uint32_t n, const double* LU, uint32_t lda, const int32_t* ipiv, double* b,
                 int32_t* err, void* ws, size_t ws_bytes, void* stream);
/* The same solve by blocked substitution, one launch per 64-row block step and no waits
 * between CTAs (usable inside a conditional node of a CUDA graph); slower than the wavefront. */
int pvl_lu_solve_blocked(uint32_t n, const double* LU, uint32_t lda, const int32_t* ipiv, double* b,
                         void* ws, size_t ws_bytes, void* stream);

/* Remove the mean of x over each group g: x[off[g]:off[g+1]] -= mean.  Replaces the
 * closed-body constraint of python/pyvl/solver.py:229-233. */
int pvl_group_mean_remove(uint32_t n_groups, const uint32_t* group_offsets, double* x,
                          void* stream);

/* Border an n x n system for zero-mean circulation on m groups: with A of leading
 * dimension lda >= n + m, sets A[i, n+g] = A[n+g, i] = 1 for i in group g, zero elsewhere
 * in the border, and rhs[n+g] = 0.  The bordered system is the well-posed form of the
 * reference's closed-body constraint (solver.py:229-233). */
int pvl_border_groups(uint32_t n, uint32_t m, const uint32_t* group_offsets, double* A,
                      uint32_t lda, double* rhs, void* stream);

/* ------------------------------------------------------------------ tensor cores */

/* C = alpha * A * B + beta * C on the 5th-generation tensor cores (tcgen05, accumulators in
 * tensor memory, operands brought in by TMA): FP32 storage, TF32 multiplication, FP32
 * accumulation.  Row-major A (M x K); B given as its transpose Bt (N x K, row-major), so that
 * both operands are K-major; row-major C (M x N).  Any M and N, K a positive multiple of 32,
 * leading dimensions multiples of 4 floats (and >= K, resp. N), 16-byte aligned bases.
 * err (device int32) is set to 1 if an internal wait timed out.  No reference counterpart: it
 * builds the low-precision preconditioner that replaces the per-step FP64 factorisation in
 * the mixed path. */
int pvl_gemm_tf32(uint32_t M, uint32_t N, uint32_t K, float alpha, const float* A, uint32_t lda,
                  const float* Bt, uint32_t ldbt, float beta, float* C, uint32_t ldc, int32_t* err,
                  void* stream);

/* ------------------------------------------------------------------ mixed-precision solve */

/* y = alpha * A x + beta * y with an FP64 (pvl_gemv_f64) or FP32 (pvl_gemv_f32mat) row-major
 * matrix; vectors and accumulation FP64.  The FP64 form computes the residuals of the
 * mixed-precision solve against the FP64 system; the FP32 form applies the approximate
 * inverse.  No reference counterpart (the reference factorises every step, solver.py:223). */
int pvl_gemv_f64(uint32_t rows, uint32_t cols, double alpha, const double* A, uint32_t lda,
                 const double* x, double beta, double* y, void* stream);
int pvl_gemv_f32mat(uint32_t rows, uint32_t cols, double alpha, const float* M, uint32_t ldm,
                    const double* x, double beta, double* y, void* stream);
/* The same with an FP32 vector x (the FP32 copy of a Krylov vector): the four products of each
 * 16-byte vector are summed in FP32, the row in FP64. */
int pvl_gemv_f32(uint32_t rows, uint32_t cols, double alpha, const float* M, uint32_t ldm, const float* x,
                 double beta, double* y, void* stream);

/* ------------------------------------------------------------------ device-driven GMRES graph */

/* Outcome of one solve of the GMRES graph, written by the device. */
typedef struct pvl_gmres_status {
    uint32_t iterations;          /* Krylov columns used */
    uint32_t converged;           /* 1: the final FP64 residual met tol; 0: the FP64 fallback ran */
    double initial_rel_residual;  /* ||b - A x0|| / ||b|| */
    double final_rel_residual;    /* ||r0 - sum_j y_j A z_j|| / ||b|| (= ||b - A x||) before any fallback */
} pvl_gmres_status;

/* Bytes of the device control block (8-byte aligned) and the largest max_iter. */
size_t pvl_gmres_ctl_bytes(void);
uint32_t pvl_gmres_max_iter(void);

/* Capture the whole mixed solve as one CUDA graph: r = b - A x (x holds the seed), right-
 * preconditioned flexible GMRES with the FP32 approximate inverse Minv (ldm) inside a
 * conditional WHILE node that the device ends (rotated residual <= tol ||b||, exhausted Krylov
 * space, or max_iter columns), x += Z y, the FP64 residual r0 - sum_j y_j W_j from the stored
 * products W_j = A z_j (b - A x without another pass over A), the status record, and in a
 * conditional IF node the FP64 fallback when that residual missed tol (pvl_lu_factor of A
 * in place and pvl_lu_solve_blocked of b in place, x = b).  Then gamma = x[0..n_gamma) and,
 * with n_groups, pvl_group_mean_remove.  Buffers (all device, fixed for the graph's life):
 * V (max_iter + 1) x n, Z and W max_iter x n, r0 and w n doubles, v32 n floats (16-byte aligned), ctl of
 * pvl_gmres_ctl_bytes(), ipiv 2n, info 1, ws >= pvl_lu_workspace(n).  *graph_out receives an
 * opaque handle.  No reference counterpart (the reference factorises every step,
 * python/pyvl/solver.py:223-227). */
int pvl_gmres_graph_create(uint32_t n, double* A, uint32_t lda, const float* Minv, uint32_t ldm, double* b,
                           double* x, double* V, double* Z, double* W, double* r0, double* w, float* v32, void* ctl,
                           uint32_t max_iter, double tol, int32_t* ipiv, int32_t* info, void* ws, size_t ws_bytes, double* gamma,
                           uint32_t n_gamma, uint32_t n_groups, const uint32_t* group_offsets,
                           pvl_gmres_status* status, uint64_t* graph_out);
/* Enqueue one solve on stream; counts the graph's fixed kernels in pvl_launch_count(). */
int pvl_gmres_graph_launch(uint64_t graph, void* stream);
/* Add the kernels of `iterations` Krylov columns (and of the fallback) to pvl_launch_count()
 * once the host has read a solve's status. */
int pvl_gmres_graph_account(uint64_t graph, uint32_t iterations, uint32_t fell_back);
int pvl_gmres_graph_destroy(uint64_t graph);

/* One classical Gram-Schmidt pass against the k rows of V (row stride ldv):
 * c = V w; w -= V^T c; h[0..k) += c.  h needs 2k doubles ([k, 2k) is scratch). */
int pvl_basis_project(uint32_t n, uint32_t k, const double* V, uint32_t ldv, double* w, double* h,
                      void* stream);

/* nrm[0] = ||w||_2 and, when v != NULL, v = w / ||w||. */
int pvl_normalize(uint32_t n, const double* w, double* v, double* nrm, void* stream);

/* x += sum_{i<k} c[i] Z_i (rows of Z, stride ldz; c on the device). */
int pvl_combine(uint32_t n, uint32_t k, const double* Z, uint32_t ldz, const double* c, double* x,
                void* stream);

/* y += alpha x (FP64). */
int pvl_axpy_f64(uint32_t n, double alpha, const double* x, double* y, void* stream);

/* b (npad x npad, row stride ldb, FP32) = a (n x n, FP64) padded with the identity: the input
 * of the FP32 factorisation (whose inverse needs a multiple of 64 rows). */
int pvl_pad_convert_f32(uint32_t n, const double* a, uint32_t lda, float* b, uint32_t ldb, uint32_t npad,
                        void* stream);

/* FP32 LU with partial pivoting of the n x n row-major A (in place), the low-precision
 * factorisation of the mixed path: the FP64 factorisation's panel/pivot/TRSM steps in FP32
 * and the trailing update on the tensor cores (pvl_gemm_tf32).  ipiv as pvl_lu_factor
 * (2n int32: LAPACK interchanges, then the row permutation).  lda a multiple of 4 and A
 * 16-byte aligned; ws of pvl_lu32_workspace(n) bytes, which keeps the inverted diagonal
 * blocks for pvl_lu32_inverse.  *err = 1 if a tensor-core wait timed out.  Replaces
 * scipy.linalg.lu_factor (solver.py:223) inside the preconditioner only. */
size_t pvl_lu32_workspace(uint32_t n);
int pvl_lu32_factor(uint32_t n, float* A, uint32_t lda, int32_t* ipiv, int32_t* info, int32_t* err,
                    void* ws, size_t ws_bytes, void* stream);

/* X = U^-1 L^-1 P from pvl_lu32_factor's factors (same ws, not modified in between):
 * blocked triangular inversion, diagonal blocks in FP32 on CUDA cores, rank-64 updates on the
 * tensor cores; with perm (the second half of ipiv) the row permutation is folded into X's
 * columns so that A^-1 b ~ X b (perm NULL: X = U^-1 L^-1).  Y (n x ldy) is scratch.  n a
 * multiple of 64; leading dimensions multiples of 4, arrays 16-byte aligned.  The mixed solve
 * applies X with pvl_gemv_f32mat. */
int pvl_lu32_inverse(uint32_t n, const float* LU, uint32_t lda, const int32_t* perm, float* X, uint32_t ldx,
                     float* Y, uint32_t ldy, int32_t* err, void* ws, size_t ws_bytes, void* stream);

/* ------------------------------------------------------------------ learned warm start */
/* The per-panel MLP that seeds the mixed solve: 12 inputs -> 128 -> 128 -> 1 (ReLU), BF16
 * weights and activations, FP32 accumulation.  params_bf16 / params are the flat parameter
 * vector (pvl_mlp_param_count() values: W1 128x12, b1, W2 128x128, b2, w3, b3) as BF16 and
 * as FP32.  No reference counterpart (the reference solves every step from scratch,
 * python/pyvl/solver.py:223-227). */
uint32_t pvl_mlp_param_count(void);
uint32_t pvl_mlp_input_count(void);

/* Inputs of each panel from the device state of a step: g0/g1 the circulations of the last
 * two steps, rem0/rem1 what those steps' solutions added to their own Jacobi corrections,
 * resid = b - A g0 for the new system (A, lda; rhs = b) and rnorm[0] = ||resid||, rhs_prev
 * the last step's RHS, normals and control-point velocities ((n, 3) each).  Increments are
 * divided by s = ||resid|| / sqrt(n).  X (n, 12) = (input - mean) * inv_std;
 * base = g0 + resid / diag(A) (one Jacobi correction). */
int pvl_mlp_features(uint32_t n, const double* g0, const double* g1, const double* rem0, const double* rem1,
                     const double* resid, const double* rnorm, const double* A, uint32_t lda, const double* rhs, const double* rhs_prev,
                     const double* normals, const double* cp_vel, const float* mean, const float* inv_std,
                     float* X, double* base, void* stream);

/* out[i] = base[i] + scale * mul[0] * mlp(X[i]) (base and mul may be NULL; mul on the device). */
int pvl_mlp_forward(uint32_t n, const float* X, const void* params_bf16, double scale, const double* mul,
                    const double* base, double* out, void* stream);

/* grad = d/dparams mean_i (mlp(X[i]) - T[i])^2 and *loss (device floats; loss may be NULL),
 * over n samples with up to n_ctas persistent CTAs; ws of pvl_mlp_train_workspace(n_ctas)
 * bytes.  The partial gradients of the CTAs are summed in a fixed order. */
size_t pvl_mlp_train_workspace(uint32_t n_ctas);
int pvl_mlp_gradient(uint32_t n, const float* X, const float* T, const void* params_bf16, uint32_t n_ctas,
                     float* grad, float* loss, void* ws, size_t ws_bytes, void* stream);

/* One Adam step (step >= 1) on the FP32 parameters with moments m, v; refreshes the BF16 copy. */
int pvl_mlp_adam(float* params, void* params_bf16, const float* grad, float* m, float* v, uint32_t step,
                 float lr, float beta1, float beta2, float eps, void* stream);

/* params_bf16 = BF16(params). */
int pvl_mlp_to_bf16(const float* params, void* params_bf16, void* stream);

/* ------------------------------------------------------------------ batched cases */
/* Many independent cases of uneven size stepped with one launch per kernel over the whole
 * batch (persistent CTAs taking work items from an atomic counter).  The batch is one
 * concatenated mesh plus device job tables that keep each case's pairs inside the case; the
 * table records are the structs of csrc/batch.cu, whose sizes the *_bytes() queries return
 * (the host packs them with the same field order: see pyvl_b200/batch.py).  No reference
 * counterpart: the reference steps one geometry per solver loop (solver.py:145-265). */
size_t pvl_batch_ring_job_bytes(void);
size_t pvl_batch_sweep_job_bytes(void);
size_t pvl_batch_wake_case_bytes(void);
size_t pvl_batch_solve_case_bytes(void);
size_t pvl_batch_gmres_state_bytes(void);
uint32_t pvl_batch_gmres_max_iter(void);

/* Segment table (pvl_segments_workspace bytes) of a line set: r1, r2, unit direction,
 * length (negative below tol), line circulation (1 when line_gamma is NULL). */
int pvl_prep_segments(int precision, uint32_t n_points, uint32_t n_lines, const uint32_t* lines,
                      const double* positions, const double* line_gamma, double tol, void* segments,
                      void* stream);

/* Ring-matrix blocks of every job: out[job.out_begin + i*ld + j] = n_i . sum_{k in ring j} +-u_k(cp_i)
 * (FP64).  cpb = control points per CTA (4, 8 or 16; the autotuner's choice); n_ctas 0 = fill
 * the GPU.  counter: one device uint32 (reset by the call). */
int pvl_batch_ring_matrix(int cpb, const void* jobs, const uint32_t* job_item, uint32_t n_jobs, uint32_t n_items,
                          uint32_t* counter, const uint32_t* offsets, const uint32_t* surface_lines,
                          uint32_t n_lines, const void* segments, const double* cps, const double* normals,
                          double tol, double* out, uint32_t n_ctas, void* stream);
/* The same blocks with each distinct line of a 128-ring column tile evaluated once per control
 * point (the batched form of pvl_induction_normal_tiled): job_tile[j] = first tile of job j
 * (its column tiles are consecutive), tile_offsets / tile_lines = the tiles' distinct lines,
 * sl_local = each CSR entry's position in its tile's list, max_tile_lines = the longest list;
 * cpb = 8, 16 or 32 control points per CTA (shared memory cpb * max_tile_lines doubles).
 * fold_adj != NULL (implicit wake blocks): instead of storing entry (i, j), fold it into the
 * case's matrix (out_begin, ld of the jobs = the matrix) as pvl_batch_fold_implicit does,
 * A[i, adj[2r + 1]] -= v, A[i, adj[2r]] += v with r the ring's CSR row (its shedding line);
 * only when no body ring is adjacent to two shedding-line sides of its case. */
int pvl_batch_ring_matrix_tiled(int cpb, const void* jobs, const uint32_t* job_item, uint32_t n_jobs,
                                uint32_t n_items, uint32_t* counter, const uint32_t* offsets,
                                const uint32_t* surface_lines, const uint32_t* sl_local, const uint32_t* job_tile,
                                const uint32_t* tile_offsets, const uint32_t* tile_lines, uint32_t max_tile_lines,
                                uint32_t n_lines, const void* segments, const double* cps, const double* normals,
                                double tol, const uint32_t* fold_adj, double* out, uint32_t n_ctas, void* stream);

/* Segment sweeps of every job into per-job partials (FP64); tile = (threads, points per
 * thread) in {(128,1),(128,2),(128,4),(256,1),(256,2)}; rows: device uint32 (the step's row
 * count for jobs whose point count grows with the wake).  A job with seg_rows set has its
 * segments in row order and sweeps only the first seg_upto[seg_rows + min(*rows, rows_max)]
 * of them (seg_upto: device table of the row prefixes; NULL sweeps every segment). */
int pvl_batch_sweep(int threads, int ppt, const void* jobs, const uint32_t* job_item, uint32_t n_jobs,
                    uint32_t n_items, uint32_t* counter, const uint32_t* rows, const uint32_t* seg_upto,
                    uint32_t rows_max, const void* segments, const double* pts, const uint32_t* pidx, double tol,
                    double* partials, uint32_t n_ctas, void* stream);

/* Reduce the sweeps' partials: mode 0 jobs add n . v to out (the RHS), mode 1 jobs write
 * U_case + v (node velocities; uinf is (n_cases, 3)).  pt_item: first thread of each job. */
int pvl_batch_sweep_reduce(const void* jobs, const uint32_t* pt_item, uint32_t n_jobs, uint32_t n_total,
                           const uint32_t* rows, const double* partials, const double* normals,
                           const double* uinf, double* out, void* stream);

/* Per-case wake bookkeeping of pvl_wake_fold_implicit / pvl_wake_advect_cols / pvl_wake_shed
 * over every case (row_case, node_case, circ_case: the case of each row / node / circulation). */
int pvl_batch_fold_implicit(const void* cases, const uint32_t* row_case, uint32_t n_rows,
                            const double* implicit, const uint32_t* adjacent, double* A, void* stream);
int pvl_batch_wake_advect(const void* cases, const uint32_t* node_case, uint32_t n_nodes, uint32_t R,
                          const uint32_t* rows, const double* old_pos, const double* node_vel,
                          const uint32_t* col_slot, const double* body, const uint32_t* bordering_nodes,
                          double* new_pos, void* stream);
int pvl_batch_wake_shed(const void* cases, const uint32_t* circ_case, uint32_t n_circ, uint32_t R,
                        const double* old_circ, const uint32_t* adjacent, const double* gamma,
                        double* new_circ, void* stream);

/* *value += 1 on the device (the step counter of a captured step). */
int pvl_batch_increment(uint32_t* value, void* stream);

/* Jacobi right-preconditioned GMRES of every case with FP64 residuals, entirely on the device
 * (no host synchronisation: capturable in a CUDA graph).  x holds the start and receives the
 * solution; max_iter (<= 16) iterations are launched, converged cases skip their work.
 * fail_flags[c] = 1 where ||b - A x||_c > 10 tol ||b||_c; fail_count accumulates their number. */
size_t pvl_batch_gmres_workspace(uint32_t n_rows, uint32_t n_cases, uint32_t max_iter);
int pvl_batch_gmres(const void* cases, const uint32_t* row_case, uint32_t n_rows, uint32_t n_cases,
                    const double* A, const double* b, double* x, uint32_t max_iter, double tol,
                    uint8_t* fail_flags, uint32_t* fail_count, void* ws, size_t ws_bytes, void* stream);

/* ------------------------------------------------------------------ forces */

/* Kutta-Joukowski line forces F_k = (r_end - r_begin) x (0.5 c_k (v_p1 + v_p2)),
 * c_k = circ[dual.p1] - circ[dual.p2] (INVALID sides skipped); circ is the ring
 * circulation divided by 2 pi.  Replaces Mesh.line_forces (src/meshobject.c:1288-1396). */
int pvl_line_forces(uint32_t n_lines, const uint32_t* primal_lines, const uint32_t* dual_lines,
                    const double* circ, const double* positions, const double* velocity,
                    double* out, void* stream);

/* ------------------------------------------------------------------ measurement */

/* Number of kernels this library has enqueued since it was loaded (all threads).  No
 * reference counterpart: it lets a benchmark state how many of the library's kernels ran. */
unsigned long long pvl_launch_count(void);

#ifdef __cplusplus
}
#endif

#endif /* PVL_B200_H */
