// The mixed path's solve as one CUDA graph that the device drives to convergence (sm_100a).
//
// Right-preconditioned flexible GMRES on A x = b: A the FP64 system, M the FP32 explicit
// approximate inverse (pvl_lu32_inverse).  Per Krylov column j:
//   z_j = M v_j         FP32 matrix and FP32 copy of v_j, FP64 sums          (gemv, HBM-bound)
//   w   = A z_j         FP64                                                  (gemv, HBM-bound)
//   two classical Gram-Schmidt passes of w against v_0..v_j, ||w||, v_{j+1},
//   the Givens rotation of Hessenberg column j and the residual estimate      (one CTA)
// The columns run inside a conditional WHILE node whose condition the single-CTA kernel
// sets: the loop ends when the rotated residual meets tol ||b||, the Krylov space is
// exhausted, or max_iter columns are done (the column counter rises by one every pass, so
// the loop always ends).  After it: the triangular solve for y, x += Z y, the FP64 residual
// r = r0 - sum_j y_j (A z_j) from the stored products A z_j (the vector b - A x, which a
// further pass over A would recompute; the two differ by the rounding of the x update), and a
// status record.  A conditional IF node then runs the FP64 factorisation and a blocked
// triangular solve when that residual missed tol, so the returned x meets it without the host
// looking at the iteration in between.
//
// The host only launches the graph; the status record (iterations, residuals, whether the
// FP64 fallback ran) is read back whenever the host wants it.  This removes the host round
// trips of a host-driven Arnoldi loop (two synchronisations per solve).
// No reference counterpart: the reference factorises every step (python/pyvl/solver.py:223).
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <new>

#include "gemv.cuh"
#include "pvl_b200.h"
#include "pvl_common.cuh"

namespace {

constexpr uint32_t kMaxIter = 32;
constexpr int kCta = 1024;

// Device-resident state of one solve (fixed address, captured into the graph).
struct Ctl {
    double bnorm, beta, target;
    uint32_t j;      // Krylov columns completed
    uint32_t done;   // the loop has ended
    double cs[kMaxIter], sn[kMaxIter], g[kMaxIter + 1];
    double H[kMaxIter][kMaxIter + 2];  // column j of the (rotated) Hessenberg matrix, rows 0..j+1
    double hpass[kMaxIter + 1];        // this Gram-Schmidt pass's projections
};

__device__ __forceinline__ double warp_sum(double v)
{
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum over the CTA in a fixed order (deterministic); every thread gets the result.
__device__ double block_sum(double v, double* red)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    if (lane == 0)
        red[warp] = v;
    __syncthreads();
    if (warp == 0) {
        v = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.0;
        v = warp_sum(v);
        if (lane == 0)
            red[32] = v;
    }
    __syncthreads();
    const double r = red[32];
    __syncthreads();
    return r;
}

// ||b||, beta = ||r|| (r = b - A x already in w), v_0 = r / beta and its FP32 copy.
__global__ void __launch_bounds__(kCta) gmres_start_kernel(uint32_t n, const double* __restrict__ b,
                                                           const double* __restrict__ r, double* __restrict__ r0,
                                                           double* __restrict__ V, float* __restrict__ v32,
                                                           Ctl* __restrict__ ctl, double tol, uint32_t max_iter,
                                                           cudaGraphConditionalHandle loop)
{
    __shared__ double red[33];
    double sb = 0.0, sr = 0.0;
    for (uint32_t e = threadIdx.x; e < n; e += kCta) {
        sb = fma(b[e], b[e], sb);
        sr = fma(r[e], r[e], sr);
    }
    const double bn = sqrt(block_sum(sb, red));
    const double be = sqrt(block_sum(sr, red));
    const double inv = be > 0.0 ? 1.0 / be : 0.0;
    for (uint32_t e = threadIdx.x; e < n; e += kCta) {
        const double v = r[e] * inv;
        r0[e] = r[e];
        V[e] = v;
        v32[e] = (float)v;
    }
    if (threadIdx.x == 0) {
        ctl->bnorm = bn;
        ctl->beta = be;
        ctl->target = tol * bn;
        ctl->j = 0;
        ctl->g[0] = be;
        const uint32_t done = !(be > tol * bn) || max_iter == 0;  // a NaN residual ends it too
        ctl->done = done;
        cudaGraphSetConditional(loop, done ? 0u : 1u);
    }
}

// Column j = ctl->j after W_j = A z_j: w = W_j (W_j stays for the final residual), Gram-Schmidt
// (two classical passes), normalisation, Givens rotation, convergence test; sets the loop
// condition.
__global__ void __launch_bounds__(kCta) gmres_arnoldi_kernel(uint32_t n, double* __restrict__ V,
                                                             const double* __restrict__ W, double* __restrict__ w,
                                                             float* __restrict__ v32, Ctl* __restrict__ ctl,
                                                             uint32_t max_iter, cudaGraphConditionalHandle loop)
{
    __shared__ double red[32][kMaxIter + 1];
    __shared__ double tot[33];
    const uint32_t j = ctl->j;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double* h = ctl->H[j];
    for (uint32_t e = threadIdx.x; e < n; e += kCta)  // each thread works on its own entries only
        w[e] = W[(size_t)j * n + e];
    for (int pass = 0; pass < 2; ++pass) {
        for (uint32_t i = 0; i <= j; ++i) {
            const double* vi = V + (size_t)i * n;
            double s = 0.0;
            for (uint32_t e = threadIdx.x; e < n; e += kCta)
                s = fma(vi[e], w[e], s);
            s = warp_sum(s);
            if (lane == 0)
                red[warp][i] = s;
        }
        __syncthreads();
        if (threadIdx.x <= j) {
            double c = 0.0;
            for (int q = 0; q < kCta / 32; ++q)
                c += red[q][threadIdx.x];
            ctl->hpass[threadIdx.x] = c;
            h[threadIdx.x] = pass == 0 ? c : h[threadIdx.x] + c;
        }
        __syncthreads();
        for (uint32_t e = threadIdx.x; e < n; e += kCta) {
            double s = w[e];
            for (uint32_t i = 0; i <= j; ++i)
                s = fma(-ctl->hpass[i], V[(size_t)i * n + e], s);
            w[e] = s;
        }
        __syncthreads();
    }
    double ss = 0.0;
    for (uint32_t e = threadIdx.x; e < n; e += kCta)
        ss = fma(w[e], w[e], ss);
    const double hn = sqrt(block_sum(ss, tot));
    const double inv = hn > 0.0 ? 1.0 / hn : 0.0;
    double* vn = V + (size_t)(j + 1) * n;
    for (uint32_t e = threadIdx.x; e < n; e += kCta) {
        const double v = w[e] * inv;
        vn[e] = v;
        v32[e] = (float)v;
    }
    if (threadIdx.x == 0) {
        h[j + 1] = hn;
        for (uint32_t i = 0; i < j; ++i) {  // the previous rotations
            const double t = ctl->cs[i] * h[i] + ctl->sn[i] * h[i + 1];
            h[i + 1] = -ctl->sn[i] * h[i] + ctl->cs[i] * h[i + 1];
            h[i] = t;
        }
        const double den = hypot(h[j], h[j + 1]);
        const double c = den == 0.0 ? 1.0 : h[j] / den, s = den == 0.0 ? 0.0 : h[j + 1] / den;
        ctl->cs[j] = c;
        ctl->sn[j] = s;
        h[j] = c * h[j] + s * h[j + 1];
        h[j + 1] = 0.0;
        ctl->g[j + 1] = -s * ctl->g[j];
        ctl->g[j] = c * ctl->g[j];
        const uint32_t jn = j + 1;
        ctl->j = jn;
        const uint32_t done = !(fabs(ctl->g[jn]) > ctl->target) || hn == 0.0 || jn >= max_iter;
        ctl->done = done;
        cudaGraphSetConditional(loop, done ? 0u : 1u);
    }
}

// The same column step with this thread's PER entries of w (e = threadIdx.x + i * kCta) held in
// registers, the projections and the Givens inputs in shared memory: the only global-memory
// round trips left are the loads of W_j and of the basis rows.  For n <= PER * kCta.
template <int PER>
__global__ void __launch_bounds__(kCta) gmres_arnoldi_reg_kernel(uint32_t n, double* __restrict__ V,
                                                                 const double* __restrict__ W,
                                                                 float* __restrict__ v32, Ctl* __restrict__ ctl,
                                                                 uint32_t max_iter, cudaGraphConditionalHandle loop)
{
    __shared__ double red[32][kMaxIter + 1];
    __shared__ double tot[33];
    __shared__ double hs[kMaxIter + 2], hp[kMaxIter + 1], cs[kMaxIter], sn[kMaxIter];
    const uint32_t j = ctl->j;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x < j) {  // the previous rotations, for the Givens step at the end
        cs[threadIdx.x] = ctl->cs[threadIdx.x];
        sn[threadIdx.x] = ctl->sn[threadIdx.x];
    }
    double w[PER];
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const uint32_t e = threadIdx.x + q * kCta;
        w[q] = e < n ? W[(size_t)j * n + e] : 0.0;
    }
    for (int pass = 0; pass < 2; ++pass) {
        for (uint32_t i = 0; i <= j; ++i) {
            const double* vi = V + (size_t)i * n;
            double t = 0.0;
#pragma unroll
            for (int q = 0; q < PER; ++q) {
                const uint32_t e = threadIdx.x + q * kCta;
                if (e < n)
                    t = fma(vi[e], w[q], t);
            }
            t = warp_sum(t);
            if (lane == 0)
                red[warp][i] = t;
        }
        __syncthreads();
        if (threadIdx.x <= j) {
            double c = 0.0;
            for (int q = 0; q < kCta / 32; ++q)
                c += red[q][threadIdx.x];
            hp[threadIdx.x] = c;
            hs[threadIdx.x] = pass == 0 ? c : hs[threadIdx.x] + c;
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < PER; ++q) {
            const uint32_t e = threadIdx.x + q * kCta;
            if (e < n) {
                double t = w[q];
                for (uint32_t i = 0; i <= j; ++i)
                    t = fma(-hp[i], V[(size_t)i * n + e], t);
                w[q] = t;
            }
        }
        __syncthreads();  // hp is rewritten by the next pass
    }
    double ss = 0.0;
#pragma unroll
    for (int q = 0; q < PER; ++q)
        ss = fma(w[q], w[q], ss);
    const double hn = sqrt(block_sum(ss, tot));
    const double inv = hn > 0.0 ? 1.0 / hn : 0.0;
    double* vn = V + (size_t)(j + 1) * n;
#pragma unroll
    for (int q = 0; q < PER; ++q) {
        const uint32_t e = threadIdx.x + q * kCta;
        if (e < n) {
            const double v = w[q] * inv;
            vn[e] = v;
            v32[e] = (float)v;
        }
    }
    if (threadIdx.x == 0) {
        double gj = ctl->g[j];
        hs[j + 1] = hn;
        for (uint32_t i = 0; i < j; ++i) {  // the previous rotations
            const double t = cs[i] * hs[i] + sn[i] * hs[i + 1];
            hs[i + 1] = -sn[i] * hs[i] + cs[i] * hs[i + 1];
            hs[i] = t;
        }
        const double den = hypot(hs[j], hs[j + 1]);
        const double c = den == 0.0 ? 1.0 : hs[j] / den, sg = den == 0.0 ? 0.0 : hs[j + 1] / den;
        hs[j] = c * hs[j] + sg * hs[j + 1];
        hs[j + 1] = 0.0;
        double* h = ctl->H[j];
        for (uint32_t i = 0; i <= j + 1; ++i)
            h[i] = hs[i];
        ctl->cs[j] = c;
        ctl->sn[j] = sg;
        const double gn = -sg * gj;
        ctl->g[j + 1] = gn;
        ctl->g[j] = c * gj;
        const uint32_t jn = j + 1;
        ctl->j = jn;
        const uint32_t done = !(fabs(gn) > ctl->target) || hn == 0.0 || jn >= max_iter;
        ctl->done = done;
        cudaGraphSetConditional(loop, done ? 0u : 1u);
    }
}

// y from the rotated Hessenberg system, x += Z y, r = r0 - W y (held in r), rel = ||r|| / ||b||,
// the status record and the fallback condition.
__global__ void __launch_bounds__(kCta) gmres_update_kernel(uint32_t n, const double* __restrict__ Z,
                                                            const double* __restrict__ W,
                                                            const double* __restrict__ r0, double* __restrict__ x,
                                                            double* __restrict__ r, const Ctl* __restrict__ ctl,
                                                            double tol, pvl_gmres_status* __restrict__ status,
                                                            cudaGraphConditionalHandle fallback)
{
    __shared__ double y[kMaxIter];
    __shared__ double red[33];
    __shared__ double R[kMaxIter][kMaxIter + 1], gs[kMaxIter];  // R[l][i] = rotated H, column l
    const uint32_t k = ctl->j;
    for (uint32_t e = threadIdx.x; e < k * k; e += kCta) {  // the triangle, loaded in parallel
        const uint32_t l = e / k, i = e % k;
        if (i <= l)
            R[l][i] = ctl->H[l][i];
    }
    if (threadIdx.x < k)
        gs[threadIdx.x] = ctl->g[threadIdx.x];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (uint32_t i = k; i-- > 0;) {  // back substitution (rows of R)
            double s = gs[i];
            for (uint32_t l = i + 1; l < k; ++l)
                s -= R[l][i] * y[l];
            const double d = R[i][i];
            y[i] = d != 0.0 ? s / d : 0.0;
        }
    }
    __syncthreads();
    double q = 0.0;
    for (uint32_t e = threadIdx.x; e < n; e += kCta) {
        double s = x[e], t = r0[e];
        for (uint32_t i = 0; i < k; ++i) {
            s = fma(y[i], Z[(size_t)i * n + e], s);
            t = fma(-y[i], W[(size_t)i * n + e], t);
        }
        x[e] = s;
        r[e] = t;
        q = fma(t, t, q);
    }
    const double rn = sqrt(block_sum(q, red));
    if (threadIdx.x == 0) {
        const double bn = fmax(ctl->bnorm, 1e-300);
        const double rel = rn / bn;
        const uint32_t ok = rel <= tol;  // false for NaN
        status->iterations = k;
        status->converged = ok;
        status->initial_rel_residual = ctl->beta / bn;
        status->final_rel_residual = rel;
        cudaGraphSetConditional(fallback, ok ? 0u : 1u);
    }
}

struct SolverGraph {
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t graph = nullptr;
    unsigned long long fixed_kernels = 0, column_kernels = 0, fallback_kernels = 0;
};

// Add a conditional node to the graph being captured on `s` after its current dependencies,
// make it the new dependency and return its body graph.
int add_conditional(cudaStream_t s, cudaGraphConditionalHandle h, cudaGraphConditionalNodeType type,
                    cudaGraph_t* body)
{
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    PVL_CUDA_CHECK(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &nd));
    if (cs != cudaStreamCaptureStatusActive)
        return pvl_fail(PVL_ERR_CUDA, "gmres graph: stream is not capturing");
    // zero-filled storage: the parameter union has no usable default constructor
    alignas(cudaGraphNodeParams) unsigned char raw[sizeof(cudaGraphNodeParams)];
    std::memset(raw, 0, sizeof(raw));
    cudaGraphNodeParams* p = reinterpret_cast<cudaGraphNodeParams*>(raw);
    p->type = cudaGraphNodeTypeConditional;
    p->conditional.handle = h;
    p->conditional.type = type;
    p->conditional.size = 1;
    cudaGraphNode_t node;
    PVL_CUDA_CHECK(cudaGraphAddNode(&node, g, deps, nd, p));
    PVL_CUDA_CHECK(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    *body = p->conditional.phGraph_out[0];
    return PVL_OK;
}

int capture_graph(SolverGraph* sg, cudaStream_t s, cudaStream_t s2, uint32_t n, double* A, uint32_t lda,
                  const float* Minv, uint32_t ldm, double* b, double* x, double* V, double* Z, double* W, double* r0,
                  double* w, float* v32, Ctl* ctl, uint32_t max_iter, double tol, int32_t* ipiv, int32_t* info, void* ws, size_t ws_bytes,
                  double* gamma, uint32_t n_gamma, uint32_t n_groups, const uint32_t* group_offsets,
                  pvl_gmres_status* status)
{
    cudaStreamCaptureStatus cs;
    cudaGraph_t g = nullptr;
    PVL_CUDA_CHECK(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, nullptr, nullptr));
    cudaGraphConditionalHandle loop, fallback;
    PVL_CUDA_CHECK(cudaGraphConditionalHandleCreate(&loop, g, 0, cudaGraphCondAssignDefault));
    PVL_CUDA_CHECK(cudaGraphConditionalHandleCreate(&fallback, g, 0, cudaGraphCondAssignDefault));
    const unsigned long long c0 = pvl_launch_count();
    // r = b - A x, v_0
    pvl::launch_gemv<double, double>(n, n, -1.0, A, lda, x, 0, 1.0, b, w, 0, nullptr, s);
    PVL_LAUNCH_CHECK();
    gmres_start_kernel<<<1, kCta, 0, s>>>(n, b, w, r0, V, v32, ctl, tol, max_iter, loop);
    PVL_LAUNCH_CHECK();
    // the Krylov columns
    cudaGraph_t body;
    if (int r = add_conditional(s, loop, cudaGraphCondTypeWhile, &body))
        return r;
    const unsigned long long c1 = pvl_launch_count();
    PVL_CUDA_CHECK(cudaStreamBeginCaptureToGraph(s2, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    pvl::launch_gemv<float, float>(n, n, 1.0, Minv, ldm, v32, 0, 0.0, nullptr, Z, n, &ctl->j, s2);
    pvl_count_launch();
    pvl::launch_gemv<double, double>(n, n, 1.0, A, lda, Z, n, 0.0, nullptr, W, n, &ctl->j, s2);
    pvl_count_launch();
    if (n <= 1u * kCta)
        gmres_arnoldi_reg_kernel<1><<<1, kCta, 0, s2>>>(n, V, W, v32, ctl, max_iter, loop);
    else if (n <= 2u * kCta)
        gmres_arnoldi_reg_kernel<2><<<1, kCta, 0, s2>>>(n, V, W, v32, ctl, max_iter, loop);
    else if (n <= 4u * kCta)
        gmres_arnoldi_reg_kernel<4><<<1, kCta, 0, s2>>>(n, V, W, v32, ctl, max_iter, loop);
    else if (n <= 8u * kCta)
        gmres_arnoldi_reg_kernel<8><<<1, kCta, 0, s2>>>(n, V, W, v32, ctl, max_iter, loop);
    else if (n <= 16u * kCta)
        gmres_arnoldi_reg_kernel<16><<<1, kCta, 0, s2>>>(n, V, W, v32, ctl, max_iter, loop);
    else
        gmres_arnoldi_kernel<<<1, kCta, 0, s2>>>(n, V, W, w, v32, ctl, max_iter, loop);
    pvl_count_launch();
    const cudaError_t eb = cudaGetLastError();
    cudaGraph_t body_out = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(s2, &body_out);
    if (eb != cudaSuccess || ee != cudaSuccess)
        return pvl_fail(PVL_ERR_CUDA, "gmres graph: column body: %s", cudaGetErrorString(eb != cudaSuccess ? eb : ee));
    sg->column_kernels = pvl_launch_count() - c1;
    const unsigned long long c2 = pvl_launch_count();
    // x += Z y, the residual r0 - W y, the status
    gmres_update_kernel<<<1, kCta, 0, s>>>(n, Z, W, r0, x, w, ctl, tol, status, fallback);
    PVL_LAUNCH_CHECK();
    // the FP64 fallback: factorise A in place, solve for b in place, x = b
    if (int r = add_conditional(s, fallback, cudaGraphCondTypeIf, &body))
        return r;
    const unsigned long long c3 = pvl_launch_count();
    PVL_CUDA_CHECK(cudaStreamBeginCaptureToGraph(s2, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal));
    int rf = pvl_lu_factor(n, A, lda, ipiv, info, ws, ws_bytes, s2);
    if (!rf)
        rf = pvl_lu_solve_blocked(n, A, lda, ipiv, b, ws, ws_bytes, s2);
    const cudaError_t ec = rf ? cudaSuccess : cudaMemcpyAsync(x, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, s2);
    body_out = nullptr;
    const cudaError_t ef = cudaStreamEndCapture(s2, &body_out);
    if (rf)
        return rf;
    if (ec != cudaSuccess || ef != cudaSuccess)
        return pvl_fail(PVL_ERR_CUDA, "gmres graph: fallback body: %s", cudaGetErrorString(ec != cudaSuccess ? ec : ef));
    sg->fallback_kernels = pvl_launch_count() - c3;
    const unsigned long long c4 = pvl_launch_count();
    // the circulation
    if (n_gamma) {
        PVL_CUDA_CHECK(cudaMemcpyAsync(gamma, x, sizeof(double) * n_gamma, cudaMemcpyDeviceToDevice, s));
        if (n_groups)
            if (int r = pvl_group_mean_remove(n_groups, group_offsets, gamma, s))
                return r;
    }
    sg->fixed_kernels = (c1 - c0) + (c3 - c2) + (pvl_launch_count() - c4);
    return PVL_OK;
}

}  // namespace

extern "C" size_t pvl_gmres_ctl_bytes(void) { return sizeof(Ctl); }

extern "C" uint32_t pvl_gmres_max_iter(void) { return kMaxIter; }

extern "C" int pvl_gmres_graph_create(uint32_t n, double* A, uint32_t lda, const float* Minv, uint32_t ldm, double* b,
                                      double* x, double* V, double* Z, double* W, double* r0, double* w,
                                      float* v32, void* ctl, uint32_t max_iter, double tol, int32_t* ipiv, int32_t* info, void* ws,
                                      size_t ws_bytes, double* gamma, uint32_t n_gamma, uint32_t n_groups,
                                      const uint32_t* group_offsets, pvl_gmres_status* status, uint64_t* graph_out)
{
    if (!graph_out)
        return pvl_fail(PVL_ERR_ARG, "pvl_gmres_graph_create: graph_out is NULL");
    *graph_out = 0;
    if (n == 0 || !A || !Minv || !b || !x || !V || !Z || !W || !r0 || !w || !v32 || !ctl || !ipiv || !info || !ws || !status)
        return pvl_fail(PVL_ERR_ARG, "pvl_gmres_graph_create: empty system or null pointer argument");
    if (max_iter == 0 || max_iter > kMaxIter)
        return pvl_fail(PVL_ERR_ARG, "pvl_gmres_graph_create: max_iter %u outside 1..%u", max_iter, kMaxIter);
    if (lda < n || ldm < n || n_gamma > n || (n_gamma && !gamma) || (n_groups && !group_offsets))
        return pvl_fail(PVL_ERR_ARG, "pvl_gmres_graph_create: inconsistent sizes");
    if ((((uintptr_t)v32) & 15u) || (((uintptr_t)ctl) & 7u))
        return pvl_fail(PVL_ERR_ARG, "pvl_gmres_graph_create: v32 must be 16-byte and ctl 8-byte aligned");
    if (ws_bytes < pvl_lu_workspace(n))
        return pvl_fail(PVL_ERR_ALLOC, "pvl_gmres_graph_create: workspace %zu < %zu", ws_bytes, pvl_lu_workspace(n));
    SolverGraph* sg = new (std::nothrow) SolverGraph();
    if (!sg)
        return pvl_fail(PVL_ERR_ALLOC, "pvl_gmres_graph_create: out of host memory");
    cudaStream_t s = nullptr, s2 = nullptr;
    int rc = PVL_OK;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
        cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking) != cudaSuccess) {
        rc = pvl_fail(PVL_ERR_CUDA, "pvl_gmres_graph_create: stream creation failed");
    } else if (cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        rc = pvl_fail(PVL_ERR_CUDA, "pvl_gmres_graph_create: capture failed to start");
    } else {
        rc = capture_graph(sg, s, s2, n, A, lda, Minv, ldm, b, x, V, Z, W, r0, w, v32, static_cast<Ctl*>(ctl), max_iter, tol,
                           ipiv, info, ws, ws_bytes, gamma, n_gamma, n_groups, group_offsets, status);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(s, &g);
        sg->graph = g;
        if (!rc && e != cudaSuccess)
            rc = pvl_fail(PVL_ERR_CUDA, "pvl_gmres_graph_create: capture: %s", cudaGetErrorString(e));
        if (!rc) {
            const cudaError_t ei = cudaGraphInstantiate(&sg->exec, g, 0);
            if (ei != cudaSuccess)
                rc = pvl_fail(PVL_ERR_CUDA, "pvl_gmres_graph_create: instantiate: %s", cudaGetErrorString(ei));
        }
    }
    cudaGetLastError();
    if (s2)
        cudaStreamDestroy(s2);
    if (s)
        cudaStreamDestroy(s);
    if (rc) {
        if (sg->exec)
            cudaGraphExecDestroy(sg->exec);
        if (sg->graph)
            cudaGraphDestroy(sg->graph);
        delete sg;
        return rc;
    }
    *graph_out = reinterpret_cast<uint64_t>(sg);
    return PVL_OK;
}

extern "C" int pvl_gmres_graph_launch(uint64_t graph, void* stream)
{
    SolverGraph* sg = reinterpret_cast<SolverGraph*>(graph);
    if (!sg || !sg->exec)
        return pvl_fail(PVL_ERR_ARG, "pvl_gmres_graph_launch: no graph");
    PVL_CUDA_CHECK(cudaGraphLaunch(sg->exec, (cudaStream_t)stream));
    for (unsigned long long i = 0; i < sg->fixed_kernels; ++i)
        pvl_count_launch();
    return PVL_OK;
}

extern "C" int pvl_gmres_graph_account(uint64_t graph, uint32_t iterations, uint32_t fell_back)
{
    SolverGraph* sg = reinterpret_cast<SolverGraph*>(graph);
    if (!sg)
        return pvl_fail(PVL_ERR_ARG, "pvl_gmres_graph_account: no graph");
    const unsigned long long k = (unsigned long long)iterations * sg->column_kernels +
                                 (fell_back ? sg->fallback_kernels : 0ull);
    for (unsigned long long i = 0; i < k; ++i)
        pvl_count_launch();
    return PVL_OK;
}

extern "C" int pvl_gmres_graph_destroy(uint64_t graph)
{
    SolverGraph* sg = reinterpret_cast<SolverGraph*>(graph);
    if (!sg)
        return PVL_OK;
    if (sg->exec)
        cudaGraphExecDestroy(sg->exec);
    if (sg->graph)
        cudaGraphDestroy(sg->graph);
    delete sg;
    return PVL_OK;
}
