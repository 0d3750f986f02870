// pvl_line_velocity_noalloc: the segment-sum velocity of pvl_line_velocity for callers that
// cannot allocate device memory.
//
// Some hosts of this library own every byte of device memory through their own pool and
// do not allow a library to call cudaMalloc behind their back; others run the velocity
// evaluation inside loops where an allocation, and the device-wide synchronisation a
// cudaFree implies, is not acceptable.  Such callers can still pass their inputs and
// outputs, but not a workspace.  This entry point gives them the same computation with
// its scratch (the segment table and the per-range partial sums) in a fixed array that
// lives in this library's device image, so nothing is allocated at call time.
//
// Limits and rules:
//  * the array holds PVL_NOALLOC_SCRATCH_BYTES (32 MiB); every GPU that loads the library
//    keeps that much device memory until the process exits;
//  * a call whose workspace need (pvl_line_velocity_workspace) exceeds the array is rejected
//    with PVL_ERR_ARG before anything is enqueued;
//  * all calls share the one array: two calls whose kernels overlap on the GPU (different
//    streams, or concurrent host threads) race on it; calls serialised on one stream are
//    safe.  The array keeps the contents of the last call; nothing in it needs to start at
//    zero, because every byte the computation reads is written earlier in the same call;
//  * the first call on each device looks up the array's device address with
//    cudaGetSymbolAddress (once per device and CUDA context, with that device current).  Make
//    that first call before any stream capture begins.  A device reset or a new primary
//    context reloads the module, possibly at another address: the lookup is redone when the
//    current context differs from the one the address was found in.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "pvl_common.cuh"

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[PVL_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
struct ScratchAddr {
    CUcontext ctx;  // the context the address was looked up in
    void* addr;
};
ScratchAddr g_scratch[kMaxDevices] = {};
std::mutex g_scratch_mutex;

// Device address of g_noalloc_scratch on the current device, looked up once per device and
// context (the caller has made the device current, so the runtime's context is current too).
int scratch_for_current_device(void** out)
{
    int dev = 0;
    PVL_CUDA_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kMaxDevices)
        return pvl_fail(PVL_ERR_ARG, "pvl_line_velocity_noalloc: device index %d out of range", dev);
    void* cur = nullptr;
    if (int rc = pvl_current_context(&cur))
        return rc;
    CUcontext ctx = static_cast<CUcontext>(cur);
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    ScratchAddr& s = g_scratch[dev];
    if (!s.addr || !ctx || s.ctx != ctx) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);  // makes the primary context current
        if (e != cudaSuccess || !p)
            return pvl_fail(PVL_ERR_CUDA, "pvl_line_velocity_noalloc: cudaGetSymbolAddress failed: %s",
                            cudaGetErrorString(e));
        if (!ctx) {
            if (int rc = pvl_current_context(&cur))
                return rc;
            ctx = static_cast<CUcontext>(cur);
            if (!ctx)
                return pvl_fail(PVL_ERR_CUDA, "pvl_line_velocity_noalloc: no current CUDA context");
        }
        s.ctx = ctx;
        s.addr = p;
    }
    *out = s.addr;
    return PVL_OK;
}

}  // namespace

extern "C" int pvl_line_velocity_noalloc(int precision, uint32_t n_points, uint32_t n_lines, const uint32_t* lines,
                                         const double* positions, const double* line_gamma, uint32_t n_pts,
                                         const double* pts, const double* normals, double tol, double alpha,
                                         double beta, double* out, void* stream)
{
    if (n_pts == 0)
        return PVL_OK;
    const size_t need = pvl_line_velocity_workspace(n_lines, n_pts, precision);
    if (need > (size_t)PVL_NOALLOC_SCRATCH_BYTES)
        return pvl_fail(PVL_ERR_ARG,
                        "pvl_line_velocity_noalloc: %u segments x %u points need %zu bytes of scratch, more than the "
                        "%zu-byte static array; use pvl_line_velocity with a caller workspace",
                        n_lines, n_pts, need, (size_t)PVL_NOALLOC_SCRATCH_BYTES);
    void* scratch = nullptr;
    if (int r = scratch_for_current_device(&scratch))
        return r;
    return pvl_line_velocity(precision, n_points, n_lines, lines, positions, line_gamma, n_pts, pts, normals, tol,
                             alpha, beta, out, scratch, (size_t)PVL_NOALLOC_SCRATCH_BYTES, stream);
}
