// Thread-local error reporting for the C ABI (pvl_last_error) and the ABI version.
#include <cstdarg>
#include <cstdio>
#include <map>
#include <mutex>
#include <utility>

#include <cuda.h>
#include <cuda_runtime.h>

#include "pvl_status.h"

namespace {
thread_local char g_last_error[1024] = "";
}

int pvl_fail(int code, const char* fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
    return code;
}

extern "C" const char* pvl_last_error(void) { return g_last_error; }

extern "C" int pvl_version(void) { return 100; }

// The driver's cuCtxGetCurrent, reached through the runtime (the library links no libcuda).
int pvl_current_context(void** ctx)
{
    using CtxGetCurrent = CUresult (*)(CUcontext*);
    static CtxGetCurrent fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            p = nullptr;
        return reinterpret_cast<CtxGetCurrent>(p);
    }();
    if (!fn)
        return pvl_fail(PVL_ERR_CUDA, "cuCtxGetCurrent is not available");
    CUcontext c = nullptr;
    if (fn(&c) != CUDA_SUCCESS)
        return pvl_fail(PVL_ERR_CUDA, "cuCtxGetCurrent failed");
    *ctx = c;
    return PVL_OK;
}

// cudaFuncSetAttribute(MaxDynamicSharedMemorySize) is a per-device setting of a kernel: keep
// the largest value set for each (kernel, device) and call the runtime only when a launch on
// the current device needs more.  Thread-safe.
int pvl_smem_optin(const void* fn, size_t bytes)
{
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, size_t> done;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess)
        return pvl_fail(PVL_ERR_CUDA, "cudaGetDevice failed");
    std::lock_guard<std::mutex> lock(mu);
    size_t& have = done[std::make_pair(fn, dev)];
    if (have >= bytes)
        return PVL_OK;
    const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess)
        return pvl_fail(PVL_ERR_CUDA, "cudaFuncSetAttribute(%zu bytes): %s", bytes, cudaGetErrorString(e));
    have = bytes;
    return PVL_OK;
}
