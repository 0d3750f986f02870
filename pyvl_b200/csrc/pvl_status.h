// Status codes and the thread-local error message shared by every C-ABI entry point.
#pragma once

#include "../../include/pvl_b200.h"

// Record a formatted message for pvl_last_error() and return `code`.
int pvl_fail(int code, const char* fmt, ...);

#include <stddef.h>

// The calling thread's current CUDA context (the runtime's primary context once a runtime call
// has run on the device).  Returns PVL_OK or PVL_ERR_CUDA with the message set.
int pvl_current_context(void** ctx);

// Opt the kernel `fn` in to `bytes` of dynamic shared memory on the current device (once per
// kernel and device; thread-safe).  Returns PVL_OK or a PVL_ERR_* code with the message set.
int pvl_smem_optin(const void* fn, size_t bytes);
#define PVL_SMEM_OPTIN(fn, bytes)                                                    \
    do {                                                                             \
        const int pvl_rc_ = pvl_smem_optin(reinterpret_cast<const void*>(fn), bytes); \
        if (pvl_rc_ != PVL_OK)                                                       \
            return pvl_rc_;                                                          \
    } while (0)
