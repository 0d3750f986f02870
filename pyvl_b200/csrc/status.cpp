// Thread-local error reporting for the C ABI (pvl_last_error) and the ABI version.
#include <cstdarg>
#include <cstdio>

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
