// Status codes and the thread-local error message shared by every C-ABI entry point.
#pragma once

#include "../../include/pvl_b200.h"

// Record a formatted message for pvl_last_error() and return `code`.
int pvl_fail(int code, const char* fmt, ...);
