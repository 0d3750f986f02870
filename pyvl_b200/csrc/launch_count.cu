// pvl_launch_count(): every kernel enqueued through the C ABI is counted at its launch site
// (PVL_LAUNCH_CHECK / pvl_count_launch), so that a caller can state how many of this
// library's kernels ran in a timed region.
#include <atomic>

#include "pvl_common.cuh"

namespace {
std::atomic<unsigned long long> g_launches{0};
}

void pvl_count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

extern "C" unsigned long long pvl_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }
