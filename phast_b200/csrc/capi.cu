// Library-level entry points: version and the kernel-launch counter.
#include <atomic>

#include "common.cuh"

namespace phastb {
static std::atomic<long long> g_launches{0};
void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }
}  // namespace phastb

extern "C" {

const char* phastb_version(void) { return "phastb 0.1 sm_100a"; }

long long phastb_launch_count(void) { return phastb::g_launches.load(std::memory_order_relaxed); }

void phastb_launch_count_reset(void) { phastb::g_launches.store(0, std::memory_order_relaxed); }

}  // extern "C"
