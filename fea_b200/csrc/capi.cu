// Library-level entry points: version and launch instrumentation.
#include <atomic>

#include "common.cuh"

namespace fea {
static std::atomic<long long> g_launches{0};
void count_launch(int n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
}  // namespace fea

extern "C" int32_t fea_version(void) { return 1; }
extern "C" int64_t fea_launch_count(void) { return (int64_t)fea::g_launches.load(); }
