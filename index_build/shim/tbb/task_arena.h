// Shim of tbb::this_task_arena (see detail_pool.h).
#pragma once
#include <tbb/detail_pool.h>

namespace tbb {
namespace this_task_arena {
inline int max_concurrency() { return shim::pool::get().concurrency(); }
}  // namespace this_task_arena
}  // namespace tbb
