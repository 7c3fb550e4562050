// sort.hpp — sort / top-N of a batch (native/prism-executor/src/sort.rs).
#pragma once

#include "prism_gpu.h"
#include "runtime.hpp"

namespace prism {

// The batch's rows ordered by `keys` (most significant first), the first
// `limit` of them (limit < 0: all). An empty batch or key list returns the
// batch unchanged.
Batch sort_batch(Ctx& ctx, const Batch& b, const prism_sort_key* keys, int n_keys, int64_t limit);

}  // namespace prism
