// sort.hpp — sort / top-N of a batch (native/prism-executor/src/sort.rs).
#pragma once

#include "prism_gpu.h"
#include "runtime.hpp"

namespace prism {

// The batch's rows ordered by `keys` (most significant first), the first
// `limit` of them (limit < 0: all). An empty batch or key list returns the
// batch unchanged.
Batch sort_batch(Ctx& ctx, const Batch& b, const prism_sort_key* keys, int n_keys, int64_t limit);

// One stable radix-partition pass of 64-bit keys by bits [shift, shift +
// bits) of key * mul (bits <= 8): keys and their positions in partition
// order (positions ascending inside a partition). The two kernels are timed
// (when profiling) under the given names.
void radix_partition(Ctx& ctx, const uint64_t* keys, int64_t n, uint64_t mul, int shift, int bits,
                     uint64_t* kout, uint32_t* pos_out, const char* hist_name, const char* scatter_name);

}  // namespace prism
