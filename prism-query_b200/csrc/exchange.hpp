// exchange.hpp — the exchange step of multi-GPU aggregation: a device batch
// packed into one contiguous device buffer (one collective moves it),
// unpacked on the receiving GPU, and the reducer's merge of per-worker
// partial aggregates (prism-bench/src/handler.rs:270-344) on the GPU.
#pragma once

#include <vector>

#include "agg.hpp"
#include "runtime.hpp"

namespace prism {

struct WorkerAggs {
  std::vector<prism_agg_expr> aggs;  // the worker-side aggregate list
  std::vector<int32_t> map;          // per original aggregate: 2 worker indices (the second -1 unless AVG)
};

// expand_worker_aggregates (handler.rs:397-428): AVG becomes SUM then COUNT
// of its column; every other aggregate stays. Worker outputs are named
// "agg_<index>".
WorkerAggs expand_worker_aggregates(const prism_agg_config& original);

// Bytes that pack_batch writes for `b` (a multiple of 16).
uint64_t packed_size(const Batch& b);
// Writes `b` into the device buffer `dst` (capacity >= packed_size(b)),
// stream-ordered on the context's stream.
void pack_batch(Ctx& ctx, const Batch& b, void* dst, uint64_t capacity);
// Reads a packed batch from device memory [src, src + size); the result owns
// a copy of the payload. Synchronises the context's stream (the header is
// read on the host).
Batch unpack_batch(Ctx& ctx, const void* src, uint64_t size);
// The same format on the host: a Batch of HOST pointers (host_batch) packed
// into host memory, and a host packed buffer read back (columns point into
// `payload`, a copy this call makes). No device is involved.
void pack_host(const Batch& b, void* dst, uint64_t capacity);
Batch unpack_host(const void* src, uint64_t size, std::shared_ptr<std::vector<uint8_t>>& payload);

// The reducer merge: hash aggregation of the partials with the final merge
// configuration (handler.rs:430-457), then the original aggregates rebuilt
// from the merged columns (handler.rs:459-530).
Batch merge_partial_aggregates(Ctx& ctx, const std::vector<const Batch*>& partials, const prism_agg_config& original,
                               const AggTuning& tune);

}  // namespace prism
