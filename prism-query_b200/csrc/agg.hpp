// agg.hpp — hash aggregation (native/prism-executor/src/hash_aggregate.rs)
// and the fused filter -> project -> aggregate path.
#pragma once

#include "plan.hpp"
#include "runtime.hpp"

namespace prism {

struct AggTuning {
  int block = 512;
  int smem_groups = 1024;   // dense accumulator rows per CTA (hash mode)
  int blocks_per_sm = 1;
  // fused join -> aggregate kernel shape: one 1,024-thread block per SM
  // (the autotuner's pick on the 15M x 150M Utf8 join -> GROUP BY with the
  // packed key records: 0.708 ms per 10M-row batch, against 0.763 for 3
  // blocks of 512) and a block table of at most 512 slots, which leaves
  // most of the SM's 228 KB to L1 for the skewed build-side reads
  int join_block = 1024;
  int join_min_blocks = 1;
  int join_rows = 2;
  int join_table_log2 = 9;
  int hash_block = 1024;  // threads per block of the hashed-groups kernel (1024: 0.068 ms vs 0.080 at 512 on 1M rows x 1,024 groups)
  // fields the environment set (the tuning table leaves them alone)
  enum : uint32_t { FIX_JOIN_SHAPE = 1, FIX_HASH_BLOCK = 2 };
  uint32_t fixed = 0;
};

struct JoinTable;

// A fused join -> aggregate (prism-substrait/src/executor.rs:333-842): the
// aggregated batches are probe batches joined with `table`'s build side on
// `probe_keys` inside the aggregation kernel; the projection indexes the
// joined schema (probe columns, then build columns).
struct JoinAggSpec {
  const JoinTable* table = nullptr;
  std::vector<int> probe_keys;
  // build column whose values the lookup hands to the kernel per probe row
  // (fixed width 4 or 8, no nulls, referenced by the projection), or -1
  int inline_col = -1;
};

// Aggregates `batches` (all with one schema). When `pred`/`exprs` are given
// the aggregate config indexes the projected schema [cols..., expr_i...]
// and the filter/projection is evaluated inside the aggregation kernel.
// With `join`, the fused join -> aggregate kernel runs instead (fused must
// be true); shapes it does not cover fail with PRISM_ERR_INVALID_ARGUMENT
// and a message naming the fused path, so the caller can materialize.
Batch aggregate(Ctx& ctx, const std::vector<const Batch*>& batches, const prism_agg_config& cfg,
                const prism_predicate* pred, const int32_t* cols, int n_cols, const prism_expr* exprs,
                int n_exprs, int arith_mode, bool fused, const AggTuning& tune, const JoinAggSpec* join = nullptr);

}  // namespace prism
