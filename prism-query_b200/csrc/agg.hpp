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
};

// Aggregates `batches` (all with one schema). When `pred`/`exprs` are given
// the aggregate config indexes the projected schema [cols..., expr_i...]
// and the filter/projection is evaluated inside the aggregation kernel.
Batch aggregate(Ctx& ctx, const std::vector<const Batch*>& batches, const prism_agg_config& cfg,
                const prism_predicate* pred, const int32_t* cols, int n_cols, const prism_expr* exprs,
                int n_exprs, int arith_mode, bool fused, const AggTuning& tune);

}  // namespace prism
