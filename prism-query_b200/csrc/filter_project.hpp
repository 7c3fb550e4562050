// filter_project.hpp — predicate evaluation, filtering and projection
// (native/prism-executor/src/filter_project.rs).
#pragma once

#include "plan.hpp"
#include "runtime.hpp"

namespace prism {

// evaluate_predicate: one Boolean column (with nulls) named "mask".
ColP evaluate_predicate(Ctx& ctx, const Batch& b, const prism_predicate& pred);
// Ordered row indices where mask is true and valid.
MemP mask_rows(Ctx& ctx, const Column& mask, int64_t* count);
Batch filter_rows(Ctx& ctx, const Batch& b, const uint32_t* rows, int64_t n);
Batch filter_by_mask(Ctx& ctx, const Batch& b, const Column& mask);
Batch project(const Batch& b, const int32_t* cols, int n_cols);
// project_batch_with_exprs: passthrough columns then expr_i columns.
Batch project_with_exprs(Ctx& ctx, const Batch& b, const int32_t* cols, int n_cols, const prism_expr* exprs,
                         int n_exprs, int arith_mode);

}  // namespace prism
