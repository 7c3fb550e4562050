/*
 * oracle.h — TEST INFRASTRUCTURE ONLY.
 *
 * C API of the CPU oracle: a C++17 restatement of the reference operators
 *   native/prism-executor/src/hash_join.rs       (join build / probe / assemble)
 *   native/prism-executor/src/hash_aggregate.rs  (grouped + global aggregation)
 *   native/prism-executor/src/filter_project.rs  (predicates, filter, projection)
 *   native/prism-substrait/src/executor.rs:333-842 (fused join -> aggregate)
 * used by the test-suite as the parity checker and by bench.py as the timed
 * CPU baseline. The GPU product never links, loads or calls this library.
 *
 * Inputs are borrowed Arrow C Data Interface struct arrays (one RecordBatch
 * each); all batches of one call share `schema`. Outputs are owned by the
 * caller (call their release callbacks). Return value: 0 or a PRISM_ERR_*
 * code; oracle_last_error() holds the message (thread-local).
 *
 * n_threads reproduces the reference's rayon chunking
 * (chunk = max(1, n_batches / n_threads), hash_aggregate.rs:217) so that the
 * f64 accumulation order is the reference's; it is also the worker-thread
 * count when the oracle is timed as the CPU baseline.
 */
#ifndef PRISM_ORACLE_H
#define PRISM_ORACLE_H

#include "../include/prism_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

const char* oracle_last_error(void);

/* hash_join (hash_join.rs:312-365) */
int oracle_hash_join(const struct ArrowArray* probe, const struct ArrowSchema* probe_schema,
                     const struct ArrowArray* build, const struct ArrowSchema* build_schema,
                     const prism_join_config* config, int n_threads, struct ArrowArray* out,
                     struct ArrowSchema* out_schema);

/* probe_matches_chunked (hash_join.rs:286-309): outs[i] = (probe_idx, build_idx) */
int oracle_probe_matches_chunked(const struct ArrowArray* const* probes,
                                 const struct ArrowSchema* probe_schema, int n_probes,
                                 const struct ArrowArray* build,
                                 const struct ArrowSchema* build_schema,
                                 const int32_t* probe_keys, const int32_t* build_keys,
                                 int n_keys, int n_threads, struct ArrowArray* outs,
                                 struct ArrowSchema* out_schemas);

/* hash_join_probe_chunked (hash_join.rs:206-282); *n_out = batches written */
int oracle_hash_join_probe_chunked(const struct ArrowArray* const* probes,
                                   const struct ArrowSchema* probe_schema, int n_probes,
                                   const struct ArrowArray* build,
                                   const struct ArrowSchema* build_schema,
                                   const prism_join_config* config, int n_threads,
                                   struct ArrowArray* outs, struct ArrowSchema* out_schemas,
                                   int* n_out);

/* Match count only (no output materialisation): the timed CPU-baseline probe
 * of hash_join.rs:143-200 over the given probe batches. Returns matches. */
int64_t oracle_join_count_matches(const struct ArrowArray* const* probes,
                                  const struct ArrowSchema* probe_schema, int n_probes,
                                  const struct ArrowArray* build,
                                  const struct ArrowSchema* build_schema,
                                  const int32_t* probe_keys, const int32_t* build_keys,
                                  int n_keys, int n_threads, int materialize_pairs);

/* hash_aggregate_batches (hash_aggregate.rs:182-339, 343-447) */
int oracle_hash_aggregate_batches(const struct ArrowArray* const* batches,
                                  const struct ArrowSchema* schema, int n_batches,
                                  const prism_agg_config* config, int n_threads,
                                  struct ArrowArray* out, struct ArrowSchema* out_schema);

/* evaluate_predicate (filter_project.rs:65-123): 1-column Boolean batch */
int oracle_evaluate_predicate(const struct ArrowArray* batch, const struct ArrowSchema* schema,
                              const prism_predicate* predicate, struct ArrowArray* out,
                              struct ArrowSchema* out_schema);
/* sort_batch / sort_batch_limit (sort.rs:35-78); limit < 0: all rows */
int oracle_sort_batch(const struct ArrowArray* batch, const struct ArrowSchema* schema,
                      const prism_sort_key* keys, int n_keys, int64_t limit, struct ArrowArray* out,
                      struct ArrowSchema* out_schema);
/* filter_batch (filter_project.rs:126-135); mask = 1-column Boolean batch */
int oracle_filter_batch(const struct ArrowArray* batch, const struct ArrowSchema* schema,
                        const struct ArrowArray* mask, const struct ArrowSchema* mask_schema,
                        struct ArrowArray* out, struct ArrowSchema* out_schema);
/* project_batch (filter_project.rs:138-160) */
int oracle_project_batch(const struct ArrowArray* batch, const struct ArrowSchema* schema,
                         const int32_t* cols, int n_cols, struct ArrowArray* out,
                         struct ArrowSchema* out_schema);
/* filter_and_project (filter_project.rs:163-180); predicate may be NULL */
int oracle_filter_and_project(const struct ArrowArray* batch, const struct ArrowSchema* schema,
                              const prism_predicate* predicate, const int32_t* cols,
                              int n_cols, struct ArrowArray* out,
                              struct ArrowSchema* out_schema);
/* project_batch_with_exprs (filter_project.rs:305-333) */
int oracle_project_batch_with_exprs(const struct ArrowArray* batch,
                                    const struct ArrowSchema* schema, const int32_t* cols,
                                    int n_cols, const prism_expr* exprs, int n_exprs,
                                    int arith_mode, struct ArrowArray* out,
                                    struct ArrowSchema* out_schema);

/* Filter -> project -> hash_aggregate_batches over a list of batches, the
 * reference executor's Filter/Project/Aggregate node sequence
 * (native/prism-substrait/src/executor.rs:91-186). */
int oracle_filter_project_aggregate(const struct ArrowArray* const* batches,
                                    const struct ArrowSchema* schema, int n_batches,
                                    const prism_predicate* predicate, const int32_t* cols,
                                    int n_cols, const prism_expr* exprs, int n_exprs,
                                    int arith_mode, const prism_agg_config* agg,
                                    int n_threads, struct ArrowArray* out,
                                    struct ArrowSchema* out_schema);

/* try_execute_fused_join_aggregate (executor.rs:333-458) */
int oracle_join_aggregate(const struct ArrowArray* const* probes,
                          const struct ArrowSchema* probe_schema, int n_probes,
                          const struct ArrowArray* build, const struct ArrowSchema* build_schema,
                          const int32_t* probe_keys, const int32_t* build_keys, int n_keys,
                          const int32_t* cols, int n_cols, const prism_expr* exprs,
                          int n_exprs, const prism_agg_config* agg, int n_threads,
                          struct ArrowArray* out, struct ArrowSchema* out_schema);

/* Correctly rounded sum of n doubles (exact big-integer accumulation). */
double oracle_exact_sum_f64(const double* values, int64_t n);

#ifdef __cplusplus
}
#endif

#endif /* PRISM_ORACLE_H */
