/*
 * prism_gpu.h — C ABI of the B200 (sm_100a) hash join / hash aggregate /
 * filter-project engine.
 *
 * The entry points mirror the Rust operator API of prism-executor
 * (native/prism-executor/src/lib.rs:5-15) one function per reference
 * function, with arrow-rs `RecordBatch` carried across the boundary as the
 * Arrow C Data Interface (prism_arrow_c.h). Every function:
 *   - borrows its inputs; outputs are new objects owned by the caller;
 *   - returns a status code (PRISM_OK or one of PRISM_ERR_*) and never aborts
 *     the process; the message of the last failure on a context is available
 *     from prism_last_error();
 *   - is safe to call from several host threads on the same context (calls
 *     are serialised on the context's stream; use one context per stream for
 *     overlap).
 *
 * Two call styles exist:
 *   1. "Arrow" style (suffix _arrow): host ArrowArray/ArrowSchema in, host
 *      ArrowArray/ArrowSchema out. Each call uploads its inputs, runs on the
 *      device and downloads the result — the drop-in replacement for the
 *      reference function of the same name.
 *   2. Resident style: prism_batch handles that live in device memory
 *      (imported once with prism_batch_import / prism_batch_import_device and
 *      exported with prism_batch_export). Operators chain on the device with
 *      no host round trip; build-side hash tables stay resident across probes
 *      (the analogue of the reference's PartitionStore,
 *      native/prism-flight/src/shuffle_writer.rs:42-86). A resident result may
 *      still be in flight when the call returns: it is ordered on the
 *      context's stream, so calls on the same context and prism_batch_export
 *      see it complete; other streams or host readers of its device buffers
 *      call prism_ctx_synchronize first.
 *
 * Tree-shaped configuration (Predicate, ScalarExpr) crosses as flat arrays of
 * POD nodes in post-order (children before parent).
 */
#ifndef PRISM_GPU_H
#define PRISM_GPU_H

#include <stddef.h>
#include <stdint.h>

#include "prism_arrow_c.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Status codes. 1..7 mirror the PrismError variants                         */
/* (native/prism-executor/src/error.rs:6-27); 8..11 are device conditions.   */
/* ------------------------------------------------------------------------ */
#define PRISM_OK 0
#define PRISM_ERR_ARROW 1
#define PRISM_ERR_SCHEMA_MISMATCH 2
#define PRISM_ERR_INVALID_ARGUMENT 3
#define PRISM_ERR_EXECUTION 4
#define PRISM_ERR_JOIN 5
#define PRISM_ERR_UNSUPPORTED_AGGREGATION 6
#define PRISM_ERR_INTERNAL 7
#define PRISM_ERR_TABLE_FULL 8
#define PRISM_ERR_NO_MEMORY 9
#define PRISM_ERR_TIMEOUT 10
#define PRISM_ERR_CUDA 11

/* ------------------------------------------------------------------------ */
/* Configuration PODs                                                        */
/* ------------------------------------------------------------------------ */

/* JoinType (native/prism-executor/src/hash_join.rs:48-56). */
#define PRISM_JOIN_INNER 0
#define PRISM_JOIN_LEFT 1
#define PRISM_JOIN_RIGHT 2
#define PRISM_JOIN_FULL 3
#define PRISM_JOIN_LEFT_SEMI 4
#define PRISM_JOIN_LEFT_ANTI 5

/* HashJoinConfig (hash_join.rs:59-64). probe_keys[i] pairs with build_keys[i]. */
typedef struct prism_join_config {
  int32_t join_type;
  int32_t n_keys;
  const int32_t* probe_keys;
  const int32_t* build_keys;
} prism_join_config;

/* AggFunc (native/prism-executor/src/hash_aggregate.rs:79-86). */
#define PRISM_AGG_SUM 0
#define PRISM_AGG_COUNT 1
#define PRISM_AGG_AVG 2
#define PRISM_AGG_MIN 3
#define PRISM_AGG_MAX 4
#define PRISM_AGG_COUNT_DISTINCT 5

/* AggExpr (hash_aggregate.rs:90-94). */
typedef struct prism_agg_expr {
  int32_t column;
  int32_t func;
  const char* output_name; /* NUL-terminated UTF-8 */
} prism_agg_expr;

/* HashAggConfig (hash_aggregate.rs:98-101). */
typedef struct prism_agg_config {
  int32_t n_group_by;
  const int32_t* group_by;
  int32_t n_aggs;
  const prism_agg_expr* aggs;
} prism_agg_config;

/* ScalarValue (native/prism-executor/src/filter_project.rs:55-62). */
#define PRISM_SCALAR_INT32 0
#define PRISM_SCALAR_INT64 1
#define PRISM_SCALAR_FLOAT64 2
#define PRISM_SCALAR_UTF8 3
#define PRISM_SCALAR_BOOLEAN 4
#define PRISM_SCALAR_DATE32 5

typedef struct prism_scalar {
  int32_t type;     /* PRISM_SCALAR_* */
  int32_t reserved;
  int64_t i64;      /* INT32, INT64, DATE32, BOOLEAN (0/1) */
  double f64;       /* FLOAT64 */
  const char* str;  /* UTF8 bytes (not necessarily NUL-terminated) */
  int64_t str_len;
} prism_scalar;

/* Predicate (filter_project.rs:22-51). */
#define PRISM_PRED_LITERAL 0
#define PRISM_PRED_EQ 1
#define PRISM_PRED_NE 2
#define PRISM_PRED_LT 3
#define PRISM_PRED_LE 4
#define PRISM_PRED_GT 5
#define PRISM_PRED_GE 6
#define PRISM_PRED_IS_NULL 7
#define PRISM_PRED_IS_NOT_NULL 8
#define PRISM_PRED_AND 9
#define PRISM_PRED_OR 10
#define PRISM_PRED_NOT 11
#define PRISM_PRED_LIKE 12
#define PRISM_PRED_ILIKE 13

/* One predicate node. LITERAL uses value.i64 (0/1); comparisons use column +
 * value; IS_NULL/IS_NOT_NULL use column; LIKE/ILIKE use column + value.str as
 * the pattern; AND/OR pop two operands, NOT pops one. */
typedef struct prism_pred_node {
  int32_t op;
  int32_t column;
  prism_scalar value;
} prism_pred_node;

typedef struct prism_predicate {
  const prism_pred_node* nodes; /* post-order */
  int32_t n_nodes;
} prism_predicate;

/* ScalarExpr (filter_project.rs:186-213). */
#define PRISM_EXPR_COLUMN 0
#define PRISM_EXPR_LITERAL 1
#define PRISM_EXPR_ADD 2
#define PRISM_EXPR_SUB 3
#define PRISM_EXPR_MUL 4
#define PRISM_EXPR_DIV 5
#define PRISM_EXPR_NEG 6
#define PRISM_EXPR_IF_THEN 7

/* One expression node. ADD..DIV pop two operands (left pushed first), NEG
 * pops one. IF_THEN pops n_clauses "then" expressions followed by the else
 * expression when has_else != 0 (all pushed in that order); clause i's
 * predicate is preds[clauses[clause_begin + i].pred_begin ...
 * + pred_len) of the enclosing prism_expr. */
typedef struct prism_expr_node {
  int32_t op;
  int32_t column;
  prism_scalar literal;
  int32_t n_clauses;
  int32_t has_else;
  int32_t clause_begin;
  int32_t reserved;
} prism_expr_node;

typedef struct prism_expr_clause {
  int32_t pred_begin;
  int32_t pred_len;
} prism_expr_clause;

typedef struct prism_expr {
  const prism_expr_node* nodes; /* post-order */
  int32_t n_nodes;
  const prism_pred_node* preds; /* pool for IF_THEN clause predicates */
  int32_t n_preds;
  const prism_expr_clause* clauses;
  int32_t n_clauses;
} prism_expr;

/* Arithmetic mode of projected expressions.
 * F64: the reference's semantics — both operands of every binary operation
 *      are cast to Float64 (filter_project.rs:233-247).
 * EXACT: integer and decimal operands are computed exactly in 128-bit
 *      integers (decimal scales add under MUL and align under ADD/SUB); the
 *      result column is Decimal128(38, s); sums over it are exact. Division
 *      and any Float64 operand fall back to F64 for that node. */
#define PRISM_ARITH_F64 0
#define PRISM_ARITH_EXACT 1

/* Special output-column codes for prism_join_project. */
#define PRISM_COL_PROBE_ROW_INDEX (-1)
#define PRISM_COL_BUILD_ROW_INDEX (-2)

/* ------------------------------------------------------------------------ */
/* Opaque handles                                                            */
/* ------------------------------------------------------------------------ */
typedef struct prism_ctx prism_ctx;
typedef struct prism_batch prism_batch;
typedef struct prism_hash_table prism_hash_table;

/* ------------------------------------------------------------------------ */
/* Context                                                                   */
/* ------------------------------------------------------------------------ */

/* Creates a context on CUDA device `device`. memory_budget_bytes caps the
 * device memory the context's allocator may hold (0 = 90% of free memory);
 * allocations over budget fail with PRISM_ERR_NO_MEMORY. */
int prism_ctx_create(int device, uint64_t memory_budget_bytes, prism_ctx** out);
void prism_ctx_destroy(prism_ctx* ctx);
/* Message of the last failed call on this context ("" if none). The pointer
 * stays valid until the next call on the context. */
const char* prism_last_error(const prism_ctx* ctx);
/* Runs subsequent work on `cuda_stream` (a cudaStream_t; NULL restores the
 * context's own stream). */
int prism_ctx_set_stream(prism_ctx* ctx, void* cuda_stream);
int prism_ctx_synchronize(prism_ctx* ctx);
/* Device bytes currently held by the context's allocator. */
uint64_t prism_ctx_bytes_in_use(const prism_ctx* ctx);
/* Number of kernels this context has launched since creation. */
uint64_t prism_ctx_kernel_launches(const prism_ctx* ctx);
/* Per-kernel device timing: when enabled, the hot kernels (probe, build
 * insert, aggregation, predicate, expression) are bracketed by CUDA events on
 * the context's stream. prism_ctx_kernel_stats synchronises and returns the
 * launch count and summed device milliseconds of the kernel `name` since
 * profiling was (re-)enabled. */
int prism_ctx_set_profiling(prism_ctx* ctx, int enable);
int prism_ctx_kernel_stats(prism_ctx* ctx, const char* name, uint64_t* launches, double* total_ms);
/* Per-query kernels compiled at run time (NVRTC, process-wide cache): sets
 * *enabled (0 when PRISM_JIT=0 or libnvrtc.so.12 is absent; the
 * interpreting kernels then run), the number of compilations so far and their
 * summed wall time. No counterpart in the reference (its operators are
 * compiled Rust). Any pointer may be NULL. */
int prism_jit_stats(int32_t* enabled, int64_t* compiles, double* total_ms);
const char* prism_version(void);

/* ------------------------------------------------------------------------ */
/* Device-resident batches                                                   */
/* ------------------------------------------------------------------------ */

/* Copies a host RecordBatch (exported as a struct array) to the device.
 * The caller keeps ownership of `array`/`schema` (they are not released). */
int prism_batch_import(prism_ctx* ctx, const struct ArrowArray* array,
                       const struct ArrowSchema* schema, prism_batch** out);
/* Wraps a batch whose buffers already live in device memory (device_type
 * ARROW_DEVICE_CUDA) without copying; the caller keeps the buffers alive for
 * the lifetime of the batch. Host (ARROW_DEVICE_CPU / CUDA_HOST) arrays are
 * copied as by prism_batch_import. */
int prism_batch_import_device(prism_ctx* ctx, const struct ArrowDeviceArray* array,
                              const struct ArrowSchema* schema, prism_batch** out);
/* Copies a device batch back to host memory as a struct array. The caller
 * owns the result and must call its release callbacks. */
int prism_batch_export(prism_ctx* ctx, const prism_batch* batch,
                       struct ArrowArray* out_array, struct ArrowSchema* out_schema);
int64_t prism_batch_num_rows(const prism_batch* batch);
int32_t prism_batch_num_columns(const prism_batch* batch);
/* Device buffers of column `col` without a copy (the batch keeps them alive):
 * values (fixed width; a Utf8 column's offsets), validity bitmap (NULL when
 * the column has no nulls), element width in bytes and Arrow type id as in
 * the engine (0 when unknown). Lets a caller hand result columns to its own
 * device code (as ArrowDeviceArray export would). No counterpart in the
 * reference, whose batches are host memory. */
int prism_batch_column_device(const prism_batch* batch, int32_t col, const void** values, const uint8_t** validity,
                              int32_t* width);
void prism_batch_free(prism_batch* batch);

/* ------------------------------------------------------------------------ */
/* Hash join (native/prism-executor/src/hash_join.rs)                        */
/* ------------------------------------------------------------------------ */

/* HashTable::build (hash_join.rs:87-141). The table keeps a reference to the
 * build batch; the batch must outlive the table. */
int prism_hash_table_build(prism_ctx* ctx, const prism_batch* build,
                           const int32_t* key_cols, int32_t n_keys,
                           prism_hash_table** out);
/* HashTable::probe (hash_join.rs:143-200). Output: 2 columns
 * (probe_idx UInt32, build_idx UInt32), probe rows ascending and, per probe
 * row, build rows ascending — the reference's emission order. */
int prism_hash_table_probe(prism_ctx* ctx, const prism_hash_table* table,
                           const prism_batch* probe, const int32_t* key_cols,
                           int32_t n_keys, prism_batch** out);
/* Probe that allocates nothing. No counterpart in the reference: it exists
 * for callers that may not allocate device memory while they run — e.g. a
 * host engine that reserved its whole device-memory budget up front and owns
 * every buffer through its own pool, or a plugin whose host forbids driver
 * allocations mid-query. The caller passes device pointers: `probe_keys`
 * (n_probe Int64 keys) and the outputs `out_probe_idx` / `out_build_idx`
 * (UInt32, room for `out_capacity` matches); results equal
 * prism_hash_table_probe's, in the same order. The table must have a single
 * Int64 key column. Scratch is a file-scope device array of 1 MiB that every
 * GPU loading the library keeps until exit; it bounds n_probe to
 * 268,435,456 rows (larger inputs are rejected with
 * PRISM_ERR_INVALID_ARGUMENT). The first call on each device looks up that
 * array's device address (cudaGetSymbolAddress) with the device current; make
 * that first call before any stream capture. Every call shares the array and
 * clears the part it uses; calls that overlap on the GPU race. When more
 * matches exist than out_capacity, the first out_capacity matches (in the
 * order above, also when a probe row's matches straddle the capacity) are
 * written and nothing past them, *out_matches receives the full count and
 * the call returns PRISM_ERR_INVALID_ARGUMENT. */
int prism_hash_table_probe_noalloc(prism_ctx* ctx, const prism_hash_table* table,
                                   const int64_t* probe_keys, int64_t n_probe,
                                   uint32_t* out_probe_idx, uint32_t* out_build_idx,
                                   int64_t out_capacity, int64_t* out_matches);
int64_t prism_hash_table_num_rows(const prism_hash_table* table);
int prism_hash_table_has_duplicates(const prism_hash_table* table);
/* How the table is laid out in HBM (no reference counterpart; the Rust
 * HashTable is one hashbrown map per partition): PRISM_TABLE_HASH
 * (open-addressing slots), PRISM_TABLE_DENSE (a direct row per key value,
 * chosen for unique Int64 keys over a compact range); -1 for a null table. */
#define PRISM_TABLE_HASH 0
#define PRISM_TABLE_DENSE 1
int prism_hash_table_layout(const prism_hash_table* table);
void prism_hash_table_free(prism_hash_table* table);

/* Fused probe + gather: emits the selected columns of the inner join of
 * `probe` with the table's build batch, in the reference's match order.
 * out_cols index the joined schema (probe columns, then build columns, as in
 * executor.rs:474-551 project_join_matches); PRISM_COL_PROBE_ROW_INDEX and
 * PRISM_COL_BUILD_ROW_INDEX emit the matched row indices as UInt32. */
int prism_join_project(prism_ctx* ctx, const prism_hash_table* table,
                       const prism_batch* probe, const int32_t* probe_keys,
                       int32_t n_keys, const int32_t* out_cols, int32_t n_out,
                       prism_batch** out);
/* prism_join_project with flags. PRISM_JOIN_ANY_ORDER: the caller takes the
 * matches as a multiset (the executor's fused join -> aggregate consumes
 * them that way, executor.rs:474-551): the matches come in no particular
 * order (each 2,048-row tile's matches form one contiguous run of the output),
 * so the probe needs one pass and no ordering step. The set of output rows is
 * the same as without the flag. */
#define PRISM_JOIN_ANY_ORDER 1u
int prism_join_project_ex(prism_ctx* ctx, const prism_hash_table* table,
                          const prism_batch* probe, const int32_t* probe_keys,
                          int32_t n_keys, const int32_t* out_cols, int32_t n_out,
                          uint32_t flags, prism_batch** out);

/* hash_join (hash_join.rs:312-365). */
int prism_hash_join(prism_ctx* ctx, const prism_batch* probe, const prism_batch* build,
                    const prism_join_config* config, prism_batch** out);
/* probe_matches_chunked (hash_join.rs:286-309): one (probe_idx, build_idx)
 * batch per probe batch, written to out[0..n_probes). */
int prism_probe_matches_chunked(prism_ctx* ctx, const prism_batch* const* probes,
                                int32_t n_probes, const prism_batch* build,
                                const int32_t* probe_keys, const int32_t* build_keys,
                                int32_t n_keys, prism_batch** out);
/* hash_join_probe_chunked (hash_join.rs:206-282): empty outputs are
 * dropped; *n_out receives the number written to out (capacity n_probes). */
int prism_hash_join_probe_chunked(prism_ctx* ctx, const prism_batch* const* probes,
                                  int32_t n_probes, const prism_batch* build,
                                  const prism_join_config* config, prism_batch** out,
                                  int32_t* n_out);

/* ------------------------------------------------------------------------ */
/* Hash aggregation (native/prism-executor/src/hash_aggregate.rs)            */
/* ------------------------------------------------------------------------ */

/* hash_aggregate (hash_aggregate.rs:174-176). */
int prism_hash_aggregate(prism_ctx* ctx, const prism_batch* batch,
                         const prism_agg_config* config, prism_batch** out);
/* hash_aggregate_batches (hash_aggregate.rs:182-339). Groups are emitted in
 * first-seen order over the concatenated batches, as the reference does. */
int prism_hash_aggregate_batches(prism_ctx* ctx, const prism_batch* const* batches,
                                 int32_t n_batches, const prism_agg_config* config,
                                 prism_batch** out);

/* ------------------------------------------------------------------------ */
/* Filter / project (native/prism-executor/src/filter_project.rs)            */
/* ------------------------------------------------------------------------ */

/* evaluate_predicate (filter_project.rs:65-123): one Boolean column. */
int prism_evaluate_predicate(prism_ctx* ctx, const prism_batch* batch,
                             const prism_predicate* predicate, prism_batch** out_mask);
/* filter_batch (filter_project.rs:126-135); mask = a 1-column Boolean batch. */
int prism_filter_batch(prism_ctx* ctx, const prism_batch* batch, const prism_batch* mask,
                       prism_batch** out);
/* project_batch (filter_project.rs:138-160). */
int prism_project_batch(prism_ctx* ctx, const prism_batch* batch, const int32_t* cols,
                        int32_t n_cols, prism_batch** out);
/* filter_and_project (filter_project.rs:163-180); predicate may be NULL. */
int prism_filter_and_project(prism_ctx* ctx, const prism_batch* batch,
                             const prism_predicate* predicate, const int32_t* cols,
                             int32_t n_cols, prism_batch** out);
/* evaluate_scalar_expr (filter_project.rs:216-294): one column. */
int prism_evaluate_scalar_expr(prism_ctx* ctx, const prism_batch* batch,
                               const prism_expr* expr, int32_t arith_mode,
                               prism_batch** out);
/* project_batch_with_exprs (filter_project.rs:305-333). */
int prism_project_batch_with_exprs(prism_ctx* ctx, const prism_batch* batch,
                                   const int32_t* cols, int32_t n_cols,
                                   const prism_expr* exprs, int32_t n_exprs,
                                   int32_t arith_mode, prism_batch** out);

/* ------------------------------------------------------------------------ */
/* Fused operators                                                           */
/* ------------------------------------------------------------------------ */

/* filter -> project_batch_with_exprs -> hash_aggregate_batches in one pass
 * over the input (no filtered or projected intermediate is materialised).
 * The aggregate config indexes the projected schema (cols, then expr_i). */
int prism_filter_project_aggregate(prism_ctx* ctx, const prism_batch* const* batches,
                                   int32_t n_batches, const prism_predicate* predicate,
                                   const int32_t* cols, int32_t n_cols,
                                   const prism_expr* exprs, int32_t n_exprs,
                                   int32_t arith_mode, const prism_agg_config* agg,
                                   prism_batch** out);
/* Inner join -> project -> aggregate, the semantics of the reference's fused
 * join-aggregate (native/prism-substrait/src/executor.rs:333-458): cols and
 * exprs index the joined schema; the aggregate config indexes the projected
 * schema. No joined rows are materialised. */
int prism_join_aggregate(prism_ctx* ctx, const prism_batch* const* probes, int32_t n_probes,
                         const prism_batch* build, const int32_t* probe_keys,
                         const int32_t* build_keys, int32_t n_keys, const int32_t* cols,
                         int32_t n_cols, const prism_expr* exprs, int32_t n_exprs,
                         const prism_agg_config* agg, prism_batch** out);

/* ------------------------------------------------------------------------ */
/* Sort / top-N (native/prism-executor/src/sort.rs)                          */
/* ------------------------------------------------------------------------ */
/* SortKey (sort.rs:28-32): SortDirection Asc/Desc, NullOrdering
 * NullsFirst/NullsLast. */
typedef struct prism_sort_key {
  int32_t column;
  int32_t descending;   /* 0 Asc, 1 Desc */
  int32_t nulls_first;  /* 1 NullsFirst, 0 NullsLast */
} prism_sort_key;

/* sort_batch (sort.rs:35-54) with limit < 0, sort_batch_limit (sort.rs:56-78)
 * with limit >= 0, and topn_single_col (sort.rs:97-146) as a Float64
 * descending key with a limit: the rows ordered by the keys (most
 * significant first), integers numerically, floats by IEEE totalOrder,
 * Utf8 / dictionary values bytewise then by length, Decimal128 numerically;
 * ties keep the input order. An empty batch or key list returns the batch. */
int prism_sort_batch(prism_ctx* ctx, const prism_batch* batch, const prism_sort_key* keys, int32_t n_keys,
                     int64_t limit, prism_batch** out);

/* ------------------------------------------------------------------------ */
/* Parquet scan (native/prism-executor/src/parquet_scan.rs)                 */
/* ------------------------------------------------------------------------ */
/* ParquetScanConfig (parquet_scan.rs:29-50). */
typedef struct prism_parquet_scan_config {
  const char* const* uris;        /* local paths or file:// URIs: a file, or a directory scanned for *.parquet */
  int32_t n_uris;
  const prism_predicate* predicate; /* NULL: no row-group skipping */
  const int32_t* projection;      /* NULL: all columns */
  int32_t n_projection;
  int64_t batch_size;             /* rows per output batch (> 0) */
  int32_t skip_expand;
  /* target_schema (parquet_scan.rs:45-50, NULL: none): a struct schema. A
   * scan without a projection adapts every batch to it (adapt_batch_to_schema,
   * parquet_scan.rs:306-339): the target's fields in its order, matched by
   * name; a column of another type cast as arrow's safe cast does (a value
   * the target cannot hold becomes null; the GPU casts between numeric,
   * Boolean and Date32 types, others fail with PRISM_ERR_INTERNAL); a missing
   * column all null; a non-nullable field holding a null fails. With a
   * projection the batches stay file-native and are expanded to the target
   * schema instead of the first file's. */
  const struct ArrowSchema* target_schema;
} prism_parquet_scan_config;

typedef struct prism_parquet_scan_stats {
  int64_t files, row_groups, row_groups_skipped, pages;
  int64_t compressed_bytes;  /* column-chunk bytes read (staged to the device) */
  int64_t inflated_bytes;    /* page bytes after decompression (compressed pages only) */
  int64_t decoded_bytes;     /* Arrow bytes produced: values, offsets and string data */
} prism_parquet_scan_stats;

/* parquet_scan (parquet_scan.rs:55-168): the files of every URI (sorted
 * within a URI), their row groups minus those whose statistics rule the
 * predicate out (row_group_might_match, parquet_scan.rs:355-469), the
 * projected columns (ProjectionMask::roots: valid indices in file order; none
 * valid reads all), decoded on the GPU into device batches of at most
 * batch_size rows that never span row groups; with a projection shorter than
 * the schema and skip_expand == 0 the batches are expanded back to the first
 * file's schema with all-null columns (expand_projected_batches,
 * parquet_scan.rs:471-526). *out is a library-allocated array of *n_out
 * batches (free each with prism_batch_free, the array with prism_free_array);
 * stats may be NULL. The GPU decoder reads flat schemas of BOOLEAN, INT32,
 * DATE, INT64, FLOAT, DOUBLE and UTF8 byte-array columns, PLAIN and dictionary
 * encodings, data pages V1 and V2, UNCOMPRESSED or SNAPPY chunks; other files
 * fail with PRISM_ERR_INVALID_ARGUMENT, unreadable or malformed ones with
 * PRISM_ERR_INTERNAL (the reference's PrismError::Internal). */
int prism_parquet_scan(prism_ctx* ctx, const prism_parquet_scan_config* config, prism_batch*** out, int32_t* n_out,
                       prism_parquet_scan_stats* stats);

/* The scan in two steps, for tables kept in HBM still compressed (a
 * compressed table takes a fraction of its decoded size in the 180 GB):
 * prism_parquet_prepare reads every selected column chunk (the same file,
 * row-group and column selection as prism_parquet_scan) into device memory
 * and walks its page headers; prism_parquet_decode decodes the prepared
 * chunks on the GPU into batches, as often as called (each call returns new
 * batches, as prism_parquet_scan would), on the context that prepared them
 * (their inflate buffer is reused, in that context's stream order). A
 * prepared scan holds the compressed chunks plus that buffer (the inflated
 * page bytes). No counterpart in the reference. */
typedef struct prism_parquet_prepared prism_parquet_prepared;
int prism_parquet_prepare(prism_ctx* ctx, const prism_parquet_scan_config* config, prism_parquet_prepared** out,
                          prism_parquet_scan_stats* stats);
int prism_parquet_decode(prism_ctx* ctx, const prism_parquet_prepared* prepared, prism_batch*** out, int32_t* n_out,
                         prism_parquet_scan_stats* stats);
int64_t prism_parquet_prepared_rows(const prism_parquet_prepared* prepared);
int64_t prism_parquet_prepared_bytes(const prism_parquet_prepared* prepared);
void prism_parquet_prepared_free(prism_parquet_prepared* prepared);

/* parquet_row_count (parquet_scan.rs:240-266): rows of the row groups the
 * predicate (NULL: none) might match, from the footers alone. */
int prism_parquet_row_count(const char* const* uris, int32_t n_uris, const prism_predicate* predicate,
                            int64_t* count);

/* Frees an array the library allocated (not the batches in it). */
void prism_free_array(void* array);

/* ------------------------------------------------------------------------ */
/* Distributed aggregation: the exchange step                               */
/* (native/prism-bench/src/handler.rs:270-344)                              */
/* ------------------------------------------------------------------------ */
/* The reference runs the aggregation on every worker with AVG expanded into
 * SUM + COUNT, ships each worker's partial batch to a reducer over Flight,
 * and merges there. The replacement: each GPU computes its partial with
 * prism_hash_aggregate_batches (or the fused paths) under the expanded
 * config, packs it into one device buffer, the buffers are all-gathered
 * (ncclAllGather over NVLink; pad every rank's buffer to the largest size),
 * and every rank unpacks them and merges on the GPU.
 *
 * expand_worker_aggregates (handler.rs:397-428): writes the worker
 * aggregate list of `original` (AVG -> SUM then COUNT of its column, every
 * other aggregate unchanged, output names "agg_<i>" with process lifetime)
 * into out_aggs (room for 2 * original->n_aggs entries); *n_out = its
 * length. Group-by columns are unchanged. Host-only; no context needed. */
int prism_expand_worker_aggregates(const prism_agg_config* original, prism_agg_expr* out_aggs,
                                   int32_t capacity, int32_t* n_out);

/* Bytes prism_batch_pack writes for `batch` (a multiple of 16). */
int prism_batch_packed_size(const prism_batch* batch, uint64_t* size);

/* Writes `batch` (header + every buffer, 16-byte aligned) into the device
 * buffer device_dst of `capacity` bytes, stream-ordered on the context's
 * stream: synchronise it (or order on it) before a collective reads the
 * buffer. No counterpart in the reference (Flight IPC encoding,
 * handler.rs:570-624). */
int prism_batch_pack(prism_ctx* ctx, const prism_batch* batch, void* device_dst, uint64_t capacity);

/* Reads a packed batch from device memory [device_src, device_src + size)
 * into a new device batch that owns a copy of the payload (the source may be
 * reused once this returns). Checks the header and every buffer range
 * against `size`; synchronises the context's stream. */
int prism_batch_unpack(prism_ctx* ctx, const void* device_src, uint64_t size, prism_batch** out);
/* The same packed format on the host, for exchanges whose transport is host
 * memory (a gloo or TCP group, a file): a host struct array packed into host
 * memory, and a host packed buffer read back into a host struct array (the
 * result owns a copy). No device or context is needed; a packed buffer made
 * by either side unpacks on either side. */
int prism_arrow_packed_size(const struct ArrowArray* batch, const struct ArrowSchema* schema, uint64_t* size);
int prism_arrow_pack(const struct ArrowArray* batch, const struct ArrowSchema* schema, void* host_dst,
                     uint64_t capacity);
int prism_arrow_unpack(const void* host_src, uint64_t size, struct ArrowArray* out,
                       struct ArrowSchema* out_schema);

/* The reducer merge (handler.rs:327-344): hash_aggregate_batches over the
 * partials (in the given order: the reference puts the reducer's own first,
 * then its peers) with build_final_merge_config (handler.rs:430-457: SUM for
 * SUM / COUNT / COUNT DISTINCT partials, MIN / MAX for MIN / MAX), then
 * reconstruct_original_aggregate_batch (handler.rs:459-530): the group
 * columns, then per original aggregate COUNT / COUNT DISTINCT as Int64, AVG
 * as SUM / COUNT (0 when the count is 0), SUM / MIN / MAX as Float64, a null
 * read as 0. Every partial has original->n_group_by group columns followed by
 * the expanded worker aggregates. COUNT DISTINCT merges by summing the
 * workers' distinct counts, as the reference does. */
int prism_merge_partial_aggregates(prism_ctx* ctx, const prism_batch* const* partials, int32_t n_partials,
                                   const prism_agg_config* original, prism_batch** out);

/* ------------------------------------------------------------------------ */
/* Serving loop (prism_serve_submit/poll of the design)                       */
/* ------------------------------------------------------------------------ */
/* Requests of uneven sizes against resident tables, answered by worker
 * threads that each own a context and stream: small requests of one shape
 * that arrive close together share a launch, the smallest ready job goes to
 * the next free worker, and a job starts only while its device footprint
 * fits the budget. Every result equals the result of the request run alone.
 * No counterpart in the reference (its Flight handler runs one operator call
 * at a time, prism-flight/src/handler.rs; PartitionStore,
 * shuffle_writer.rs:42-86, is the resident-table analogue).
 *
 * Lifetimes: tables, request batches and key buffers stay owned by the
 * caller and must outlive their requests; result batches belong to the
 * caller (prism_batch_free) and stay valid after prism_server_destroy, which
 * therefore retires its worker contexts instead of destroying them (their
 * streams stay until exit; their unused device memory is released).
 * Key buffers and request batches must be complete on the device when
 * submitted. Results are complete when poll returns them. */
typedef struct prism_server prism_server;

/* workers: 1-64 worker threads; budget_bytes: device bytes admitted jobs may
 * hold at once (0 = 120 GB); requests below coalesce_rows rows may share a
 * launch with up to max_coalesce - 1 others. */
int prism_server_create(int32_t device, uint64_t budget_bytes, int32_t workers, int64_t coalesce_rows,
                        int32_t max_coalesce, prism_server** out);
/* Registers a resident table (single Int64 key); probes emit
 * (probe row, build column payload_col). */
int prism_server_add_table(prism_server* server, const prism_hash_table* table, int32_t payload_col,
                           int32_t* table_id);
/* Submits a probe of table_id with n device-resident Int64 keys; the result
 * batch is [probe_idx (UInt32, rows of `keys`, ascending), payload]. */
int prism_serve_probe(prism_server* server, int32_t table_id, const int64_t* keys, int64_t n, int64_t* ticket);
/* The device work queue (no counterpart in the reference): with enable != 0,
 * probes of registered tables with unique Int64 keys and a fixed-width,
 * null-free payload, of at most max_rows rows (0: any), no longer go to the
 * worker threads: their descriptors go into a ring in device memory, and ONE
 * persistent kernel (ctas_per_sm CTAs per SM, 1 or 2; 0: 1, which leaves
 * room beside it for a GROUP BY kernel's block on every SM) drains it tile
 * by tile (2,048 probe rows), requests of different tables and sizes sharing
 * the launch; a host thread reports each request when its last tile is done.
 * Their matches come as a multiset: runs of consecutive probe rows in any
 * order, rows ascending inside a run. Every wait of the kernel is bounded:
 * idle CTAs exit after about 0.1 ms (the kernel is relaunched when work
 * arrives), and a CTA that waits wait_limit_ms (0: 1000) for a request's
 * descriptor gives up, every request then in flight fails with
 * PRISM_ERR_TIMEOUT, and the queue is reset and stays usable. enable = 0
 * sends new probes back to the workers. */
int prism_server_set_device_queue(prism_server* server, int32_t enable, int64_t max_rows, int32_t ctas_per_sm,
                                  int32_t wait_limit_ms);
/* Failure injection for tests of the bounded wait above: publishes a request
 * whose descriptor is never written; its ticket (and every request in flight
 * with it) fails with PRISM_ERR_TIMEOUT after wait_limit_ms. */
int prism_server_inject_unready(prism_server* server, int64_t* ticket);
/* Submits hash_aggregate(batch, config) (the config is copied). */
int prism_serve_aggregate(prism_server* server, const prism_batch* batch, const prism_agg_config* config,
                          int64_t* ticket);
/* Waits up to wait_ms (-1: until done, 0: no wait) for a ticket. Returns
 * PRISM_OK with the result in *out, the request's own error status (message
 * in prism_server_last_error), or PRISM_ERR_TIMEOUT while it is not done.
 * A ticket's result is returned once; poll one ticket from one thread. */
int prism_serve_poll(prism_server* server, int64_t ticket, int32_t wait_ms, prism_batch** out);
/* Waits up to wait_ms (-1: until one is) for a finished ticket not yet
 * reported by this call, in completion order; PRISM_ERR_TIMEOUT when none.
 * (Its result is then taken with prism_serve_poll.) */
int prism_serve_wait_any(prism_server* server, int32_t wait_ms, int64_t* ticket);
const char* prism_server_last_error(prism_server* server);
/* Finishes every submitted request, then stops the workers. */
void prism_server_destroy(prism_server* server);

/* ------------------------------------------------------------------------ */
/* Autotuner and the per-shape tuning table                                  */
/* ------------------------------------------------------------------------ */
/* No counterpart in the reference, whose one knob on this path is the
 * compile-time HASH_PARTITIONS = 64 (hash_join.rs:43). Each prism_tune_* call
 * times candidate settings of one operator on the caller's data (CUDA
 * events, median of repeated runs after a warm-up), records the fastest for
 * the input's shape class in the process-wide tuning table, and reports
 * every candidate in *result (may be NULL). Later calls of that shape class
 * use the record; settings given through the environment (PRISM_JOIN_DENSE,
 * PRISM_JOIN_PARTITION, PRISM_JOIN_AGG_SHAPE, PRISM_HASH_AGG_BLOCK) take
 * precedence. Shape classes: joins and join -> aggregates by key kind
 * (single Int64 or general) and log2 of the build rows; hashed-groups
 * aggregation by log2 of the input rows. The table is loaded from the file
 * named by PRISM_TUNING_FILE at first use, and saved / loaded explicitly
 * below (a text file, one record per line). */
#define PRISM_TUNE_MAX_CANDIDATES 16
typedef struct prism_tune_result {
  int32_t n_candidates;
  int32_t best;                                /* index of the fastest */
  double ms[PRISM_TUNE_MAX_CANDIDATES];        /* median time of each candidate */
  char desc[PRISM_TUNE_MAX_CANDIDATES][64];    /* each candidate's settings */
} prism_tune_result;
/* Join table layout (dense rows / hash slots), load factor and the
 * radix-partitioned build + probe (off, 2^8 or 2^6 partitions), timed as a
 * table build plus one probe (flags: PRISM_JOIN_ANY_ORDER as the calls to
 * be tuned will pass it). */
int prism_tune_join(prism_ctx* ctx, const prism_batch* build, const prism_batch* probe, const int32_t* build_keys,
                    const int32_t* probe_keys, int32_t n_keys, uint32_t flags, prism_tune_result* result);
/* The fused join -> aggregate kernel's shape (threads per block, blocks per
 * SM, probe rows in flight, group-table slots), timed as whole
 * prism_join_aggregate calls with these arguments. */
int prism_tune_join_aggregate(prism_ctx* ctx, const prism_batch* const* probes, int32_t n_probes,
                              const prism_batch* build, const int32_t* probe_keys, const int32_t* build_keys,
                              int32_t n_keys, const int32_t* cols, int32_t n_cols, const prism_expr* exprs,
                              int32_t n_exprs, const prism_agg_config* agg, prism_tune_result* result);
/* The hashed-groups aggregation kernel's block size, timed as whole
 * prism_hash_aggregate_batches calls. */
int prism_tune_hash_aggregate(prism_ctx* ctx, const prism_batch* const* batches, int32_t n_batches,
                              const prism_agg_config* config, prism_tune_result* result);
int prism_tuning_save(const char* path);
int prism_tuning_load(const char* path);  /* merges the file's records into the table */
void prism_tuning_clear(void);
/* The table in its file format: copies at most capacity - 1 bytes and a NUL;
 * returns the full length. */
int64_t prism_tuning_dump(char* buf, int64_t capacity);

/* ------------------------------------------------------------------------ */
/* Arrow-style wrappers: host batches in, host batch out                     */
/* ------------------------------------------------------------------------ */
int prism_hash_join_arrow(prism_ctx* ctx, const struct ArrowArray* probe,
                          const struct ArrowSchema* probe_schema,
                          const struct ArrowArray* build,
                          const struct ArrowSchema* build_schema,
                          const prism_join_config* config, struct ArrowArray* out,
                          struct ArrowSchema* out_schema);
int prism_hash_aggregate_arrow(prism_ctx* ctx, const struct ArrowArray* batch,
                               const struct ArrowSchema* schema,
                               const prism_agg_config* config, struct ArrowArray* out,
                               struct ArrowSchema* out_schema);
/* prism_join_project_ex with a host probe batch and a host result (what
 * prism-jni would call per probe batch against a resident build table).
 * With unique Int64 build keys and fixed-width, null-free probe key and
 * gathered columns the probe streams through in chunks of 8M rows: chunk
 * i+1's upload, chunk i's probe and chunk i-1's download overlap on the
 * link's two directions; the output lands in page-locked host buffers.
 * Other inputs take one upload, the probe, one download. Results equal
 * prism_join_project_ex's for the same flags. */
int prism_join_project_arrow(prism_ctx* ctx, const prism_hash_table* table,
                             const struct ArrowArray* probe, const struct ArrowSchema* probe_schema,
                             const int32_t* probe_keys, int32_t n_keys, const int32_t* out_cols,
                             int32_t n_out, uint32_t flags, struct ArrowArray* out,
                             struct ArrowSchema* out_schema);
int prism_sort_batch_arrow(prism_ctx* ctx, const struct ArrowArray* batch, const struct ArrowSchema* schema,
                           const prism_sort_key* keys, int32_t n_keys, int64_t limit, struct ArrowArray* out,
                           struct ArrowSchema* out_schema);
int prism_filter_and_project_arrow(prism_ctx* ctx, const struct ArrowArray* batch,
                                   const struct ArrowSchema* schema,
                                   const prism_predicate* predicate, const int32_t* cols,
                                   int32_t n_cols, struct ArrowArray* out,
                                   struct ArrowSchema* out_schema);

#ifdef __cplusplus
}
#endif

#endif /* PRISM_GPU_H */
