// join.hpp — device hash table and probe of the hash join
// (native/prism-executor/src/hash_join.rs).
#pragma once

#include "runtime.hpp"

namespace prism {

struct JoinTable {
  Ctx* ctx = nullptr;
  Batch build;               // shares the build batch's device columns
  std::vector<int> key_cols;
  bool int64_fast = false;   // single Int64 key: keyed by raw value, validity ignored
  int log2cap = 0;
  uint64_t capacity = 0;     // power of two (+1 side slot at [capacity])
  MemP slots;                // ulonglong2 per slot: x = key (or row hash), y = cnt << 32 | row
  // dense mode (single Int64 key, unique keys spanning a range at most about
  // twice the row count): dense_rows[key - dmin] = build row, or NO_MATCH;
  // no hash slots are built
  bool dense = false;
  int64_t dmin = 0;
  uint64_t drange = 0;
  MemP dense_rows;
  // dense mode: {row, value} pairs in key order for one fixed 8-byte build
  // column (dense_pair_src), so a probe gathering it reads one 16-byte entry
  MemP dense_pairs;
  const void* dense_pair_src = nullptr;
  bool has_dups = false;     // some slot holds more than one build row
  MemP dup_rows;             // build rows grouped by slot, ascending inside a slot
  int64_t n_dup_rows = 0;
  std::vector<DCol> key_views;
  MemP key_views_dev;
  // packed build keys (single Utf8 key of at most JOIN_KREC_MAX bytes per
  // row): 64-byte records per build row, see join_device.cuh
  MemP key_records;
  // slot entries (single Utf8 key, see join_device.cuh): 64 bytes per slot
  // with the slot words, the key and the raw value of build column
  // entry_col (-1: none) for the fused join -> aggregate
  MemP key_entries;
  int entry_col = -1;
};

struct JoinTuning {
  // target slot load; 0: automatic (0.5, or up to 0.7 when that halves a
  // table larger than L2: fewer of its slot lines miss L2)
  double load_factor = 0;
  int probe_blocks_per_sm = 2;
  bool dense = true;  // allow dense mode for single Int64 keys
  bool dense_pairs = false;  // dense mode: {row, value} pairs for one 8-byte build column
  // radix-partitioned build / probe of hash slots (single Int64 key): -1 once
  // the slots outgrow L2, 0 never, 1 always; 2^partition_bits partitions
  int partition = -1;
  int partition_bits = 8;
  bool key_records = true;  // packed build keys for a single Utf8 key column
  // slot entries instead of row records for the fused join -> aggregate
  // (single Utf8 key); measured: the same kernel time as the records and a
  // dearer build (one random key read per slot), so off unless asked for
  bool key_entries = false;
  // fields the environment set (the tuning table leaves them alone)
  enum : uint32_t { FIX_DENSE = 1, FIX_PARTITION = 2, FIX_LOAD = 4 };
  uint32_t fixed = 0;
};

std::unique_ptr<JoinTable> build_join_table(Ctx& ctx, const Batch& build, const std::vector<int>& keys,
                                            const JoinTuning& tune);

// Packs the slot entries of a hash table over a single Utf8 key, with the
// raw values of build column inline_col (fixed width 4 or 8, no nulls; -1:
// none). Returns false (and builds nothing) for any other table.
bool build_key_entries(Ctx& ctx, JoinTable& t, int inline_col);

// The first half of the split join -> aggregate (hash table over a single
// Utf8 key with packed key records or slot entries, Utf8 probe key): per
// probe row of `pkey` (n rows) the verified build row, JOIN_NO_MATCH, or
// JOIN_MATCH_SLOT | slot for a slot of several build rows, into out_match;
// and the raw value of build column inline_col (fixed width 4 or 8, no
// nulls; -1: none) at the matched row into out_inl. Returns false (nothing
// launched) for any other table.
bool match_rows_utf8(Ctx& ctx, const JoinTable& t, const Column& pkey, int64_t n, int inline_col, uint32_t* out_match,
                     void* out_inl);

// Output spec of a probe: which index arrays to emit and which fixed-width
// null-free columns to gather inside the probe kernel.
struct ProbeGather {
  int side;          // 0 probe, 1 build
  const void* src;   // column values
  int width;         // 4 or 8
  void* dst;         // output values (capacity rows)
};

struct ProbeResult {
  int64_t matches = 0;
  MemP probe_idx, build_idx;  // u32 arrays (may be empty if not requested)
};

// Probes `probe` (key columns `keys`, types checked against the table) and
// emits matches in the reference's order: probe rows ascending, build rows
// ascending within a probe row. With `any_order` the matches come as a
// multiset (in no particular order), which needs neither look-back nor a
// second pass.
// `row_base` is added to the emitted probe row indices (the probe batch is
// rows [row_base, row_base + probe.rows) of a larger one). Fused gathers write into caller buffers of
// `gather_capacity` rows (must be >= the match count; use probe_count first).
ProbeResult probe_join_table(Ctx& ctx, const JoinTable& t, const Batch& probe, const std::vector<int>& keys,
                             bool want_probe_idx, bool want_build_idx, std::vector<ProbeGather>& gathers,
                             int64_t gather_capacity, const JoinTuning& tune, bool any_order = false,
                             int64_t row_base = 0);

// Number of matches of `probe` against the table (no output).
int64_t probe_count(Ctx& ctx, const JoinTable& t, const Batch& probe, const std::vector<int>& keys,
                    const JoinTuning& tune);

// Upper bound on the match count usable without a counting pass (-1 if none).
int64_t match_upper_bound(const JoinTable& t, int64_t probe_rows);

void check_join_keys(const Batch& probe, const std::vector<int>& pk, const Batch& build, const std::vector<int>& bk);

}  // namespace prism

// The opaque resident-table handle of the C ABI.
struct prism_hash_table {
  prism_ctx* ctx = nullptr;
  std::unique_ptr<prism::JoinTable> t;
};
