// tuning.hpp — the per-shape tuning table and the autotuner that fills it.
//
// The reference has one compile-time knob on this path (HASH_PARTITIONS =
// 64, native/prism-executor/src/hash_join.rs:43). Here the join table's
// layout (dense rows or hash slots, load factor), the radix-partitioned build
// and probe (on/off, fan-out), the fused join -> aggregate kernel's shape
// and the hashed-groups kernel's block size are chosen per shape: the
// autotuner times candidate settings on the caller's own data with CUDA
// events and records the fastest per shape class; every later call of that
// class reads it. The table can be saved to and loaded from a text file
// (PRISM_TUNING_FILE is loaded at first use). Settings given through the
// environment (PRISM_JOIN_DENSE, PRISM_JOIN_PARTITION, PRISM_JOIN_AGG_SHAPE,
// PRISM_HASH_AGG_BLOCK) take precedence over the table.
#pragma once

#include <string>

#include "agg.hpp"
#include "join.hpp"

namespace prism {

// Shape class of a join: key kind (single Int64 or general) and the build
// side's row count bucket (log2); probes are tuned with their build side.
struct JoinShape {
  int key_kind = 0;  // 0 single Int64 key, 1 general keys
  int build_log2 = 0;
};
JoinShape join_shape(const Batch& build, const std::vector<int>& keys);

// Overlays the recorded choice for `shape` on `t` (fields the environment
// set stay); returns whether a record existed.
bool apply_join_tuning(const JoinShape& shape, JoinTuning& t);
bool apply_join_agg_tuning(const JoinShape& shape, AggTuning& t);
bool apply_agg_tuning(int64_t rows, AggTuning& t);

void record_join_tuning(const JoinShape& shape, const JoinTuning& t);
void record_join_agg_tuning(const JoinShape& shape, const AggTuning& t);
void record_agg_tuning(int64_t rows, const AggTuning& t);

void tuning_clear();
void tuning_save(const std::string& path);
void tuning_load(const std::string& path);
std::string tuning_dump();  // the table in its file format

}  // namespace prism
