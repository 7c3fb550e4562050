// prims.hpp — device-wide primitives shared by the operators.
#pragma once

#include "runtime.hpp"

namespace prism {

// Exclusive scan of n u32 values into u64 offsets; returns the total
// (synchronises the stream to read it).
uint64_t scan_u32(Ctx& ctx, const uint32_t* in, uint64_t* out, int64_t n);
// Same without a host round trip: the total is written to *total_dev.
void scan_u32_async(Ctx& ctx, const uint32_t* in, uint64_t* out, int64_t n, uint64_t* total_dev);

// Ordered positions of the set bits (or unset bits, invert = true) of an
// n-bit bitmap; *count receives their number.
MemP compact_bits(Ctx& ctx, const uint8_t* bitmap, int64_t n, bool invert, int64_t* count);

// Stable sort of (key, val) u32 pairs by the low `bits` bits of key.
void stable_sort_pairs_u32(Ctx& ctx, uint32_t* keys, uint32_t* vals, int64_t n, int bits);

// Gather: out[i] = col[idx[i]]; idx_valid (bitmap, may be null) marks null
// indices whose outputs are null. Validity is always materialised when the
// source has one or idx_valid is given.
ColP take(Ctx& ctx, const Column& col, const uint32_t* idx, const uint8_t* idx_valid, int64_t n,
          const std::string& name, bool nullable);

// Filter: keep rows whose bit is set in keep (bitmap over col.length rows).
ColP filter_column(Ctx& ctx, const Column& col, const uint32_t* kept_rows, int64_t n_kept);

// Bitmap of n bits from a per-row byte predicate (nonzero = set).
void pack_bits(Ctx& ctx, const uint8_t* bytes, int64_t n, uint8_t* bitmap);

// Marks bitmap bits idx[i] (bitmap pre-zeroed by the caller).
void scatter_bits(Ctx& ctx, const uint32_t* idx, int64_t n, uint8_t* bitmap);

// Device column that repeats a null-free fixed-width value (index arrays).
ColP u32_column(Ctx& ctx, const std::string& name, MemP mem, uint32_t* ptr, int64_t n);

// The parts of one column (same type; Utf8, dictionary indices, fixed width,
// validity) concatenated into a new column (agg.cu).
ColP concat_columns(Ctx& ctx, const std::vector<const Column*>& parts);

}  // namespace prism
