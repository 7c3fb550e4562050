// common.cuh — shared device types and helpers of the B200 engine.
#pragma once

#ifdef __CUDACC_RTC__
// compiled by NVRTC for per-query kernels: no system headers (LP64 types)
typedef signed char int8_t;
typedef short int16_t;
typedef int int32_t;
typedef long int64_t;
typedef unsigned char uint8_t;
typedef unsigned short uint16_t;
typedef unsigned int uint32_t;
typedef unsigned long uint64_t;
typedef unsigned long uintptr_t;
#else
#include <cuda_runtime.h>
#include <stdint.h>
#endif

namespace prism {

// Physical column types (Arrow formats handled by the engine).
enum Ty : int32_t {
  TY_NULL = 0, TY_BOOL, TY_I8, TY_I16, TY_I32, TY_I64, TY_U8, TY_U16, TY_U32, TY_U64,
  TY_F32, TY_F64, TY_DATE32, TY_UTF8, TY_DEC128, TY_DICT
};

__host__ __device__ inline int width_of(int t) {
  switch (t) {
    case TY_I8: case TY_U8: return 1;
    case TY_I16: case TY_U16: return 2;
    case TY_I32: case TY_U32: case TY_F32: case TY_DATE32: return 4;
    case TY_I64: case TY_U64: case TY_F64: return 8;
    case TY_DEC128: return 16;
    default: return 0;
  }
}

// Device view of one column. Bitmaps always start at bit 0 (the importer
// realigns offsets); `values` points at element 0; for UTF8,
// data + offsets[i] .. data + offsets[i+1] is row i (offsets may not start
// at zero). TY_DICT: values holds indices of index_type; dict_* describe the
// Utf8 (or integer) dictionary.
struct DCol {
  int32_t type;
  int32_t index_type;
  int64_t length;
  const uint8_t* validity;  // nullptr: all valid
  const void* values;
  const int32_t* offsets;
  const uint8_t* data;
  const int32_t* dict_offsets;
  const uint8_t* dict_data;
  int64_t dict_length;
  int32_t scale;
  int32_t dict_type;
};

__device__ __forceinline__ bool dcol_valid(const DCol& c, int64_t i) {
  return c.validity == nullptr || ((c.validity[i >> 3] >> (i & 7)) & 1);
}

// Raw integer value (ints, date, bool, dictionary index).
__device__ __forceinline__ int64_t dcol_ival(const DCol& c, int64_t i) {
  int t = c.type == TY_DICT ? c.index_type : c.type;
  switch (t) {
    case TY_BOOL: return (static_cast<const uint8_t*>(c.values)[i >> 3] >> (i & 7)) & 1;
    case TY_I8: return static_cast<const int8_t*>(c.values)[i];
    case TY_I16: return static_cast<const int16_t*>(c.values)[i];
    case TY_I32: case TY_DATE32: return static_cast<const int32_t*>(c.values)[i];
    case TY_I64: return static_cast<const int64_t*>(c.values)[i];
    case TY_U8: return static_cast<const uint8_t*>(c.values)[i];
    case TY_U16: return static_cast<const uint16_t*>(c.values)[i];
    case TY_U32: return static_cast<const uint32_t*>(c.values)[i];
    case TY_U64: return (int64_t) static_cast<const uint64_t*>(c.values)[i];
    default: return 0;
  }
}

// arrow cast-to-Float64 of the raw slot value.
__device__ __forceinline__ double dcol_fval(const DCol& c, int64_t i) {
  switch (c.type) {
    case TY_F64: return static_cast<const double*>(c.values)[i];
    case TY_F32: return (double) static_cast<const float*>(c.values)[i];
    case TY_U64: return (double) static_cast<const uint64_t*>(c.values)[i];
    case TY_DEC128: {
      const int64_t* p = static_cast<const int64_t*>(c.values) + 2 * i;
      __int128 v = ((__int128)p[1] << 64) | (unsigned __int128)(uint64_t)p[0];
      double s = 1.0;
      for (int k = 0; k < c.scale; ++k) s *= 10.0;
      return (double)v / s;
    }
    default: return (double)dcol_ival(c, i);
  }
}

__device__ __forceinline__ __int128 dcol_i128(const DCol& c, int64_t i) {
  if (c.type == TY_DEC128) {
    const int64_t* p = static_cast<const int64_t*>(c.values) + 2 * i;
    return ((__int128)p[1] << 64) | (unsigned __int128)(uint64_t)p[0];
  }
  if (c.type == TY_U64) return (__int128)(uint64_t)dcol_ival(c, i);
  return (__int128)dcol_ival(c, i);
}

// Value of row i as arrow's cast hands it to arithmetic and aggregation:
// the cast of an integer, Float32 or Boolean column (arrow-rs numeric_cast /
// unary_opt) writes 0 into the slots of null rows, while a Float64 column
// (no cast) and the Decimal128 -> Float64 cast (unary) keep the raw slot.
__device__ __forceinline__ bool keeps_null_slot(const DCol& c) { return c.type == TY_F64 || c.type == TY_DEC128; }
__device__ __forceinline__ double dcol_fval_cast(const DCol& c, int64_t i) {
  return (keeps_null_slot(c) || dcol_valid(c, i)) ? dcol_fval(c, i) : 0.0;
}
__device__ __forceinline__ int64_t dcol_ival_cast(const DCol& c, int64_t i) {
  return (keeps_null_slot(c) || dcol_valid(c, i)) ? dcol_ival(c, i) : 0;
}
__device__ __forceinline__ __int128 dcol_i128_cast(const DCol& c, int64_t i) {
  return (keeps_null_slot(c) || dcol_valid(c, i)) ? dcol_i128(c, i) : (__int128)0;
}

// UTF8 (or dictionary-decoded) bytes of row i.
__device__ __forceinline__ void dcol_str(const DCol& c, int64_t i, const uint8_t*& p, int32_t& n) {
  if (c.type == TY_DICT) {
    int64_t k = dcol_ival(c, i);
    if (k < 0 || k >= c.dict_length) { p = nullptr; n = 0; return; }
    int32_t a = c.dict_offsets[k], b = c.dict_offsets[k + 1];
    p = c.dict_data + a;
    n = b - a;
    return;
  }
  int32_t a = c.offsets[i], b = c.offsets[i + 1];
  p = c.data + a;
  n = b - a;
}

// ---------------------------------------------------------------- hashing --
constexpr uint64_t FX_K = 0x517cc1b727220a95ULL;
// Tag word of the engine's identity encoding for key types the reference
// hashes through their Debug text (fallback types).
constexpr uint64_t FALLBACK_TAG = 0x9E3779B97F4A7C15ULL;

__device__ __forceinline__ uint64_t fx_word(uint64_t s, uint64_t w) { return s * FX_K + w; }

// FxHasher::write over bytes (8-byte little-endian chunks, last one padded),
// then write_u8(0xff): Rust's `impl Hash for str` into FxHasher.
// Bytes [0, len) of q as a little-endian word, zero above len (1 <= len <= 8).
// Reads only the aligned 8-byte words that hold at least one of those bytes
// (so never a page without a byte of the string): one or two loads instead of
// len byte loads.
__device__ __forceinline__ uint64_t str_word(const uint8_t* q, int32_t len) {
  const uintptr_t a = reinterpret_cast<uintptr_t>(q) & 7;
  const uint64_t* w = reinterpret_cast<const uint64_t*>(q - a);
  uint64_t x = w[0] >> (8 * a);
  if ((int32_t)(8 - a) < len) x |= w[1] << (64 - 8 * a);
  return len >= 8 ? x : (x & ((1ULL << (8 * len)) - 1));
}

__device__ __forceinline__ uint64_t fx_str(uint64_t s, const uint8_t* p, int32_t n) {
  int32_t i = 0;
  for (; i + 8 <= n; i += 8) s = fx_word(s, str_word(p + i, 8));
  if (i < n) s = fx_word(s, str_word(p + i, n - i));
  return fx_word(s, 0xff);
}

// One key column's contribution to the group-identity FxHash
// (hash_array_value, native/prism-executor/src/hash_aggregate.rs:492-504).
__device__ __forceinline__ uint64_t fx_value(uint64_t s, const DCol& c, int64_t row) {
  if (!dcol_valid(c, row)) return fx_word(s, 0);
  switch (c.type) {
    case TY_I32: case TY_I64: return fx_word(s, (uint64_t)dcol_ival(c, row));
    case TY_F64: {
      double d = static_cast<const double*>(c.values)[row];
      return fx_word(s, (uint64_t)__double_as_longlong(d));
    }
    case TY_UTF8: case TY_DICT: {
      const uint8_t* p;
      int32_t n;
      dcol_str(c, row, p, n);
      return fx_str(s, p, n);
    }
    case TY_DEC128: {
      const uint64_t* p = static_cast<const uint64_t*>(c.values) + 2 * row;
      s = fx_word(s, FALLBACK_TAG ^ (uint64_t)c.type);
      s = fx_word(s, p[0]);
      return fx_word(s, p[1]);
    }
    case TY_F32: {
      float f = static_cast<const float*>(c.values)[row];
      s = fx_word(s, FALLBACK_TAG ^ (uint64_t)c.type);
      return fx_word(s, (uint64_t)(uint32_t)__float_as_uint(f));
    }
    default:
      s = fx_word(s, FALLBACK_TAG ^ (uint64_t)c.type);
      return fx_word(s, (uint64_t)dcol_ival(c, row));
  }
}

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t x) {
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdULL;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ULL;
  x ^= x >> 33;
  return x;
}

// Total-order key of a double (IEEE 754 totalOrder), as arrow-ord compares
// floats; also the order used by MIN/MAX accumulators.
__device__ __forceinline__ int64_t total_key(double d) {
  int64_t i = __double_as_longlong(d);
  return i ^ (int64_t)(((uint64_t)(i >> 63)) >> 1);
}
__device__ __forceinline__ double from_total_key(int64_t k) {
  int64_t i = k ^ (int64_t)(((uint64_t)(k >> 63)) >> 1);
  return __longlong_as_double(i);
}

// 128-bit compare-and-swap (sm_90+ atom.cas.b128) on global memory;
// returns the old low word, old high word in old_hi.
__device__ __forceinline__ unsigned long long cas128(unsigned long long* p, unsigned long long cmp_lo,
                                                     unsigned long long cmp_hi, unsigned long long new_lo,
                                                     unsigned long long new_hi, unsigned long long& old_hi) {
  unsigned long long old_lo;
  asm volatile(
      "{\n\t.reg .b128 d, c, n;\n\t"
      "mov.b128 c, {%3, %4};\n\t"
      "mov.b128 n, {%5, %6};\n\t"
      "atom.global.cas.b128 d, [%2], c, n;\n\t"
      "mov.b128 {%0, %1}, d;\n\t}"
      : "=l"(old_lo), "=l"(old_hi)
      : "l"(p), "l"(cmp_lo), "l"(cmp_hi), "l"(new_lo), "l"(new_hi)
      : "memory");
  return old_lo;
}

// Bounded spin limit for every wait on another CTA.
constexpr uint32_t SPIN_LIMIT = 1u << 22;

// Device-side error flags written by kernels (host reads after the call).
enum DevErr : uint32_t {
  DERR_NONE = 0,
  DERR_TABLE_FULL = 1,
  DERR_TIMEOUT = 2,
  DERR_OVERFLOW = 4,
  DERR_RANGE = 8,
  DERR_CAPACITY = 16,
  DERR_CORRUPT = 32,  // malformed encoded input (Parquet pages, Snappy streams), an inconsistent join table
};

#ifndef __CUDACC_RTC__
inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
#endif

}  // namespace prism
