// join_device.cuh — device-side lookup of the hash join table, shared by
// the probe kernels (join.cu) and the fused join -> aggregate kernels
// generated at run time (agg_device.cuh, compiled with NVRTC).
//
// Key identity follows hash_join.rs: a single Int64 key is matched by its raw
// value (validity ignored); any other key list by a 64-bit row hash over the
// key columns (a null contributes a marker word, as the reference hashes 0u8
// for it, hash_join.rs:394-398) followed by keys_equal
// (hash_join.rs:628-670): null flags agree and raw values are equal, Float64
// by `==` and equal bits.
#pragma once

#include "common.cuh"

namespace prism {

constexpr uint64_t JOIN_EMPTY = 0x8000000000000000ULL;  // empty slot (an Int64 key equal to it takes the side slot)
// per-row match word of the split join -> aggregate: a verified build row,
// JOIN_NO_MATCH, or this bit | the slot of several build rows
constexpr uint32_t JOIN_MATCH_SLOT = 0x80000000u;
constexpr uint64_t JOIN_FIB = 0x9E3779B97F4A7C15ULL;
constexpr uint32_t JOIN_NO_MATCH = 0xFFFFFFFFu;

__device__ __forceinline__ uint64_t join_slot_of(uint64_t k, int shift) { return (k * JOIN_FIB) >> shift; }

// Row hash over the key columns; equal keys hash equal across the two sides
// (types are checked on the host).
__device__ __forceinline__ uint64_t join_key_hash(const DCol* cols, int n, int64_t row) {
  uint64_t h = 0x2545F4914F6CDD1DULL;
  for (int i = 0; i < n; ++i) {
    const DCol& c = cols[i];
    uint64_t w;
    if (!dcol_valid(c, row)) w = 0x6a09e667f3bcc909ULL;
    else if (c.type == TY_UTF8 || c.type == TY_DICT) {
      const uint8_t* p;
      int32_t len;
      dcol_str(c, row, p, len);
      w = fx_str(0, p, len);
    } else if (c.type == TY_F64) w = (uint64_t)__double_as_longlong(static_cast<const double*>(c.values)[row]);
    else if (c.type == TY_F32) w = (uint64_t)__float_as_uint(static_cast<const float*>(c.values)[row]);
    else if (c.type == TY_DEC128) {
      const uint64_t* p = static_cast<const uint64_t*>(c.values) + 2 * row;
      w = p[0] ^ mix64(p[1]);
    } else w = (uint64_t)dcol_ival(c, row);
    h = mix64(h ^ w) + JOIN_FIB;
  }
  return h == JOIN_EMPTY ? JOIN_EMPTY + 1 : h;  // the empty marker stays free
}

__device__ __forceinline__ bool join_bytes_equal(const uint8_t* a, int32_t na, const uint8_t* b, int32_t nb) {
  if (na != nb) return false;
  for (int32_t i = 0; i < na; i += 8) {
    int32_t len = na - i < 8 ? na - i : 8;
    if (str_word(a + i, len) != str_word(b + i, len)) return false;
  }
  return true;
}

__device__ __forceinline__ bool join_rows_equal(const DCol* pc, const DCol* bc, int n, int64_t pr, int64_t br) {
  for (int i = 0; i < n; ++i) {
    const DCol& a = pc[i];
    const DCol& b = bc[i];
    if (dcol_valid(a, pr) != dcol_valid(b, br)) return false;
    switch (a.type) {
      case TY_UTF8: case TY_DICT: {
        const uint8_t *x, *y;
        int32_t nx, ny;
        dcol_str(a, pr, x, nx);
        dcol_str(b, br, y, ny);
        if (!join_bytes_equal(x, nx, y, ny)) return false;
        break;
      }
      case TY_F64: {
        double x = static_cast<const double*>(a.values)[pr], y = static_cast<const double*>(b.values)[br];
        if (!(x == y) || __double_as_longlong(x) != __double_as_longlong(y)) return false;
        break;
      }
      case TY_F32: {
        float x = static_cast<const float*>(a.values)[pr], y = static_cast<const float*>(b.values)[br];
        if (!(x == y) || __float_as_uint(x) != __float_as_uint(y)) return false;
        break;
      }
      case TY_DEC128: {
        const uint64_t* x = static_cast<const uint64_t*>(a.values) + 2 * pr;
        const uint64_t* y = static_cast<const uint64_t*>(b.values) + 2 * br;
        if (x[0] != y[0] || x[1] != y[1]) return false;
        break;
      }
      case TY_NULL: break;
      default:
        if (dcol_ival(a, pr) != dcol_ival(b, br)) return false;
    }
  }
  return true;
}

// Packed build keys of a single Utf8 key column: one 64-byte record per
// build row, word 0 = the key's byte length, bit 63 set for a null key, and
// words 1..7 its raw bytes zero-padded (keys of at most 56 bytes; longer
// ones keep the column). A probe compares against one aligned record (its
// first 32 bytes unless the key is longer than 24 bytes) instead of the
// build offsets and then the bytes they point to: one dependent load less.
// The comparison is keys_equal's (hash_join.rs:628-670): null flags agree
// and the raw bytes are equal.
constexpr uint64_t JOIN_KREC_NULL = 1ULL << 63;
constexpr int JOIN_KREC_MAX = 56;

__device__ __forceinline__ bool join_rec_equal(const DCol& pc, int64_t pr, const ulonglong2* __restrict__ rec,
                                               uint32_t row) {
  const ulonglong2* r = rec + (size_t)row * 4;
  const ulonglong2 h0 = __ldg(r), h1 = __ldg(r + 1);
  const uint8_t* p;
  int32_t n;
  dcol_str(pc, pr, p, n);
  const uint64_t want = (uint64_t)(uint32_t)n | (dcol_valid(pc, pr) ? 0ULL : JOIN_KREC_NULL);
  if (want != h0.x) return false;
  uint64_t w[7] = {h0.y, h1.x, h1.y, 0, 0, 0, 0};
  if (n > 24) {
    const ulonglong2 h2 = __ldg(r + 2), h3 = __ldg(r + 3);
    w[3] = h2.x;
    w[4] = h2.y;
    w[5] = h3.x;
    w[6] = h3.y;
  }
#pragma unroll
  for (int k = 0; k < 7; ++k) {
    const int32_t i = 8 * k;
    if (i < n && str_word(p + i, n - i < 8 ? n - i : 8) != w[k]) return false;
  }
  return true;
}

// Slot entries of a single Utf8 key (the fused join -> aggregate's table):
// one 64-byte entry per hash slot, in slot order, so a probe row's lookup
// is one aligned 64-byte read whose address follows from the row hash alone:
//   e[0] = {row hash (JOIN_EMPTY: free slot), the slot word cnt << 32 | row}
//   e[1] = {key length | bit 63 null | bit 62 longer than JOIN_ENT_BYTES, key bytes 0..7}
//   e[2] = {key bytes 8..15, 16..23}
//   e[3] = {key bytes 24..31, the raw value of one fixed-width build column at row}
// Bytes past the key's length are zero. A slot with several build rows
// (cnt > 1) keeps only the slot words; its rows are compared against the
// column.
constexpr uint64_t JOIN_ENT_LONG = 1ULL << 62;
constexpr int JOIN_ENT_BYTES = 32;

// A probe key of a Utf8 column as the entries hold it: the length word
// (bit 63: null) and the first JOIN_ENT_BYTES bytes as little-endian words,
// zero above the length. The bytes come from independent aligned 8-byte
// loads of only the words that hold a byte of the key.
struct JoinKeyWords {
  uint64_t len;  // length | JOIN_KREC_NULL
  uint64_t w[4];
};

// false (k unset) for a key longer than JOIN_ENT_BYTES
__device__ __forceinline__ bool join_key_words(const DCol& c, int64_t i, JoinKeyWords& k) {
  const int32_t a = c.offsets[i], n = c.offsets[i + 1] - a;
  if (n < 0 || n > JOIN_ENT_BYTES) return false;
  const uint8_t* p = c.data + a;
  const uint32_t al = (uint32_t)(reinterpret_cast<uintptr_t>(p) & 7);
  const uint64_t* q = reinterpret_cast<const uint64_t*>(p - al);
  const int32_t nw = (int32_t)(al + n + 7) >> 3;  // at most 5
  uint64_t x[5];
#pragma unroll
  for (int j = 0; j < 5; ++j) x[j] = j < nw ? q[j] : 0ULL;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const uint64_t v = al ? (x[j] >> (8 * al)) | (x[j + 1] << (64 - 8 * al)) : x[j];
    const int32_t rem = n - 8 * j;
    k.w[j] = rem >= 8 ? v : rem > 0 ? v & ((1ULL << (8 * rem)) - 1) : 0ULL;
  }
  k.len = (uint64_t)(uint32_t)n | (dcol_valid(c, i) ? 0ULL : JOIN_KREC_NULL);
  return true;
}

// join_key_hash of a single Utf8 key from its words (fx_str over the
// zero-padded words is fx_str over the bytes)
__device__ __forceinline__ uint64_t join_words_hash(const JoinKeyWords& k) {
  const int32_t n = (int32_t)(uint32_t)k.len;
  uint64_t w;
  if (k.len & JOIN_KREC_NULL) {
    w = 0x6a09e667f3bcc909ULL;
  } else {
    uint64_t s = 0;
#pragma unroll
    for (int j = 0; j < 4; ++j)
      if (8 * j < n) s = fx_word(s, k.w[j]);
    w = fx_word(s, 0xff);
  }
  const uint64_t h = mix64(0x2545F4914F6CDD1DULL ^ w) + JOIN_FIB;
  return h == JOIN_EMPTY ? JOIN_EMPTY + 1 : h;
}

// keys_equal of a probe key's words against build row `row`'s packed key
// record (words 0..4: length, key bytes 0..31, zero past the length)
__device__ __forceinline__ bool join_words_rec_equal(const JoinKeyWords& k, const ulonglong2* __restrict__ rec,
                                                     uint32_t row) {
  const ulonglong2* r = rec + (size_t)row * 4;
  const ulonglong2 r0 = __ldg(r), r1 = __ldg(r + 1);
  if (r0.x != k.len || r0.y != k.w[0] || r1.x != k.w[1] || r1.y != k.w[2]) return false;
  return (uint32_t)k.len <= 24 || __ldg(r + 2).x == k.w[3];
}

// keys_equal of a probe key's words against an entry with cnt == 1 and no
// JOIN_ENT_LONG flag (both sides zero-padded)
__device__ __forceinline__ bool join_words_equal(const JoinKeyWords& k, const ulonglong2& e1, const ulonglong2& e2,
                                                 const ulonglong2& e3) {
  return k.len == e1.x && k.w[0] == e1.y && k.w[1] == e2.x && k.w[2] == e2.y && k.w[3] == e3.x;
}

}  // namespace prism
