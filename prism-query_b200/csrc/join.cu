// join.cu — open-addressing device hash table, build and ordered probe.
//
// Replaces HashTable::build / HashTable::probe
// (native/prism-executor/src/hash_join.rs:87-200). The reference partitions
// `(hash, row)` pairs 64 ways and builds one hashbrown map of row lists per
// partition; here one linear-probing table in HBM holds 16-byte slots
// {key, cnt << 32 | row} inserted with 64-bit atomicCAS, and rows of keys
// that occur more than once live in contiguous ascending segments.
//
// The probe is one pass over the probe keys: each CTA takes a tile of 2048
// rows, resolves its slots (4 independent 16-byte loads in flight per lane),
// ranks the matches with warp scans, obtains the tile's output offset by
// decoupled look-back over the preceding tiles, and writes matches in the
// reference's order (probe row ascending, build rows ascending) — no second
// read of the probe side and no post-sort.
#include "join.hpp"
#include "bulk.cuh"
#include "join_device.cuh"
#include "prims.hpp"
#include "sort.hpp"

namespace prism {

namespace {

constexpr uint64_t EMPTY = JOIN_EMPTY;
constexpr uint64_t Y_INIT = 0;  // cnt 0

constexpr int PW = 16;             // warps per probe CTA
constexpr int PI = 4;              // rows per lane
constexpr int PT = PW * 32 * PI;   // rows per tile (2048)

__device__ __forceinline__ uint64_t slot_of(uint64_t k, int shift) { return join_slot_of(k, shift); }

struct KeysFast {
  static constexpr bool kFast = true;
  const int64_t* k;
  __device__ __forceinline__ uint64_t key(int64_t r) const { return (uint64_t)__ldg(k + r); }
};
struct KeysGeneral {
  static constexpr bool kFast = false;
  const DCol* cols;
  int n;
  __device__ __forceinline__ uint64_t key(int64_t r) const { return join_key_hash(cols, n, r); }
};
// row hashes computed beforehand (the radix-partitioned build of general keys)
struct KeysHashed {
  static constexpr bool kFast = false;
  const uint64_t* h;
  __device__ __forceinline__ uint64_t key(int64_t r) const { return __ldg(h + r); }
};

__global__ void row_hash_kernel(const DCol* cols, int n, int64_t rows, uint64_t* __restrict__ h) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < rows; i += (int64_t)gridDim.x * blockDim.x)
    h[i] = join_key_hash(cols, n, i);
}

// The radix-partitioned build and probe (single Int64 key, hash slots): on
// when the tuning asks for it, or by default (partition < 0) once the slots
// outgrow L2 — then a stretch of tiles in partition order touches one
// 1/2^bits slice of the table, which stays in L2.
bool use_partitioned(const Ctx& ctx, const JoinTable& t, const JoinTuning& tune) {
  if (t.dense || t.capacity == 0) return false;
  if (tune.partition >= 0) return tune.partition > 0;
  return (t.capacity + 1) * sizeof(ulonglong2) > (uint64_t)ctx.l2_bytes;
}
int partition_bits(const JoinTable& t, const JoinTuning& tune) {
  const int b = tune.partition_bits > 0 ? tune.partition_bits : 8;
  return std::max(1, std::min(std::min(b, 8), t.log2cap));
}

__global__ void init_slots_kernel(ulonglong2* slots, uint64_t n) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    slots[i] = make_ulonglong2(EMPTY, Y_INIT);
}

// rowmap: the build row of element i (radix-partitioned build), or null (row i)
template <class K>
__global__ void insert_kernel(K keys, int64_t n, ulonglong2* slots, int shift, uint64_t mask, uint64_t cap,
                              uint32_t* dupflag, uint32_t* err, const uint32_t* __restrict__ rowmap) {
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    uint64_t k = keys.key(e);
    const int64_t i = rowmap ? (int64_t)rowmap[e] : e;
    uint64_t s;
    bool winner = false;
    if (K::kFast && k == EMPTY) {
      s = cap;  // side slot for the sentinel value
      winner = true;
    } else {
      // one 128-bit CAS claims an empty slot with {key, count 1 | row};
      // finding the key already there falls through to the count update
      s = slot_of(k, shift);
      uint64_t steps = 0;
      bool ok = false;
      while (steps <= mask) {
        unsigned long long old_y;
        unsigned long long prev = cas128((unsigned long long*)&slots[s], EMPTY, Y_INIT, k,
                                         (1ULL << 32) | (uint32_t)i, old_y);
        if (prev == EMPTY && old_y == Y_INIT) { ok = winner = true; break; }
        if (prev == k) { ok = true; break; }
        s = (s + 1) & mask;
        ++steps;
      }
      if (!ok) { atomicOr(err, DERR_TABLE_FULL); continue; }
      if (winner) continue;  // inserted with its count and row
    }
    // one atomic: count the row, and let the slot's first inserter record
    // its row (slots with several rows get sorted segments afterwards)
    unsigned long long add = (1ULL << 32) | (winner && !(K::kFast && k == EMPTY) ? (uint32_t)i : 0u);
    unsigned long long old = atomicAdd((unsigned long long*)&slots[s].y, add);
    if (K::kFast && k == EMPTY && (old >> 32) == 0) {
      // side slot: the first arrival stores its row (count already added)
      atomicOr((unsigned long long*)&slots[s].y, (unsigned long long)(uint32_t)i);
    }
    if ((old >> 32) >= 1) *dupflag = 1;
  }
}

// For each build row: its slot, and whether the slot holds several rows.
template <class K>
__global__ void locate_kernel(K keys, int64_t n, const ulonglong2* __restrict__ slots, int shift, uint64_t mask,
                              uint64_t cap, uint32_t* __restrict__ row_slot, uint8_t* __restrict__ is_dup) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t k = keys.key(i);
    uint64_t s;
    if (K::kFast && k == EMPTY) s = cap;
    else {
      s = slot_of(k, shift);
      uint64_t steps = 0;
      while (slots[s].x != k && steps <= mask) { s = (s + 1) & mask; ++steps; }
    }
    row_slot[i] = (uint32_t)s;
    is_dup[i] = (slots[s].y >> 32) > 1 ? 1 : 0;
  }
}

__global__ void gather_u32_kernel(const uint32_t* src, const uint32_t* idx, int64_t n, uint32_t* dst) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = src[idx[i]];
}

// One 64-byte record per build row of a single Utf8 key column (see
// join_device.cuh): length word (bit 63: null), then the raw bytes, zero
// padded; a key longer than JOIN_KREC_MAX bytes sets *too_long (the caller
// then drops the records).
__global__ void pack_key_records_kernel(DCol c, int64_t n, ulonglong2* __restrict__ rec, uint32_t* too_long) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint8_t* p;
    int32_t len;
    dcol_str(c, i, p, len);
    if (len > JOIN_KREC_MAX) {
      atomicOr(too_long, 1u);
      continue;
    }
    uint64_t w[8];
    w[0] = (uint64_t)(uint32_t)len | (dcol_valid(c, i) ? 0ULL : JOIN_KREC_NULL);
#pragma unroll
    for (int k = 0; k < 7; ++k) {
      const int32_t o = 8 * k;
      w[k + 1] = o < len ? str_word(p + o, len - o < 8 ? len - o : 8) : 0ULL;
    }
    ulonglong2* r = rec + (size_t)i * 4;
#pragma unroll
    for (int k = 0; k < 4; ++k) r[k] = make_ulonglong2(w[2 * k], w[2 * k + 1]);
  }
}

// The slot entries of a single Utf8 key column (layout in join_device.cuh),
// one thread per slot: the slot words, and for a slot of one build row its
// key (length, null flag, bytes) and the raw value of the inlined column
// (inl_width 4 or 8 bytes, 0: none).
__global__ void pack_key_entries_kernel(const ulonglong2* __restrict__ slots, uint64_t n_slots, DCol c,
                                        const void* __restrict__ inl, int inl_width, ulonglong2* __restrict__ ent) {
  for (uint64_t s = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; s < n_slots;
       s += (uint64_t)gridDim.x * blockDim.x) {
    const ulonglong2 sl = slots[s];
    uint64_t w[6] = {0, 0, 0, 0, 0, 0};
    if (sl.x != JOIN_EMPTY && (sl.y >> 32) == 1) {
      const uint32_t row = (uint32_t)sl.y;
      const uint8_t* p;
      int32_t len;
      dcol_str(c, row, p, len);
      w[0] = (uint64_t)(uint32_t)len | (dcol_valid(c, row) ? 0ULL : JOIN_KREC_NULL);
      if (len > JOIN_ENT_BYTES) {
        w[0] |= JOIN_ENT_LONG;
      } else {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int32_t o = 8 * k;
          w[k + 1] = o < len ? str_word(p + o, len - o < 8 ? len - o : 8) : 0ULL;
        }
      }
      if (inl_width == 8) w[5] = static_cast<const unsigned long long*>(inl)[row];
      else if (inl_width == 4) w[5] = static_cast<const uint32_t*>(inl)[row];
    }
    ulonglong2* e = ent + s * 4;
    e[0] = sl;
    e[1] = make_ulonglong2(w[0], w[1]);
    e[2] = make_ulonglong2(w[2], w[3]);
    e[3] = make_ulonglong2(w[4], w[5]);
  }
}

// Row hashes of M probe rows of a Utf8 column (idx[k] >= n: none), with the
// loads of all M rows in flight together: first every row's two offsets,
// then every row's key words (keys of at most JOIN_ENT_BYTES bytes), then
// the hashes. join_key_words per row would wait for each row's offsets
// before loading its words, one row after another.
template <int M>
__device__ __forceinline__ void hash_utf8_rows(const DCol& pk, const int64_t (&idx)[M], int64_t n, uint64_t (&h)[M]) {
  int32_t ka[M], kn[M];
#pragma unroll
  for (int k = 0; k < M; ++k) {
    ka[k] = 0;
    kn[k] = 0;
    if (idx[k] < n) {
      ka[k] = pk.offsets[idx[k]];
      kn[k] = pk.offsets[idx[k] + 1] - ka[k];
    }
  }
  uint64_t x[M][5];
#pragma unroll
  for (int k = 0; k < M; ++k) {
    const uint8_t* p = pk.data + ka[k];
    const uint32_t al = (uint32_t)(reinterpret_cast<uintptr_t>(p) & 7);
    const uint64_t* q = reinterpret_cast<const uint64_t*>(p - al);
    const int32_t nw = idx[k] < n && kn[k] >= 0 && kn[k] <= JOIN_ENT_BYTES ? (int32_t)(al + kn[k] + 7) >> 3 : 0;
#pragma unroll
    for (int j = 0; j < 5; ++j) x[k][j] = j < nw ? q[j] : 0ULL;
  }
#pragma unroll
  for (int k = 0; k < M; ++k) {
    h[k] = 0;
    if (idx[k] >= n) continue;
    if (kn[k] < 0 || kn[k] > JOIN_ENT_BYTES) {
      h[k] = join_key_hash(&pk, 1, idx[k]);  // a long key: the general hash
      continue;
    }
    const uint32_t al = (uint32_t)(reinterpret_cast<uintptr_t>(pk.data + ka[k]) & 7);
    JoinKeyWords kw;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const uint64_t v = al ? (x[k][j] >> (8 * al)) | (x[k][j + 1] << (64 - 8 * al)) : x[k][j];
      const int32_t rem = kn[k] - 8 * j;
      kw.w[j] = rem >= 8 ? v : rem > 0 ? v & ((1ULL << (8 * rem)) - 1) : 0ULL;
    }
    kw.len = (uint64_t)(uint32_t)kn[k] | (dcol_valid(pk, idx[k]) ? 0ULL : JOIN_KREC_NULL);
    h[k] = join_words_hash(kw);
  }
}

// ------------------------------------- per-row match of a Utf8 probe key --
// The first half of the split join -> aggregate over a single Utf8 key: one
// pass over a probe batch writes, per probe row, the build row whose key
// equals its key (verified), or JOIN_NO_MATCH, or JOIN_MATCH_SLOT | slot for
// a slot of several build rows (the aggregation compares those rows
// itself); and the raw value of one fixed-width build column at the matched
// row (IW bytes, 0 for none). Each thread keeps MR rows in flight through
// the whole lookup with only their hash and slot words live (the key words
// are read again for the verification, from L1 / L2), so an SM has 4,096
// lookups outstanding where the fused kernel's per-row state allows
// 1,024-2,048.
constexpr int MB = 256;  // threads per CTA
constexpr int MR = 4;    // rows per thread

// over the hash slots and the row records (packed key records)
template <int IW>
__global__ void __launch_bounds__(MB, 4) match_rows_kernel(DCol pk, int64_t n, const ulonglong2* __restrict__ slots,
                                                           int shift, uint64_t mask, const ulonglong2* __restrict__ rec,
                                                           const void* __restrict__ inl, uint32_t* __restrict__ out_match,
                                                           void* __restrict__ out_inl) {
  const int64_t base = (int64_t)blockIdx.x * (MB * MR) + threadIdx.x;
  uint64_t h[MR], s[MR];
  ulonglong2 e[MR];
  int64_t rows[MR];
#pragma unroll
  for (int k = 0; k < MR; ++k) rows[k] = base + k * MB;
  hash_utf8_rows<MR>(pk, rows, n, h);
#pragma unroll
  for (int k = 0; k < MR; ++k) {
    const int64_t idx = base + k * MB;
    s[k] = join_slot_of(h[k], shift);
    e[k] = idx < n ? __ldg(slots + s[k]) : make_ulonglong2(JOIN_EMPTY, 0);
  }
  uint32_t m[MR];
#pragma unroll
  for (int k = 0; k < MR; ++k) {
    const int64_t idx = base + k * MB;
    m[k] = JOIN_NO_MATCH;
    if (idx >= n) continue;
    for (uint64_t steps = 0; e[k].x != h[k] && e[k].x != JOIN_EMPTY && steps <= mask; ++steps) {
      s[k] = (s[k] + 1) & mask;
      e[k] = __ldg(slots + s[k]);
    }
    if (e[k].x != h[k]) continue;
    const uint32_t row = (uint32_t)e[k].y, cnt = (uint32_t)(e[k].y >> 32);
    if (cnt != 1) {
      m[k] = JOIN_MATCH_SLOT | (uint32_t)s[k];
      continue;
    }
    JoinKeyWords kw;
    bool eq;
    if (join_key_words(pk, idx, kw)) {
      // record words 0..4: length, key bytes 0..31 (zero past the length)
      const ulonglong2* r = rec + (size_t)row * 4;
      const ulonglong2 r0 = __ldg(r), r1 = __ldg(r + 1);
      eq = r0.x == kw.len && r0.y == kw.w[0] && r1.x == kw.w[1] && r1.y == kw.w[2];
      if (eq && (uint32_t)kw.len > 24) eq = __ldg(r + 2).x == kw.w[3];
    } else {
      eq = join_rec_equal(pk, idx, rec, row);
    }
    if (eq) m[k] = row;
  }
#pragma unroll
  for (int k = 0; k < MR; ++k) {
    const int64_t idx = base + k * MB;
    if (idx >= n) continue;
    __stcs(out_match + idx, m[k]);
    if (IW == 4)
      __stcs(static_cast<uint32_t*>(out_inl) + idx,
             m[k] < JOIN_MATCH_SLOT ? __ldg(static_cast<const uint32_t*>(inl) + m[k]) : 0u);
    if (IW == 8)
      __stcs(static_cast<unsigned long long*>(out_inl) + idx,
             m[k] < JOIN_MATCH_SLOT ? __ldg(static_cast<const unsigned long long*>(inl) + m[k]) : 0ULL);
  }
}

// over the 64-byte slot entries: one entry's first sector (row hash, slot
// word, length word, first key word) per row, the rest only for a row whose
// hash and length match; the inlined build value from the entry's last
// word. One random DRAM fetch per probe row instead of three (slot,
// record, column).
template <int IW>
__global__ void __launch_bounds__(MB, 4) match_entries_kernel(DCol pk, DCol bk, int64_t n,
                                                              const ulonglong2* __restrict__ ent, int shift,
                                                              uint64_t mask, uint32_t* __restrict__ out_match,
                                                              void* __restrict__ out_inl) {
  const int64_t base = (int64_t)blockIdx.x * (MB * MR) + threadIdx.x;
  uint64_t h[MR], s[MR];
  ulonglong2 e0[MR], e1[MR];
  int64_t rows[MR];
#pragma unroll
  for (int k = 0; k < MR; ++k) rows[k] = base + k * MB;
  hash_utf8_rows<MR>(pk, rows, n, h);
#pragma unroll
  for (int k = 0; k < MR; ++k) {
    const int64_t idx = base + k * MB;
    s[k] = join_slot_of(h[k], shift);
    e0[k] = make_ulonglong2(JOIN_EMPTY, 0);
    e1[k] = make_ulonglong2(0, 0);
    if (idx < n) {
      e0[k] = __ldg(ent + 4 * s[k]);
      e1[k] = __ldg(ent + 4 * s[k] + 1);
    }
  }
  uint32_t m[MR];
  unsigned long long v[MR];
#pragma unroll
  for (int k = 0; k < MR; ++k) {
    const int64_t idx = base + k * MB;
    m[k] = JOIN_NO_MATCH;
    v[k] = 0;
    if (idx >= n) continue;
    for (uint64_t steps = 0; e0[k].x != h[k] && e0[k].x != JOIN_EMPTY && steps <= mask; ++steps) {
      s[k] = (s[k] + 1) & mask;
      e0[k] = __ldg(ent + 4 * s[k]);
      e1[k] = __ldg(ent + 4 * s[k] + 1);
    }
    if (e0[k].x != h[k]) continue;
    const uint32_t row = (uint32_t)e0[k].y, cnt = (uint32_t)(e0[k].y >> 32);
    if (cnt != 1) {
      m[k] = JOIN_MATCH_SLOT | (uint32_t)s[k];
      continue;
    }
    JoinKeyWords kw;
    bool eq;
    if (e1[k].x & JOIN_ENT_LONG) {
      eq = join_rows_equal(&pk, &bk, 1, idx, row);  // a build key longer than the entry holds
      v[k] = __ldg(ent + 4 * s[k] + 3).y;
    } else if (join_key_words(pk, idx, kw) && kw.len == e1[k].x && kw.w[0] == e1[k].y) {
      const ulonglong2 e2 = __ldg(ent + 4 * s[k] + 2), e3 = __ldg(ent + 4 * s[k] + 3);
      eq = join_words_equal(kw, e1[k], e2, e3);
      v[k] = e3.y;
    } else {
      eq = false;  // a probe key longer than any entry's, or another length / first word
    }
    if (eq) m[k] = row;
  }
#pragma unroll
  for (int k = 0; k < MR; ++k) {
    const int64_t idx = base + k * MB;
    if (idx >= n) continue;
    __stcs(out_match + idx, m[k]);
    if (IW == 4) __stcs(static_cast<uint32_t*>(out_inl) + idx, m[k] < JOIN_MATCH_SLOT ? (uint32_t)v[k] : 0u);
    if (IW == 8) __stcs(static_cast<unsigned long long*>(out_inl) + idx, m[k] < JOIN_MATCH_SLOT ? v[k] : 0ULL);
  }
}

// sorted_slot[i] starts a segment -> slots[slot].row = i (cnt unchanged)
__global__ void segment_heads_kernel(const uint32_t* sorted_slot, int64_t n, ulonglong2* slots) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t s = sorted_slot[i];
    if (i == 0 || sorted_slot[i - 1] != s) {
      unsigned long long y = slots[s].y;
      slots[s].y = (y & 0xFFFFFFFF00000000ULL) | (uint32_t)i;
    }
  }
}

// ------------------------------------------------------------- the probe --
constexpr uint32_t NO_MATCH = JOIN_NO_MATCH;

struct ProbeArgs {
  int64_t n;
  const uint32_t* dense;  // dense mode (see JoinTable), else nullptr
  int64_t dmin;
  uint64_t drange;
  const ulonglong2* slots;
  int shift;
  uint64_t mask;
  uint64_t cap;
  const uint32_t* dup_rows;
  int64_t n_dup_rows;  // a slot's segment past it: the table is inconsistent (DERR_CORRUPT)
  const DCol* pcols;  // verify (general path)
  const DCol* bcols;
  int nkeys;
  uint32_t* out_probe;
  uint32_t* out_build;
  int ngather;
  int g_side[4];
  const void* g_src[4];
  int g_width[4];
  void* g_dst[4];
  uint64_t out_capacity;
  unsigned long long* tile_status;
  unsigned long long* tile_counter;
  int64_t n_tiles;
  unsigned long long* total;
  uint32_t* err;
  int any_order;  // tiles reserve their output by one atomicAdd on *total, no look-back
  int64_t prefetch_ahead;  // one-pass probe: tiles between a CTA and the tile it prefetches into L2 (0: none)
  int64_t row_base;  // added to every emitted probe row index (a chunk of a larger probe)
  const ulonglong2* krec;  // packed build keys (single Utf8 key), or null
  const ulonglong2* dpairs;  // dense mode: {row, value} of the one gathered column, or null
};

constexpr unsigned long long FLAG_A = 1ULL << 62;
constexpr unsigned long long FLAG_P = 2ULL << 62;
constexpr unsigned long long VAL_MASK = (1ULL << 62) - 1;

// Decoupled look-back (Merrill & Garland, "Single-pass Parallel Prefix Scan
// with Decoupled Look-back", 2016), run by one warp: publish this tile's
// aggregate, then inspect 32 predecessors per round trip, summing aggregates
// up to the nearest tile that already published its inclusive prefix. Tiles
// are handed out in increasing order, so every predecessor is running or
// done; the wait is still bounded and reports DERR_TIMEOUT.
__device__ unsigned long long warp_lookback(unsigned long long* status, int64_t tile, unsigned long long agg,
                                            uint32_t* err) {
  const int lane = threadIdx.x & 31;
  if (tile == 0) {
    if (lane == 0) atomicExch(&status[0], FLAG_P | agg);
    return 0;
  }
  if (lane == 0) atomicExch(&status[tile], FLAG_A | agg);
  unsigned long long excl = 0;
  int64_t t = tile - 1;
  uint32_t spins = 0;
  for (;;) {
    int64_t idx = t - lane;
    unsigned long long st = FLAG_P + 0ULL;
    if (idx >= 0) st = *(volatile unsigned long long*)&status[idx];
    unsigned long long f = st & ~VAL_MASK;
    uint32_t pmask = __ballot_sync(0xffffffffu, f == FLAG_P);
    uint32_t zmask = __ballot_sync(0xffffffffu, f == 0);
    int first_p = pmask ? __ffs(pmask) - 1 : 31;
    uint32_t need = (first_p == 31) ? 0xffffffffu : ((2u << first_p) - 1u);
    if (zmask & need) {
      if (++spins > SPIN_LIMIT) {
        if (lane == 0) atomicOr(err, DERR_TIMEOUT);
        break;
      }
      __nanosleep(32);
      continue;
    }
    unsigned long long v = lane <= first_p ? (st & VAL_MASK) : 0ULL;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    excl += v;
    if (pmask) break;
    t -= 32;
  }
  if (lane == 0) atomicExch(&status[tile], FLAG_P | (excl + agg));
  return excl;
}

__device__ __forceinline__ uint32_t warp_incl_scan32(uint32_t x) {
  int lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += y;
  }
  return x;
}

__device__ __forceinline__ void emit_one(const ProbeArgs& a, uint64_t pos, int64_t prow, uint32_t brow) {
  if (a.out_probe) a.out_probe[pos] = (uint32_t)(prow + a.row_base);
  if (a.out_build) a.out_build[pos] = brow;
#pragma unroll
  for (int g = 0; g < 4; ++g) {
    if (g >= a.ngather) break;
    int64_t src = a.g_side[g] ? (int64_t)brow : prow;
    if (a.g_width[g] == 8)
      static_cast<uint64_t*>(a.g_dst[g])[pos] = __ldg(static_cast<const unsigned long long*>(a.g_src[g]) + src);
    else
      static_cast<uint32_t*>(a.g_dst[g])[pos] = __ldg(static_cast<const unsigned int*>(a.g_src[g]) + src);
  }
}

// One CTA = PW warps; a tile = PT consecutive probe rows; warp w owns rows
// [tile*PT + w*32*PI, +32*PI) in PI lane-strided groups (coalesced loads,
// row order = item-major, lane-minor).
template <class K, bool DUPS, bool VERIFY, bool EMIT>
__global__ void __launch_bounds__(PW * 32, 2) probe_kernel(K keys, ProbeArgs a) {
  __shared__ uint32_t s_wexcl[PW];
  __shared__ unsigned long long s_excl;
  __shared__ int64_t s_tile;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (;;) {
    if (threadIdx.x == 0) s_tile = (int64_t)atomicAdd(a.tile_counter, 1ULL);
    __syncthreads();
    const int64_t tile = s_tile;
    if (tile >= a.n_tiles) break;
    const int64_t base = tile * PT + warp * (32 * PI);

    uint32_t c[PI], v[PI], cand[PI];
    if (K::kFast && a.dense != nullptr) {
      // dense mode: one direct lookup per row
#pragma unroll
      for (int it = 0; it < PI; ++it) {
        int64_t r = base + it * 32 + lane;
        c[it] = v[it] = cand[it] = 0;
        if (r < a.n) {
          uint64_t d = keys.key(r) - (uint64_t)a.dmin;
          uint32_t row = d < a.drange ? __ldg(a.dense + d) : NO_MATCH;
          if (row != NO_MATCH) {
            v[it] = row;
            cand[it] = 1;
            c[it] = 1;
          }
        }
      }
    } else {
      uint64_t key[PI];
      uint64_t s[PI];
      ulonglong2 e[PI];
#pragma unroll
      for (int it = 0; it < PI; ++it) {
        int64_t r = base + it * 32 + lane;
        key[it] = r < a.n ? keys.key(r) : EMPTY;
      }
#pragma unroll
      for (int it = 0; it < PI; ++it) {
        int64_t r = base + it * 32 + lane;
        if (r < a.n) {
          s[it] = (K::kFast && key[it] == EMPTY) ? a.cap : slot_of(key[it], a.shift);
          e[it] = __ldg(a.slots + s[it]);
        } else {
          e[it] = make_ulonglong2(EMPTY, 0);
        }
      }
#pragma unroll
      for (int it = 0; it < PI; ++it) {
        int64_t r = base + it * 32 + lane;
        c[it] = 0;
        v[it] = 0;
        cand[it] = 0;
        if (r >= a.n) continue;
        uint64_t steps = 0;
        while (e[it].x != key[it] && e[it].x != EMPTY && steps <= a.mask) {
          s[it] = (s[it] + 1) & a.mask;
          e[it] = __ldg(a.slots + s[it]);
          ++steps;
        }
        uint32_t cnt = (uint32_t)(e[it].y >> 32);
        if (e[it].x != key[it] || cnt == 0) continue;
        if (cnt > 1 && (int64_t)(uint32_t)e[it].y + cnt > a.n_dup_rows) {
          atomicOr(a.err, DERR_CORRUPT);
          continue;
        }
        v[it] = (uint32_t)e[it].y;
        cand[it] = cnt;
        if (!VERIFY) {
          c[it] = DUPS ? cnt : 1u;
        } else if (cnt == 1) {
          c[it] = (a.krec ? join_rec_equal(a.pcols[0], r, a.krec, v[it]) : join_rows_equal(a.pcols, a.bcols, a.nkeys, r, v[it]))
                      ? 1u : 0u;
        } else {
          uint32_t m = 0;
          for (uint32_t j = 0; j < cnt; ++j) {
            const uint32_t b = a.dup_rows[v[it] + j];
            m += (a.krec ? join_rec_equal(a.pcols[0], r, a.krec, b) : join_rows_equal(a.pcols, a.bcols, a.nkeys, r, b)) ? 1u : 0u;
          }
          c[it] = m;
        }
      }
    }
    // rank matches inside the warp (row order = item-major, lane-minor)
    uint32_t lex[PI];
    uint32_t run = 0;
#pragma unroll
    for (int it = 0; it < PI; ++it) {
      uint32_t incl = warp_incl_scan32(c[it]);
      lex[it] = run + incl - c[it];
      run += __shfl_sync(0xffffffffu, incl, 31);
    }
    if (lane == 0) s_wexcl[warp] = run;
    __syncthreads();
    if (warp == 0) {
      uint32_t wv = lane < PW ? s_wexcl[lane] : 0;
      uint32_t incl = warp_incl_scan32(wv);
      uint32_t tile_total = __shfl_sync(0xffffffffu, incl, 31);
      if (lane < PW) s_wexcl[lane] = incl - wv;
      if (EMIT && a.any_order) {
        if (lane == 0) s_excl = tile_total ? atomicAdd(a.total, (unsigned long long)tile_total) : 0ULL;
      } else if (EMIT) {
        unsigned long long ex = warp_lookback(a.tile_status, tile, tile_total, a.err);
        if (lane == 0) {
          s_excl = ex;
          if (tile == a.n_tiles - 1) *a.total = ex + tile_total;
        }
      } else if (lane == 0) {
        if (tile_total) atomicAdd(a.total, (unsigned long long)tile_total);
        s_excl = 0;
      }
    }
    __syncthreads();
    if (EMIT) {
      const uint64_t wbase = s_excl + s_wexcl[warp];
#pragma unroll
      for (int it = 0; it < PI; ++it) {
        if (!c[it]) continue;
        int64_t r = base + it * 32 + lane;
        uint64_t pos = wbase + lex[it];
        // a short output keeps the prefix of the matches that fits
        if (pos + c[it] > a.out_capacity) atomicOr(a.err, DERR_CAPACITY);
        if (pos >= a.out_capacity) continue;
        if ((!DUPS && !VERIFY) || cand[it] == 1) {
          emit_one(a, pos, r, v[it]);
        } else {
          for (uint32_t j = 0; j < cand[it] && pos < a.out_capacity; ++j) {
            uint32_t b = a.dup_rows[v[it] + j];
            if (VERIFY && !(a.krec ? join_rec_equal(a.pcols[0], r, a.krec, b)
                                   : join_rows_equal(a.pcols, a.bcols, a.nkeys, r, b)))
              continue;
            emit_one(a, pos++, r, b);
          }
        }
      }
    }
    __syncthreads();
  }
}

// ---------------------------------------------------- unique int64 keys ----
// Two sync-free kernels for the common case (single Int64 key, unique build
// keys): the probe writes one u32 per probe row (matched build row, or
// NO_MATCH) and one match count per tile; after an exclusive scan of the tile
// counts the emit kernel streams those words back and writes the matches at
// their final positions. Neither kernel waits on another CTA, so the random
// slot loads of many tiles overlap freely.
constexpr int QB = 256;            // threads per CTA
constexpr int QI = 8;              // rows per thread
constexpr int QT = QB * QI;        // rows per tile (2048)

__global__ void __launch_bounds__(QB, 3) probe_rows_kernel(const int64_t* __restrict__ keys, int64_t n,
                                                          const ulonglong2* __restrict__ slots, int shift,
                                                          uint64_t mask, uint64_t cap, uint32_t* __restrict__ rowv,
                                                          uint32_t* __restrict__ tile_cnt) {
  const int64_t base = (int64_t)blockIdx.x * QT;
  uint64_t key[QI], s[QI];
  ulonglong2 e[QI];
#pragma unroll
  for (int it = 0; it < QI; ++it) {
    int64_t r = base + it * QB + threadIdx.x;
    key[it] = r < n ? (uint64_t)__ldg(keys + r) : EMPTY;
  }
#pragma unroll
  for (int it = 0; it < QI; ++it) {
    int64_t r = base + it * QB + threadIdx.x;
    if (r < n) {
      s[it] = key[it] == EMPTY ? cap : slot_of(key[it], shift);
      e[it] = __ldg(slots + s[it]);
    }
  }
  uint32_t cnt = 0;
#pragma unroll
  for (int it = 0; it < QI; ++it) {
    int64_t r = base + it * QB + threadIdx.x;
    if (r >= n) continue;
    uint64_t steps = 0;
    while (e[it].x != key[it] && e[it].x != EMPTY && steps <= mask) {
      s[it] = (s[it] + 1) & mask;
      e[it] = __ldg(slots + s[it]);
      ++steps;
    }
    bool hit = e[it].x == key[it] && (e[it].y >> 32) != 0;
    rowv[r] = hit ? (uint32_t)e[it].y : NO_MATCH;
    cnt += hit ? 1u : 0u;
  }
  // CTA total
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, d);
  __shared__ uint32_t wsum[QB / 32];
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = cnt;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
#pragma unroll
    for (int w = 0; w < QB / 32; ++w) t += wsum[w];
    tile_cnt[blockIdx.x] = t;
  }
}

// dense-mode twin of probe_rows_kernel: row = dense[key - dmin]
__global__ void __launch_bounds__(QB, 4) probe_rows_dense_kernel(const int64_t* __restrict__ keys, int64_t n,
                                                                const uint32_t* __restrict__ dense, int64_t dmin,
                                                                uint64_t drange, uint32_t* __restrict__ rowv,
                                                                uint32_t* __restrict__ tile_cnt) {
  const int64_t base = (int64_t)blockIdx.x * QT;
  uint64_t d[QI];
#pragma unroll
  for (int it = 0; it < QI; ++it) {
    int64_t r = base + it * QB + threadIdx.x;
    // the key and row-word streams are touched once: evict-first loads and
    // stores, so they do not push the dense table out of L2
    d[it] = r < n ? (uint64_t)__ldcs(keys + r) - (uint64_t)dmin : ~0ULL;
  }
  uint32_t cnt = 0;
#pragma unroll
  for (int it = 0; it < QI; ++it) {
    int64_t r = base + it * QB + threadIdx.x;
    uint32_t row = d[it] < drange ? __ldg(dense + d[it]) : NO_MATCH;
    if (r < n) __stcs(rowv + r, row);
    cnt += (r < n && row != NO_MATCH) ? 1u : 0u;
  }
#pragma unroll
  for (int k = 16; k > 0; k >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, k);
  __shared__ uint32_t wsum[QB / 32];
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = cnt;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint32_t t = 0;
#pragma unroll
    for (int w = 0; w < QB / 32; ++w) t += wsum[w];
    tile_cnt[blockIdx.x] = t;
  }
}

// min / max of the build keys (dense-mode test)
// min / max of the build keys into mm[0], mm[1]: 16-byte loads when the
// keys are 16-byte aligned, a warp then block reduction, one atomic pair
// per block (blockDim.x a multiple of 32, at most 1024)
__global__ void minmax_i64_kernel(const int64_t* __restrict__ keys, int64_t n, long long* mm) {
  __shared__ long long s_lo[32], s_hi[32];
  long long lo = 0x7fffffffffffffffLL, hi = (long long)0x8000000000000000ULL;
  const int64_t tid = blockIdx.x * (int64_t)blockDim.x + threadIdx.x, nt = (int64_t)gridDim.x * blockDim.x;
  int64_t head = n;  // rows read as pairs: [0, head)
  if ((reinterpret_cast<uintptr_t>(keys) & 15) == 0) {
    head = n & ~(int64_t)1;
    const longlong2* k2 = reinterpret_cast<const longlong2*>(keys);
    for (int64_t i = tid; i < head / 2; i += nt) {
      const longlong2 k = __ldg(k2 + i);  // kept in L2 for the insert that follows
      lo = min(lo, min(k.x, k.y));
      hi = max(hi, max(k.x, k.y));
    }
  } else {
    head = 0;
  }
  for (int64_t i = head + tid; i < n; i += nt) {
    const long long k = __ldg(keys + i);
    lo = min(lo, k);
    hi = max(hi, k);
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, d));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, d));
  }
  const int warp = threadIdx.x >> 5, nw = (int)(blockDim.x >> 5);
  if ((threadIdx.x & 31) == 0) {
    s_lo[warp] = lo;
    s_hi[warp] = hi;
  }
  __syncthreads();
  if (warp == 0) {
    lo = threadIdx.x < nw ? s_lo[threadIdx.x] : 0x7fffffffffffffffLL;
    hi = threadIdx.x < nw ? s_hi[threadIdx.x] : (long long)0x8000000000000000ULL;
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
      lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, d));
      hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, d));
    }
    if (threadIdx.x == 0) {
      atomicMin(mm, lo);
      atomicMax(mm + 1, hi);
    }
  }
}

__global__ void fill_u32_kernel(uint32_t* p, uint64_t n, uint32_t v) {
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    p[i] = v;
}

// min / max accumulators and the dense insert's flag word, before the keys
__global__ void dense_scalars_init_kernel(long long* mm) {
  mm[0] = 0x7fffffffffffffffLL;
  mm[1] = (long long)0x8000000000000000ULL;
  mm[2] = 0;
}

// The key range the min / max kernel found, or ~0 when it is cap or wider.
__device__ __forceinline__ uint64_t dense_range(const long long* mm, uint64_t cap) {
  const uint64_t diff = (uint64_t)mm[1] - (uint64_t)mm[0];  // max >= min: the build has rows
  return diff < cap ? diff + 1 : ~0ULL;
}

// NO_MATCH over the first `range` entries (nothing when the range is too wide)
__global__ void fill_dense_kernel(uint32_t* dense, uint64_t cap, const long long* mm) {
  const uint64_t r = dense_range(mm, cap);
  if (r == ~0ULL) return;
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < r; i += (uint64_t)gridDim.x * blockDim.x)
    dense[i] = NO_MATCH;
}

// dense insert: dense[key - min] = row; a second row for a key sets flag 1,
// a range of cap or more sets flag 2 (no insert)
__global__ void dense_insert_kernel(const int64_t* __restrict__ keys, int64_t n, const long long* mm, uint64_t cap,
                                    uint32_t* dense, uint32_t* flag) {
  const uint64_t r = dense_range(mm, cap);
  if (r == ~0ULL) {
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(flag, 2u);
    return;
  }
  const uint64_t dmin = (uint64_t)mm[0];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t d = (uint64_t)__ldg(keys + i) - dmin;
    if (atomicCAS(dense + d, NO_MATCH, (uint32_t)i) != NO_MATCH) atomicOr(flag, 1u);
  }
}

// dense pairs: pairs[d] = {dense[d], the paired column's value at that row}
// in key order (sequential, coalesced writes; the column read where a row
// exists), four entries a grid stride apart per thread and step so their
// column reads are in flight together
__global__ void dense_pairs_kernel(const uint32_t* __restrict__ dense, uint64_t r,
                                   const unsigned long long* __restrict__ col, ulonglong2* __restrict__ pairs) {
  const uint64_t nt = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t d0 = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; d0 < r; d0 += 4 * nt) {
    uint32_t rw[4];
    unsigned long long v[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) rw[k] = d0 + k * nt < r ? __ldcs(dense + d0 + k * nt) : NO_MATCH;
#pragma unroll
    for (int k = 0; k < 4; ++k) v[k] = rw[k] != NO_MATCH ? __ldg(col + rw[k]) : 0ULL;
#pragma unroll
    for (int k = 0; k < 4; ++k)
      if (d0 + k * nt < r) __stcs(pairs + d0 + k * nt, make_ulonglong2(rw[k], v[k]));
  }
}

__global__ void __launch_bounds__(QB) emit_rows_kernel(const uint32_t* __restrict__ rowv, int64_t n,
                                                       const uint64_t* __restrict__ tile_off, ProbeArgs a) {
  __shared__ uint32_t seg[QI][QB / 32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t base = (int64_t)blockIdx.x * QT;
  uint32_t v[QI], lpos[QI];
#pragma unroll
  for (int it = 0; it < QI; ++it) {
    int64_t r = base + it * QB + threadIdx.x;
    v[it] = r < n ? __ldcs(rowv + r) : NO_MATCH;
    uint32_t m = __ballot_sync(0xffffffffu, v[it] != NO_MATCH);
    lpos[it] = __popc(m & ((1u << lane) - 1u));
    if (lane == 0) seg[it][warp] = __popc(m);
  }
  // one 8-byte gathered column (the probe-row + payload output): every
  // matched row's value is loaded here, all QI in flight, before the scan
  // and any store (the stores could alias the source, so the compiler would
  // not move these loads above them)
  const bool one8 = a.ngather == 1 && a.g_width[0] == 8;
  unsigned long long pre[QI];
  if (one8) {
    const unsigned long long* src = static_cast<const unsigned long long*>(a.g_src[0]);
    const bool bside = a.g_side[0] != 0;
#pragma unroll
    for (int it = 0; it < QI; ++it) {
      int64_t r = base + it * QB + threadIdx.x;
      pre[it] = v[it] != NO_MATCH ? __ldg(src + (bside ? (int64_t)v[it] : r)) : 0ULL;
    }
  }
  __syncthreads();
  // exclusive offsets of the (item, warp) segments in row order
  if (warp == 0) {
    uint32_t x0 = seg[lane >> 3][lane & 7], x1 = seg[(lane + 32) >> 3][(lane + 32) & 7];
    uint32_t s0 = warp_incl_scan32(x0);
    uint32_t tot0 = __shfl_sync(0xffffffffu, s0, 31);
    uint32_t s1 = warp_incl_scan32(x1) + tot0;
    seg[lane >> 3][lane & 7] = s0 - x0;
    seg[(lane + 32) >> 3][(lane + 32) & 7] = s1 - x1;
  }
  __syncthreads();
  const uint64_t off = tile_off[blockIdx.x];
#pragma unroll
  for (int it = 0; it < QI; ++it) {
    if (v[it] == NO_MATCH) continue;
    uint64_t pos = off + seg[it][warp] + lpos[it];
    if (pos >= a.out_capacity) {
      atomicOr(a.err, DERR_CAPACITY);
      continue;
    }
    if (one8) {  // output streams: evict-first stores
      if (a.out_probe) __stcs(a.out_probe + pos, (uint32_t)(a.row_base + base + it * QB + threadIdx.x));
      if (a.out_build) __stcs(a.out_build + pos, v[it]);
      __stcs(static_cast<unsigned long long*>(a.g_dst[0]) + pos, pre[it]);
    } else {
      emit_one(a, pos, base + it * QB + threadIdx.x, v[it]);
    }
  }
}

// ------------------------------------------ unique int64 keys, any order --
// One pass when the caller takes the matches as a multiset (the fused
// join -> aggregate and join_project with PRISM_JOIN_ANY_ORDER): each CTA
// loads its 2048 probe keys with 16-byte vector loads, looks them up (dense
// row or hash slot walk), loads every matched row's gathered values, ranks
// its matches with warp ballots and two warp scans (ordered so that each
// store instruction of a warp covers one contiguous run), reserves its
// output segment with ONE atomicAdd and writes the segment. No
// row words go back to HBM and no CTA waits on another; segments land in
// whatever order the CTAs reserve them.
constexpr int AB = 256;            // threads per CTA
constexpr int AV = 4;              // 16-byte key loads per thread (2 rows each)
constexpr int AT = AB * AV * 2;    // rows per tile (2048)
// resident CTAs per SM the register budget is cut for: 5 for the dense
// lookup (48 registers, no spills), 4 for the slot walk (64 registers;
// at 48 it spills)
constexpr int any_ctas(bool dense) { return dense ? 5 : 4; }

// PART: the keys come in radix-partition order (kpart, with each key's probe
// row in prow): a tile's keys share their top hash bits, so its slot loads
// stay inside one slice of the table (the partitioned probe of a table
// larger than L2).
template <bool DENSE, bool VEC, bool PART>
__global__ void __launch_bounds__(AB, any_ctas(DENSE)) probe_emit_any_kernel(const int64_t* __restrict__ keys,
                                                                const uint32_t* __restrict__ prow, int64_t n,
                                                                ProbeArgs a) {
  __shared__ uint32_t seg[2 * AV * (AB / 32)];
  __shared__ unsigned long long s_off;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t base = (int64_t)blockIdx.x * AT;
  if (VEC && a.prefetch_ahead > 0 && threadIdx.x == 0) {
    // the keys (and rows) of the tile one resident wave ahead, into L2
    const int64_t pb = base + a.prefetch_ahead * AT;
    if (pb < n) {
      const int64_t r = (n - pb < AT ? n - pb : AT) & ~(int64_t)3;
      if (r) {
        bulk_prefetch_l2(keys + pb, (uint32_t)(r * 8));
        if (PART) bulk_prefetch_l2(prow + pb, (uint32_t)(r * 4));
      }
    }
  }
  // positions of this thread: base + 2 * (it * AB + threadIdx.x) + {0, 1}
  uint64_t key[AV][2];
  int64_t row[AV][2];  // probe row of each position
#pragma unroll
  for (int it = 0; it < AV; ++it) {
    const int64_t q = base + 2 * (it * AB + threadIdx.x);
    if (VEC && q + 1 < n) {
      // streamed once: evict-first, so the table and payload stay in L2
      const longlong2 kv = __ldcs(reinterpret_cast<const longlong2*>(keys + q));
      key[it][0] = (uint64_t)kv.x;
      key[it][1] = (uint64_t)kv.y;
      if (PART) {
        const uint2 rv = __ldcs(reinterpret_cast<const uint2*>(prow + q));
        row[it][0] = rv.x;
        row[it][1] = rv.y;
      }
    } else {
      key[it][0] = q < n ? (uint64_t)__ldcs(keys + q) : 0;
      key[it][1] = q + 1 < n ? (uint64_t)__ldcs(keys + q + 1) : 0;
      if (PART) {
        row[it][0] = q < n ? __ldcs(prow + q) : 0;
        row[it][1] = q + 1 < n ? __ldcs(prow + q + 1) : 0;
      }
    }
    if (!PART) {
      row[it][0] = q;
      row[it][1] = q + 1;
    }
  }
  uint32_t brow[AV][2];
  unsigned long long pre[AV][2];
  if (DENSE) {
    // with {row, value} pairs the gathered value comes in the same read
    const ulonglong2* dp = a.dpairs;
#pragma unroll
    for (int it = 0; it < AV; ++it)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int64_t q = base + 2 * (it * AB + threadIdx.x) + j;
        const uint64_t d = key[it][j] - (uint64_t)a.dmin;
        const bool in = q < n && d < a.drange;
        if (dp) {
          const ulonglong2 e = in ? __ldg(dp + d) : make_ulonglong2(NO_MATCH, 0);
          brow[it][j] = (uint32_t)e.x;
          pre[it][j] = e.y;
        } else {
          brow[it][j] = in ? __ldg(a.dense + d) : NO_MATCH;
        }
      }
  } else {
    uint64_t s[AV][2];
    ulonglong2 e[AV][2];
#pragma unroll
    for (int it = 0; it < AV; ++it)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int64_t q = base + 2 * (it * AB + threadIdx.x) + j;
        s[it][j] = key[it][j] == EMPTY ? a.cap : slot_of(key[it][j], a.shift);
        e[it][j] = q < n ? __ldg(a.slots + s[it][j]) : make_ulonglong2(EMPTY, 0);
      }
#pragma unroll
    for (int it = 0; it < AV; ++it)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int64_t q = base + 2 * (it * AB + threadIdx.x) + j;
        uint64_t steps = 0;
        while (e[it][j].x != key[it][j] && e[it][j].x != EMPTY && steps <= a.mask) {
          s[it][j] = (s[it][j] + 1) & a.mask;
          e[it][j] = __ldg(a.slots + s[it][j]);
          ++steps;
        }
        const bool hit = q < n && e[it][j].x == key[it][j] && (e[it][j].y >> 32) != 0;
        brow[it][j] = hit ? (uint32_t)e[it][j].y : NO_MATCH;
      }
  }
  // one 8-byte gathered column (probe row + payload): its values loaded now,
  // all in flight before the ranking
  const bool one8 = a.ngather == 1 && a.g_width[0] == 8;
  if (one8 && !(DENSE && a.dpairs)) {
    const unsigned long long* src = static_cast<const unsigned long long*>(a.g_src[0]);
    const bool bside = a.g_side[0] != 0;
#pragma unroll
    for (int it = 0; it < AV; ++it)
#pragma unroll
      for (int j = 0; j < 2; ++j)
        pre[it][j] = brow[it][j] != NO_MATCH ? __ldg(src + (bside ? (int64_t)brow[it][j] : row[it][j])) : 0ULL;
  }
  // rank as (it, j, warp, lane): the matches of one (it, j) of a warp take
  // consecutive positions, so each store instruction covers one contiguous
  // run (whole sectors) instead of every other position
  uint32_t lpos[AV][2];
  const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
  for (int it = 0; it < AV; ++it)
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const uint32_t m = __ballot_sync(0xffffffffu, brow[it][j] != NO_MATCH);
      lpos[it][j] = __popc(m & lt);
      if (lane == 0) seg[(it * 2 + j) * (AB / 32) + warp] = __popc(m);
    }
  __syncthreads();
  if (warp == 0) {  // 2 * AV * 8 = 64 segments: two scans of one warp
    const uint32_t x0 = seg[lane], x1 = seg[32 + lane];
    const uint32_t i0 = warp_incl_scan32(x0);
    const uint32_t t0 = __shfl_sync(0xffffffffu, i0, 31);
    const uint32_t i1 = warp_incl_scan32(x1) + t0;
    seg[lane] = i0 - x0;
    seg[32 + lane] = i1 - x1;
    const uint32_t total = __shfl_sync(0xffffffffu, i1, 31);
    if (lane == 0) s_off = total ? atomicAdd(a.total, (unsigned long long)total) : 0ULL;
  }
  __syncthreads();
  const unsigned long long off = s_off;
#pragma unroll
  for (int it = 0; it < AV; ++it)
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      if (brow[it][j] == NO_MATCH) continue;
      const uint64_t pos = off + seg[(it * 2 + j) * (AB / 32) + warp] + lpos[it][j];
      const int64_t r = row[it][j];
      if (pos >= a.out_capacity) {
        atomicOr(a.err, DERR_CAPACITY);
        continue;
      }
      if (one8) {
        if (a.out_probe) __stcs(a.out_probe + pos, (uint32_t)(a.row_base + r));
        if (a.out_build) __stcs(a.out_build + pos, brow[it][j]);
        __stcs(static_cast<unsigned long long*>(a.g_dst[0]) + pos, pre[it][j]);
      } else {
        emit_one(a, pos, r, brow[it][j]);
      }
    }
}

// PRISM_PROBE_GRAPH=1: the one-pass probe replayed from its instantiated
// graph instead of launched call by call (measured: 47.8 vs 44.8 us per
// 8K-row probe of a resident table, 61.0 vs 63.9 us at 1M rows: the
// argument update and graph launch cost what the three calls did, so off)
bool probe_graphs_on() {
  const char* e = std::getenv("PRISM_PROBE_GRAPH");
  return e && std::strcmp(e, "1") == 0;
}

// The one-pass probe's steady shape as a graph (memset of the match counter
// -> kernel fn -> one 16-byte copy of the error word and the counter into the
// context's page-locked mirror), built and instantiated on the first call of
// each kernel variant on the context; later calls set the kernel node's
// arguments and grid and launch the instantiated graph: one launch instead
// of three calls.
void launch_probe_graph(Ctx& ctx, const void* fn, unsigned grid, void** args) {
  cudaKernelNodeParams kp{};
  kp.func = const_cast<void*>(fn);
  kp.gridDim = dim3(grid);
  kp.blockDim = dim3(AB);
  kp.sharedMemBytes = 0;
  kp.kernelParams = args;
  auto it = ctx.probe_graphs.find(fn);
  if (it == ctx.probe_graphs.end()) {
    Ctx::ProbeGraph g;
    PRISM_CUDA(cudaGraphCreate(&g.graph, 0));
    cudaMemsetParams mp{};
    mp.dst = reinterpret_cast<char*>(ctx.d_err) + 8;
    mp.value = 0;
    mp.elementSize = 4;
    mp.width = 2;
    mp.height = 1;
    cudaGraphNode_t ms = nullptr, cp = nullptr;
    PRISM_CUDA(cudaGraphAddMemsetNode(&ms, g.graph, nullptr, 0, &mp));
    PRISM_CUDA(cudaGraphAddKernelNode(&g.kernel, g.graph, &ms, 1, &kp));
    PRISM_CUDA(cudaGraphAddMemcpyNode1D(&cp, g.graph, &g.kernel, 1, ctx.h_err, ctx.d_err, 16, cudaMemcpyDeviceToHost));
    cudaError_t e = cudaGraphInstantiate(&g.exec, g.graph, 0);
    if (e != cudaSuccess) {
      cudaGraphDestroy(g.graph);
      PRISM_CUDA(e);
    }
    it = ctx.probe_graphs.emplace(fn, g).first;
  } else {
    PRISM_CUDA(cudaGraphExecKernelNodeSetParams(it->second.exec, it->second.kernel, &kp));
  }
  PRISM_CUDA(cudaGraphLaunch(it->second.exec, ctx.stream));
  ctx.note_launch();
}

// PRISM_PROBE_PREFETCH=0 turns the one-pass probe's L2 prefetch off
int64_t any_prefetch_ahead(const Ctx& ctx, bool dense) {
  const char* e = std::getenv("PRISM_PROBE_PREFETCH");
  if (e && std::strcmp(e, "0") == 0) return 0;
  return (int64_t)ctx.sm_count * any_ctas(dense);  // the resident CTAs: one wave ahead
}

template <class K, bool EMIT>
void launch_probe(Ctx& ctx, const JoinTable& t, K keys, ProbeArgs& a, int blocks_per_sm) {
  int grid = (int)std::min<int64_t>(a.n_tiles, (int64_t)ctx.sm_count * std::min(blocks_per_sm, 2));
  if (grid < 1) grid = 1;
  bool verify = !t.int64_fast;
  KernelTimer kt(ctx, EMIT ? "probe_kernel" : "probe_count_kernel");
  if (!t.has_dups && !verify)
    probe_kernel<K, false, false, EMIT><<<grid, PW * 32, 0, ctx.stream>>>(keys, a);
  else if (!verify)
    probe_kernel<K, true, false, EMIT><<<grid, PW * 32, 0, ctx.stream>>>(keys, a);
  else
    probe_kernel<K, true, true, EMIT><<<grid, PW * 32, 0, ctx.stream>>>(keys, a);
  ctx.check_launch("probe_kernel");
}

}  // namespace

void check_join_keys(const Batch& probe, const std::vector<int>& pk, const Batch& build, const std::vector<int>& bk) {
  if (pk.empty() || pk.size() != bk.size())
    fail(PRISM_ERR_INVALID_ARGUMENT, "probe and build key lists must be non-empty and of equal length");
  for (size_t i = 0; i < pk.size(); ++i) {
    if (pk[i] < 0 || pk[i] >= (int)probe.cols.size()) fail(PRISM_ERR_INVALID_ARGUMENT, "probe key column out of range");
    if (bk[i] < 0 || bk[i] >= (int)build.cols.size()) fail(PRISM_ERR_INVALID_ARGUMENT, "build key column out of range");
    int a = probe.cols[pk[i]]->type, b = build.cols[bk[i]]->type;
    bool sa = a == TY_UTF8 || a == TY_DICT, sb = b == TY_UTF8 || b == TY_DICT;
    if (a != b && !(sa && sb))
      fail(PRISM_ERR_SCHEMA_MISMATCH, "join key types differ between probe and build (column " +
                                          std::to_string(pk[i]) + " vs " + std::to_string(bk[i]) + ")");
  }
}

std::unique_ptr<JoinTable> build_join_table(Ctx& ctx, const Batch& build, const std::vector<int>& keys,
                                            const JoinTuning& tune) {
  auto t = std::make_unique<JoinTable>();
  t->ctx = &ctx;
  t->build = build;
  t->key_cols = keys;
  for (int k : keys)
    if (k < 0 || k >= (int)build.cols.size()) fail(PRISM_ERR_INVALID_ARGUMENT, "build key column out of range");
  if (keys.empty()) fail(PRISM_ERR_INVALID_ARGUMENT, "no join keys");
  int64_t n = build.rows;
  if (n >= (int64_t)UINT32_MAX) fail(PRISM_ERR_INVALID_ARGUMENT, "build side exceeds 2^32-1 rows");
  t->int64_fast = keys.size() == 1 && build.cols[keys[0]]->type == TY_I64;
  for (int k : keys) t->key_views.push_back(build.cols[k]->view());
  t->key_views_dev = ctx.alloc(t->key_views.size() * sizeof(DCol));
  ctx.h2d_staged(t->key_views_dev->ptr, t->key_views.data(), t->key_views.size() * sizeof(DCol));
  if (t->int64_fast && n > 0 && tune.dense) {
    // dense mode when the keys span a range of at most twice the rows (plus
    // 4096) and are unique: a direct row index per key value replaces the
    // hash slots (4 bytes per value of the range instead of 16 per slot at
    // load factor 0.5, and one dependent load per probe)
    const int64_t* bk = static_cast<const int64_t*>(build.cols[keys[0]]->values);
    // one host synchronisation: the array is sized for the widest range the
    // dense mode takes; the fill and the inserts read the range the min / max
    // kernel left on the device, and give up (flag 2) when it is wider
    const uint64_t dcap = (uint64_t)std::min<int64_t>(2 * n + 4096, (int64_t)1 << 28);
    // {min, max, flag word}: set by one tiny kernel, read back by one copy
    MemP mmm;
    long long* mm = ctx.alloc_t<long long>(3, mmm);
    uint32_t* df = reinterpret_cast<uint32_t*>(mm + 2);
    dense_scalars_init_kernel<<<1, 1, 0, ctx.stream>>>(mm);
    ctx.check_launch("dense_scalars_init_kernel");
    minmax_i64_kernel<<<grid_for(ctx, n, 256, 8), 256, 0, ctx.stream>>>(bk, n, mm);
    ctx.check_launch("minmax_i64_kernel");
    MemP dense = ctx.alloc(dcap * 4);
    uint32_t* dr = static_cast<uint32_t*>(dense->ptr);
    fill_dense_kernel<<<grid_for(ctx, (int64_t)dcap, 256, 8), 256, 0, ctx.stream>>>(dr, dcap, mm);
    ctx.check_launch("fill_dense_kernel");
    {
      KernelTimer kt(ctx, "insert_kernel");
      dense_insert_kernel<<<grid_for(ctx, n, 256, 16), 256, 0, ctx.stream>>>(bk, n, mm, dcap, dr, df);
    }
    ctx.check_launch("dense_insert_kernel");
    long long* hs = reinterpret_cast<long long*>(reinterpret_cast<char*>(ctx.h_err) + 64);  // pinned
    PRISM_CUDA(cudaMemcpyAsync(hs, mm, 24, cudaMemcpyDeviceToHost, ctx.stream));
    PRISM_CUDA(cudaStreamSynchronize(ctx.stream));
    const long long h[2] = {hs[0], hs[1]};
    const uint32_t hdf = (uint32_t)hs[2];
    if (!hdf) {
      t->dense = true;
      t->dmin = h[0];
      t->drange = (uint64_t)h[1] - (uint64_t)h[0] + 1;
      t->dense_rows = dense;
      if (tune.dense_pairs) {
        // the first fixed 8-byte null-free non-key column, paired with the
        // rows in key order: a probe gathering it reads one 16-byte entry
        for (int c = 0; c < (int)build.cols.size(); ++c) {
          const Column& col = *build.cols[c];
          if (c == keys[0] || col.validity || width_of(col.type) != 8) continue;
          MemP pm = ctx.alloc(t->drange * 16);
          dense_pairs_kernel<<<grid_for(ctx, (int64_t)t->drange, 256, 8), 256, 0, ctx.stream>>>(
              dr, t->drange, static_cast<const unsigned long long*>(col.values), static_cast<ulonglong2*>(pm->ptr));
          ctx.check_launch("dense_pairs_kernel");
          t->dense_pairs = pm;
          t->dense_pair_src = col.values;
          break;
        }
      }
      return t;
    }
    // a repeated key (flag 1) or a range too wide (flag 2): hash slots
  }
  const double lf = tune.load_factor > 0 ? std::min(0.9, std::max(0.1, tune.load_factor)) : 0.5;
  uint64_t cap = next_pow2((uint64_t)std::ceil((double)std::max<int64_t>(n, 1) / lf));
  if (cap < 16) cap = 16;
  // automatic load: a table larger than L2 takes the next smaller power of
  // two while its load stays at most 0.7. Measured on 10M unique keys probed
  // by 100M Zipf(1.1) keys: 2^24 slots (load 0.6, 268 MB) probe in 0.882 ms
  // against 0.954 ms for 2^25 (0.3, 537 MB), and build 0.12 ms faster.
  if (tune.load_factor <= 0 && (cap + 1) * sizeof(ulonglong2) > (uint64_t)ctx.l2_bytes &&
      (double)std::max<int64_t>(n, 1) <= 0.7 * (double)(cap / 2))
    cap /= 2;
  t->capacity = cap;
  t->log2cap = 63 - __builtin_clzll(cap);
  t->slots = ctx.alloc((cap + 1) * sizeof(ulonglong2));
  ulonglong2* slots = static_cast<ulonglong2*>(t->slots->ptr);
  init_slots_kernel<<<grid_for(ctx, (int64_t)cap + 1, 256), 256, 0, ctx.stream>>>(slots, cap + 1);
  ctx.check_launch("init_slots_kernel");

  MemP mflag;
  uint32_t* dupflag = ctx.alloc_t<uint32_t>(1, mflag);
  PRISM_CUDA(cudaMemsetAsync(dupflag, 0, 4, ctx.stream));
  int shift = 64 - t->log2cap;
  uint64_t mask = cap - 1;
  if (n > 0) {
    int g = grid_for(ctx, n, 256, 16);
    if (use_partitioned(ctx, *t, tune)) {
      // radix-partitioned build: the keys (general keys: their row hashes)
      // in the order of the top bits of their slot hash, so the inserts of a
      // stretch of CTAs hit one slice of the table (in L2) instead of the
      // whole table at random
      const int bits = partition_bits(*t, tune);
      MemP mk, mr, mh;
      uint64_t* kpart = ctx.alloc_t<uint64_t>((size_t)n, mk);
      uint32_t* rpart = ctx.alloc_t<uint32_t>((size_t)n, mr);
      const uint64_t* src = static_cast<const uint64_t*>(build.cols[keys[0]]->values);
      if (!t->int64_fast) {
        uint64_t* h = ctx.alloc_t<uint64_t>((size_t)n, mh);
        row_hash_kernel<<<grid_for(ctx, n, 256, 16), 256, 0, ctx.stream>>>(
            static_cast<const DCol*>(t->key_views_dev->ptr), (int)keys.size(), n, h);
        ctx.check_launch("row_hash_kernel");
        src = h;
      }
      radix_partition(ctx, src, n, JOIN_FIB, 64 - bits, bits, kpart, rpart, "build_partition_hist_kernel",
                      "build_partition_scatter_kernel");
      KernelTimer kt(ctx, "insert_kernel");
      if (t->int64_fast) {
        KeysFast kf{reinterpret_cast<const int64_t*>(kpart)};
        insert_kernel<<<g, 256, 0, ctx.stream>>>(kf, n, slots, shift, mask, cap, dupflag, ctx.d_err, rpart);
      } else {
        KeysHashed kh{kpart};
        insert_kernel<<<g, 256, 0, ctx.stream>>>(kh, n, slots, shift, mask, cap, dupflag, ctx.d_err, rpart);
      }
    } else {
      KernelTimer kt(ctx, "insert_kernel");
      if (t->int64_fast) {
        KeysFast kf{static_cast<const int64_t*>(build.cols[keys[0]]->values)};
        insert_kernel<<<g, 256, 0, ctx.stream>>>(kf, n, slots, shift, mask, cap, dupflag, ctx.d_err, nullptr);
      } else {
        KeysGeneral kg{static_cast<const DCol*>(t->key_views_dev->ptr), (int)keys.size()};
        insert_kernel<<<g, 256, 0, ctx.stream>>>(kg, n, slots, shift, mask, cap, dupflag, ctx.d_err, nullptr);
      }
    }
    ctx.check_launch("insert_kernel");
  }
  // packed build keys for a single Utf8 key column
  MemP mlong, mrec;
  uint32_t* too_long = nullptr;
  if (tune.key_records && keys.size() == 1 && build.cols[keys[0]]->type == TY_UTF8 && n > 0) {
    too_long = ctx.alloc_t<uint32_t>(1, mlong);
    PRISM_CUDA(cudaMemsetAsync(too_long, 0, 4, ctx.stream));
    mrec = ctx.alloc((size_t)n * 64);
    KernelTimer kt(ctx, "pack_key_records_kernel");
    pack_key_records_kernel<<<grid_for(ctx, n, 256, 16), 256, 0, ctx.stream>>>(
        t->key_views[0], n, static_cast<ulonglong2*>(mrec->ptr), too_long);
    ctx.check_launch("pack_key_records_kernel");
  }
  uint32_t hdup = 0, hlong = 0;
  PRISM_CUDA(cudaMemcpyAsync(&hdup, dupflag, 4, cudaMemcpyDeviceToHost, ctx.stream));
  if (too_long) PRISM_CUDA(cudaMemcpyAsync(&hlong, too_long, 4, cudaMemcpyDeviceToHost, ctx.stream));
  uint32_t derr = ctx.take_device_errors();
  if (too_long && !hlong) t->key_records = mrec;
  if (derr & DERR_TABLE_FULL) fail(PRISM_ERR_TABLE_FULL, "join hash table full");
  t->has_dups = hdup != 0;
  if (t->has_dups) {
    // rows of multi-row slots, in row order, stably grouped by slot
    MemP mrs, mdup;
    uint32_t* row_slot = ctx.alloc_t<uint32_t>((size_t)n, mrs);
    uint8_t* is_dup = ctx.alloc_t<uint8_t>((size_t)n, mdup);
    int g = grid_for(ctx, n, 256, 16);
    if (t->int64_fast) {
      KeysFast kf{static_cast<const int64_t*>(build.cols[keys[0]]->values)};
      locate_kernel<<<g, 256, 0, ctx.stream>>>(kf, n, slots, shift, mask, cap, row_slot, is_dup);
    } else {
      KeysGeneral kg{static_cast<const DCol*>(t->key_views_dev->ptr), (int)keys.size()};
      locate_kernel<<<g, 256, 0, ctx.stream>>>(kg, n, slots, shift, mask, cap, row_slot, is_dup);
    }
    ctx.check_launch("locate_kernel");
    MemP mbits;
    uint8_t* bits = ctx.alloc_t<uint8_t>((size_t)(n + 31) / 8 + 8, mbits);
    pack_bits(ctx, is_dup, n, bits);
    int64_t nd = 0;
    MemP rows = compact_bits(ctx, bits, n, false, &nd);
    MemP mks;
    uint32_t* seg_slot = ctx.alloc_t<uint32_t>((size_t)std::max<int64_t>(nd, 1), mks);
    if (nd) {
      gather_u32_kernel<<<grid_for(ctx, nd, 256), 256, 0, ctx.stream>>>(row_slot, static_cast<uint32_t*>(rows->ptr),
                                                                         nd, seg_slot);
      ctx.check_launch("gather_u32_kernel");
      stable_sort_pairs_u32(ctx, seg_slot, static_cast<uint32_t*>(rows->ptr), nd, t->log2cap + 1);
      segment_heads_kernel<<<grid_for(ctx, nd, 256), 256, 0, ctx.stream>>>(seg_slot, nd, slots);
      ctx.check_launch("segment_heads_kernel");
    }
    t->dup_rows = rows;
    t->n_dup_rows = nd;
  }
  return t;
}

bool build_key_entries(Ctx& ctx, JoinTable& t, int inline_col) {
  if (t.int64_fast || t.dense || !t.slots || t.key_cols.size() != 1 || t.build.cols[t.key_cols[0]]->type != TY_UTF8)
    return false;
  int w = 0;
  const void* inl = nullptr;
  if (inline_col >= 0) {
    if (inline_col >= (int)t.build.cols.size()) fail(PRISM_ERR_INTERNAL, "inlined build column out of range");
    const Column& c = *t.build.cols[inline_col];
    w = width_of(c.type == TY_DICT ? c.index_type : c.type);
    if (c.validity || c.type == TY_BOOL || (w != 4 && w != 8)) fail(PRISM_ERR_INTERNAL, "column cannot be inlined");
    inl = c.values;
  }
  const uint64_t n_slots = t.capacity + 1;
  MemP ent = ctx.alloc((size_t)n_slots * 64);
  KernelTimer kt(ctx, "pack_key_entries_kernel");
  pack_key_entries_kernel<<<grid_for(ctx, (int64_t)n_slots, 256, 16), 256, 0, ctx.stream>>>(
      static_cast<const ulonglong2*>(t.slots->ptr), n_slots, t.key_views[0], inl, w,
      static_cast<ulonglong2*>(ent->ptr));
  ctx.check_launch("pack_key_entries_kernel");
  t.key_entries = ent;
  t.entry_col = inline_col;
  return true;
}

bool match_rows_utf8(Ctx& ctx, const JoinTable& t, const Column& pkey, int64_t n, int inline_col, uint32_t* out_match,
                     void* out_inl) {
  const bool ent = t.key_entries && t.entry_col == inline_col;
  if (t.int64_fast || t.dense || !t.slots || !(t.key_records || ent) || t.key_cols.size() != 1 ||
      t.build.cols[t.key_cols[0]]->type != TY_UTF8 || pkey.type != TY_UTF8 || t.capacity >= JOIN_MATCH_SLOT ||
      (uint64_t)t.build.rows >= JOIN_MATCH_SLOT)
    return false;
  int w = 0;
  const void* inl = nullptr;
  if (inline_col >= 0) {
    const Column& c = *t.build.cols.at(inline_col);
    w = width_of(c.type == TY_DICT ? c.index_type : c.type);
    if (c.validity || c.type == TY_BOOL || (w != 4 && w != 8)) fail(PRISM_ERR_INTERNAL, "column cannot be inlined");
    inl = c.values;
  }
  if (n <= 0) return true;
  const unsigned grid = (unsigned)ceil_div(n, (int64_t)MB * MR);
  const int shift = 64 - t.log2cap;
  const uint64_t mask = t.capacity - 1;
  const DCol pk = pkey.view();
  KernelTimer kt(ctx, "match_rows_kernel");
  if (ent) {
    const ulonglong2* e = static_cast<const ulonglong2*>(t.key_entries->ptr);
    const DCol bk = t.key_views[0];
    if (w == 8)
      match_entries_kernel<8><<<grid, MB, 0, ctx.stream>>>(pk, bk, n, e, shift, mask, out_match, out_inl);
    else if (w == 4)
      match_entries_kernel<4><<<grid, MB, 0, ctx.stream>>>(pk, bk, n, e, shift, mask, out_match, out_inl);
    else
      match_entries_kernel<0><<<grid, MB, 0, ctx.stream>>>(pk, bk, n, e, shift, mask, out_match, out_inl);
    ctx.check_launch("match_entries_kernel");
    return true;
  }
  const ulonglong2* slots = static_cast<const ulonglong2*>(t.slots->ptr);
  const ulonglong2* rec = static_cast<const ulonglong2*>(t.key_records->ptr);
  if (w == 8)
    match_rows_kernel<8><<<grid, MB, 0, ctx.stream>>>(pk, n, slots, shift, mask, rec, inl, out_match, out_inl);
  else if (w == 4)
    match_rows_kernel<4><<<grid, MB, 0, ctx.stream>>>(pk, n, slots, shift, mask, rec, inl, out_match, out_inl);
  else
    match_rows_kernel<0><<<grid, MB, 0, ctx.stream>>>(pk, n, slots, shift, mask, rec, inl, out_match, out_inl);
  ctx.check_launch("match_rows_kernel");
  return true;
}

int64_t match_upper_bound(const JoinTable& t, int64_t probe_rows) {
  return t.has_dups ? -1 : probe_rows;
}

static void fill_common(Ctx& ctx, const JoinTable& t, const Batch& probe, const std::vector<int>& keys, ProbeArgs& a,
                        std::vector<DCol>& pviews, MemP& pviews_dev, bool upload_views = true) {
  a = ProbeArgs{};
  a.n = probe.rows;
  a.dense = t.dense ? static_cast<const uint32_t*>(t.dense_rows->ptr) : nullptr;
  a.dmin = t.dmin;
  a.drange = t.drange;
  a.slots = t.slots ? static_cast<const ulonglong2*>(t.slots->ptr) : nullptr;
  a.shift = 64 - t.log2cap;
  a.mask = t.capacity - 1;
  a.cap = t.capacity;
  a.dup_rows = t.dup_rows ? static_cast<const uint32_t*>(t.dup_rows->ptr) : nullptr;
  a.n_dup_rows = t.n_dup_rows;
  a.krec = t.key_records ? static_cast<const ulonglong2*>(t.key_records->ptr) : nullptr;
  a.nkeys = (int)keys.size();
  a.err = ctx.d_err;
  a.bcols = static_cast<const DCol*>(t.key_views_dev->ptr);
  a.n_tiles = ceil_div(a.n, PT);
  if (!upload_views) return;  // (the kernels of single Int64 keys read the key column directly)
  for (int k : keys) pviews.push_back(probe.cols[k]->view());
  pviews_dev = ctx.alloc(pviews.size() * sizeof(DCol));
  ctx.h2d_staged(pviews_dev->ptr, pviews.data(), pviews.size() * sizeof(DCol));
  a.pcols = static_cast<const DCol*>(pviews_dev->ptr);
}

int64_t probe_count(Ctx& ctx, const JoinTable& t, const Batch& probe, const std::vector<int>& keys,
                    const JoinTuning& tune) {
  check_join_keys(probe, keys, t.build, t.key_cols);
  if (probe.rows == 0 || t.build.rows == 0) return 0;
  ProbeArgs a;
  std::vector<DCol> pv;
  MemP pvd;
  fill_common(ctx, t, probe, keys, a, pv, pvd);
  MemP mc, mt;
  a.tile_counter = ctx.alloc_t<unsigned long long>(1, mc);
  a.total = ctx.alloc_t<unsigned long long>(1, mt);
  PRISM_CUDA(cudaMemsetAsync(a.tile_counter, 0, 8, ctx.stream));
  PRISM_CUDA(cudaMemsetAsync(a.total, 0, 8, ctx.stream));
  if (t.int64_fast)
    launch_probe<KeysFast, false>(ctx, t, KeysFast{static_cast<const int64_t*>(probe.cols[keys[0]]->values)}, a,
                                  tune.probe_blocks_per_sm);
  else
    launch_probe<KeysGeneral, false>(ctx, t, KeysGeneral{a.pcols, a.nkeys}, a, tune.probe_blocks_per_sm);
  unsigned long long total = 0;
  PRISM_CUDA(cudaMemcpyAsync(&total, a.total, 8, cudaMemcpyDeviceToHost, ctx.stream));
  uint32_t derr = ctx.take_device_errors();
  if (derr & DERR_TIMEOUT) fail(PRISM_ERR_TIMEOUT, "probe look-back timed out");
  if (derr & DERR_CORRUPT) fail(PRISM_ERR_INTERNAL, "join table inconsistent (build rows changed while it was built?)");
  return (int64_t)total;
}

ProbeResult probe_join_table(Ctx& ctx, const JoinTable& t, const Batch& probe, const std::vector<int>& keys,
                             bool want_probe_idx, bool want_build_idx, std::vector<ProbeGather>& gathers,
                             int64_t gather_capacity, const JoinTuning& tune, bool any_order, int64_t row_base) {
  check_join_keys(probe, keys, t.build, t.key_cols);
  ProbeResult res;
  if (gathers.size() > 4) fail(PRISM_ERR_INTERNAL, "at most 4 fused gathers");
  int64_t cap = gather_capacity;
  if (cap < 0) {
    int64_t ub = match_upper_bound(t, probe.rows);
    cap = ub >= 0 ? ub : probe_count(ctx, t, probe, keys, tune);
  }
  if (want_probe_idx) res.probe_idx = ctx.alloc((size_t)std::max<int64_t>(cap, 1) * 4);
  if (want_build_idx) res.build_idx = ctx.alloc((size_t)std::max<int64_t>(cap, 1) * 4);
  if (probe.rows == 0 || t.build.rows == 0) return res;
  ProbeArgs a;
  std::vector<DCol> pv;
  MemP pvd;
  const bool one_pass = any_order && t.int64_fast && !t.has_dups;
  fill_common(ctx, t, probe, keys, a, pv, pvd, !one_pass);
  a.out_probe = want_probe_idx ? static_cast<uint32_t*>(res.probe_idx->ptr) : nullptr;
  a.out_build = want_build_idx ? static_cast<uint32_t*>(res.build_idx->ptr) : nullptr;
  a.ngather = (int)gathers.size();
  for (size_t g = 0; g < gathers.size(); ++g) {
    a.g_side[g] = gathers[g].side;
    a.g_src[g] = gathers[g].src;
    a.g_width[g] = gathers[g].width;
    a.g_dst[g] = gathers[g].dst;
  }
  a.out_capacity = (uint64_t)cap;
  a.row_base = row_base;
  if (one_pass) {
    // unique Int64 keys, matches as a multiset: one pass, one atomicAdd per
    // tile on the context's match counter (bytes 8-15 of its error words),
    // read back with the error word by one copy and one synchronisation
    unsigned long long* dtot = reinterpret_cast<unsigned long long*>(reinterpret_cast<char*>(ctx.d_err) + 8);
    a.total = dtot;
    const int64_t n = probe.rows;
    const int64_t* pk = static_cast<const int64_t*>(probe.cols[keys[0]]->values);
    const bool vec = (reinterpret_cast<uintptr_t>(pk) & 15) == 0;
    const unsigned grid = (unsigned)ceil_div(n, AT);
    a.prefetch_ahead = any_prefetch_ahead(ctx, t.dense);
    if (t.dense && t.dense_pairs && gathers.size() == 1 && gathers[0].side == 1 && gathers[0].width == 8 &&
        gathers[0].src == t.dense_pair_src)
      a.dpairs = static_cast<const ulonglong2*>(t.dense_pairs->ptr);
    if (!t.dense && use_partitioned(ctx, t, tune)) {
      // radix-partitioned probe: the keys reordered by the top bits of their
      // slot hash, so each tile probes one slice of the table
      PRISM_CUDA(cudaMemsetAsync(dtot, 0, 8, ctx.stream));
      MemP mk, mr;
      uint64_t* kpart = ctx.alloc_t<uint64_t>((size_t)n, mk);
      uint32_t* rpart = ctx.alloc_t<uint32_t>((size_t)n, mr);
      const int bits = partition_bits(t, tune);
      radix_partition(ctx, reinterpret_cast<const uint64_t*>(pk), n, JOIN_FIB, 64 - bits, bits, kpart, rpart,
                      "probe_partition_hist_kernel", "probe_partition_scatter_kernel");
      {
        KernelTimer kt(ctx, "probe_emit_any_kernel");
        probe_emit_any_kernel<false, true, true><<<grid, AB, 0, ctx.stream>>>(reinterpret_cast<const int64_t*>(kpart),
                                                                               rpart, n, a);
      }
      ctx.check_launch("probe_emit_any_kernel");
      PRISM_CUDA(cudaMemcpyAsync(ctx.h_err, ctx.d_err, 16, cudaMemcpyDeviceToHost, ctx.stream));
    } else {
      const void* fn = t.dense ? (vec ? (const void*)probe_emit_any_kernel<true, true, false>
                                      : (const void*)probe_emit_any_kernel<true, false, false>)
                               : (vec ? (const void*)probe_emit_any_kernel<false, true, false>
                                      : (const void*)probe_emit_any_kernel<false, false, false>);
      const int64_t* kp = pk;
      const uint32_t* rp = nullptr;
      int64_t nn = n;
      void* args[] = {&kp, &rp, &nn, &a};
      KernelTimer kt(ctx, "probe_emit_any_kernel");
      if (probe_graphs_on()) {
        launch_probe_graph(ctx, fn, grid, args);
      } else {
        PRISM_CUDA(cudaMemsetAsync(dtot, 0, 8, ctx.stream));
        PRISM_CUDA(cudaLaunchKernel(fn, dim3(grid), dim3(AB), args, 0, ctx.stream));
        ctx.check_launch("probe_emit_any_kernel");
        PRISM_CUDA(cudaMemcpyAsync(ctx.h_err, ctx.d_err, 16, cudaMemcpyDeviceToHost, ctx.stream));
      }
    }
    PRISM_CUDA(cudaStreamSynchronize(ctx.stream));
    const uint32_t derr = ctx.h_err[0];
    const unsigned long long total = *reinterpret_cast<const unsigned long long*>(reinterpret_cast<const char*>(ctx.h_err) + 8);
    if (derr) PRISM_CUDA(cudaMemsetAsync(ctx.d_err, 0, sizeof(uint32_t), ctx.stream));
    if (derr & DERR_CAPACITY) fail(PRISM_ERR_INTERNAL, "probe output capacity exceeded");
    if (derr & DERR_TIMEOUT) fail(PRISM_ERR_TIMEOUT, "probe: a wait timed out");
    res.matches = (int64_t)total;
    return res;
  }
  a.any_order = any_order ? 1 : 0;
  if (t.int64_fast && !t.has_dups) {
    // unique Int64 keys: probe, scan of tile counts, ordered emit
    int64_t n = probe.rows, ntiles = ceil_div(n, QT);
    MemP mrow, mcnt, moff, mtot;
    uint32_t* rowv = ctx.alloc_t<uint32_t>((size_t)n, mrow);
    uint32_t* tcnt = ctx.alloc_t<uint32_t>((size_t)ntiles, mcnt);
    uint64_t* toff = ctx.alloc_t<uint64_t>((size_t)ntiles, moff);
    uint64_t* dtot = ctx.alloc_t<uint64_t>(1, mtot);
    a.err = ctx.d_err;
    {
      KernelTimer kt(ctx, "probe_rows_kernel");
      const int64_t* pk = static_cast<const int64_t*>(probe.cols[keys[0]]->values);
      if (t.dense)
        probe_rows_dense_kernel<<<(unsigned)ntiles, QB, 0, ctx.stream>>>(pk, n, a.dense, a.dmin, a.drange, rowv, tcnt);
      else
        probe_rows_kernel<<<(unsigned)ntiles, QB, 0, ctx.stream>>>(pk, n, a.slots, a.shift, a.mask, a.cap, rowv, tcnt);
    }
    ctx.check_launch("probe_rows_kernel");
    scan_u32_async(ctx, tcnt, toff, ntiles, dtot);
    {
      KernelTimer kt(ctx, "emit_rows_kernel");
      emit_rows_kernel<<<(unsigned)ntiles, QB, 0, ctx.stream>>>(rowv, n, toff, a);
    }
    ctx.check_launch("emit_rows_kernel");
    uint64_t total = 0;
    PRISM_CUDA(cudaMemcpyAsync(&total, dtot, 8, cudaMemcpyDeviceToHost, ctx.stream));
    uint32_t derr = ctx.take_device_errors();
    if (derr & DERR_CAPACITY) fail(PRISM_ERR_INTERNAL, "probe output capacity exceeded");
    res.matches = (int64_t)total;
    return res;
  }
  MemP ms, mc, mt;
  a.tile_status = ctx.alloc_t<unsigned long long>((size_t)a.n_tiles, ms);
  a.tile_counter = ctx.alloc_t<unsigned long long>(1, mc);
  a.total = ctx.alloc_t<unsigned long long>(1, mt);
  PRISM_CUDA(cudaMemsetAsync(a.tile_status, 0, (size_t)a.n_tiles * 8, ctx.stream));
  PRISM_CUDA(cudaMemsetAsync(a.tile_counter, 0, 8, ctx.stream));
  PRISM_CUDA(cudaMemsetAsync(a.total, 0, 8, ctx.stream));
  if (t.int64_fast)
    launch_probe<KeysFast, true>(ctx, t, KeysFast{static_cast<const int64_t*>(probe.cols[keys[0]]->values)}, a,
                                 tune.probe_blocks_per_sm);
  else
    launch_probe<KeysGeneral, true>(ctx, t, KeysGeneral{a.pcols, a.nkeys}, a, tune.probe_blocks_per_sm);
  unsigned long long total = 0;
  PRISM_CUDA(cudaMemcpyAsync(&total, a.total, 8, cudaMemcpyDeviceToHost, ctx.stream));
  uint32_t derr = ctx.take_device_errors();
  if (derr & DERR_TIMEOUT) fail(PRISM_ERR_TIMEOUT, "probe look-back timed out");
  if (derr & DERR_CORRUPT) fail(PRISM_ERR_INTERNAL, "join table inconsistent (build rows changed while it was built?)");
  if (derr & DERR_CAPACITY) fail(PRISM_ERR_INTERNAL, "probe output capacity exceeded");
  res.matches = (int64_t)total;
  return res;
}

// ------------------------------------------------ allocation-free probe ----
// For callers that may not allocate device memory while they run: the
// single-pass probe with its look-back scratch (one status word per
// 2048-row tile, the tile counter and the match total) in a file-scope
// device array instead of a per-call allocation.
namespace {

constexpr int64_t NOALLOC_MAX_TILES = 131072;  // x 2048 rows = 268,435,456 probe rows
constexpr int NOALLOC_MAX_DEVICES = 64;
static __device__ __align__(256) unsigned long long g_noalloc_scratch[NOALLOC_MAX_TILES + 32];

std::mutex g_noalloc_mu;
unsigned long long* g_noalloc_addr[NOALLOC_MAX_DEVICES];

// Device address of g_noalloc_scratch on `device`, looked up once per device
// with that device current. In host code the symbol's name is only a
// host-side stand-in and must never be passed to a kernel.
unsigned long long* noalloc_scratch(int device) {
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (device < 0 || device >= NOALLOC_MAX_DEVICES) fail(PRISM_ERR_INVALID_ARGUMENT, "device index out of range");
  if (!g_noalloc_addr[device]) {
    int cur = -1;
    PRISM_CUDA(cudaGetDevice(&cur));
    if (cur != device) PRISM_CUDA(cudaSetDevice(device));
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (cur != device) cudaSetDevice(cur);
    if (e != cudaSuccess) {
      cudaGetLastError();
      fail(PRISM_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
    }
    g_noalloc_addr[device] = static_cast<unsigned long long*>(p);
  }
  return g_noalloc_addr[device];
}

}  // namespace

}  // namespace prism

extern "C" int prism_hash_table_probe_noalloc(prism_ctx* c, const prism_hash_table* tab, const int64_t* probe_keys,
                                              int64_t n_probe, uint32_t* out_probe_idx, uint32_t* out_build_idx,
                                              int64_t out_capacity, int64_t* out_matches) {
  using namespace prism;
  if (!c) return PRISM_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(c->impl.mu);
  try {
    Ctx& ctx = c->impl;
    if (!tab || !tab->t || !out_matches) fail(PRISM_ERR_INVALID_ARGUMENT, "null table or out_matches");
    const JoinTable& t = *tab->t;
    if (!t.int64_fast)
      fail(PRISM_ERR_INVALID_ARGUMENT, "the allocation-free probe needs a table with one Int64 key column");
    if (n_probe < 0 || out_capacity < 0) fail(PRISM_ERR_INVALID_ARGUMENT, "negative size");
    int64_t n_tiles = ceil_div(n_probe, PT);
    if (n_tiles > NOALLOC_MAX_TILES)
      fail(PRISM_ERR_INVALID_ARGUMENT, "n_probe " + std::to_string(n_probe) +
                                           " exceeds the allocation-free probe's maximum of " +
                                           std::to_string(NOALLOC_MAX_TILES * PT) + " rows");
    if (n_probe > 0 && !probe_keys) fail(PRISM_ERR_INVALID_ARGUMENT, "null probe keys");
    if (out_capacity > 0 && (!out_probe_idx || !out_build_idx)) fail(PRISM_ERR_INVALID_ARGUMENT, "null outputs");
    *out_matches = 0;
    if (n_probe == 0 || t.build.rows == 0) return PRISM_OK;

    unsigned long long* scratch = noalloc_scratch(ctx.device);
    unsigned long long* status = scratch;
    unsigned long long* counter = scratch + NOALLOC_MAX_TILES;
    unsigned long long* total = counter + 1;
    // the array keeps the previous call's contents: clear what this call uses
    PRISM_CUDA(cudaMemsetAsync(status, 0, (size_t)n_tiles * 8, ctx.stream));
    PRISM_CUDA(cudaMemsetAsync(counter, 0, 16, ctx.stream));

    ProbeArgs a{};
    a.n = n_probe;
    a.dense = t.dense ? static_cast<const uint32_t*>(t.dense_rows->ptr) : nullptr;
    a.dmin = t.dmin;
    a.drange = t.drange;
    a.slots = t.slots ? static_cast<const ulonglong2*>(t.slots->ptr) : nullptr;
    a.shift = 64 - t.log2cap;
    a.mask = t.capacity - 1;
    a.cap = t.capacity;
    a.dup_rows = t.dup_rows ? static_cast<const uint32_t*>(t.dup_rows->ptr) : nullptr;
    a.n_dup_rows = t.n_dup_rows;
    a.nkeys = 1;
    a.out_probe = out_probe_idx;
    a.out_build = out_build_idx;
    a.ngather = 0;
    a.out_capacity = (uint64_t)out_capacity;
    a.tile_status = status;
    a.tile_counter = counter;
    a.n_tiles = n_tiles;
    a.total = total;
    a.err = ctx.d_err;
    int grid = (int)std::min<int64_t>(n_tiles, (int64_t)ctx.sm_count * 2);
    if (t.has_dups)
      probe_kernel<KeysFast, true, false, true><<<grid, PW * 32, 0, ctx.stream>>>(KeysFast{probe_keys}, a);
    else
      probe_kernel<KeysFast, false, false, true><<<grid, PW * 32, 0, ctx.stream>>>(KeysFast{probe_keys}, a);
    ctx.check_launch("probe_kernel(noalloc)");
    unsigned long long tot = 0;
    PRISM_CUDA(cudaMemcpyAsync(&tot, total, 8, cudaMemcpyDeviceToHost, ctx.stream));
    uint32_t derr = ctx.take_device_errors();
    if (derr & DERR_TIMEOUT) fail(PRISM_ERR_TIMEOUT, "probe look-back timed out");
    if (derr & DERR_CORRUPT) fail(PRISM_ERR_INTERNAL, "join table inconsistent (build rows changed while it was built?)");
    *out_matches = (int64_t)tot;
    if (derr & DERR_CAPACITY)
      fail(PRISM_ERR_INVALID_ARGUMENT, "output capacity " + std::to_string(out_capacity) + " is smaller than the " +
                                           std::to_string(tot) + " matches");
    return PRISM_OK;
  } catch (const Failure& f) {
    c->impl.last_error = f.msg;
    cudaGetLastError();
    return f.code;
  } catch (const std::exception& e) {
    c->impl.last_error = e.what();
    return PRISM_ERR_INTERNAL;
  }
}
