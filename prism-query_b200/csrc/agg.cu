// agg.cu — GROUP BY aggregation on the device.
//
// Replaces hash_aggregate / hash_aggregate_batches
// (native/prism-executor/src/hash_aggregate.rs:174-447). Semantics kept:
//   * group identity = the reference's 64-bit FxHash of the key columns
//     (hash_aggregate.rs:24-75, 483-504): a null key hashes like 0, and two
//     keys with equal hashes share a group, exactly as in the reference;
//   * every numeric input is read as its Float64 cast; the grouped path does
//     not skip nulls (it reads the raw slot), the global path does;
//   * groups are emitted in first-seen order over the concatenated batches,
//     with the key value of the group's first row.
// Accumulation is order-independent and exact: integer SUMs in 128-bit
// integers, Float64 SUMs in a 192-bit fixed-point window held as six 32-bit
// limbs in 64-bit carry-save counters, rounded once at the end (so results
// do not depend on thread scheduling). MIN/MAX use the IEEE totalOrder key.
//
// Kernel structure: each CTA keeps a shared-memory hash table of group keys
// that maps to dense shared accumulator rows (privatised, shared-memory
// atomics); rows whose group does not fit go straight to the global
// open-addressing table in HBM (64-bit atomicCAS inserts). At the end the CTA
// merges its rows into the global table. Dictionary-encoded keys and the
// global (no GROUP BY) case use dense group ids instead of hashing.
#include <algorithm>
#include <cmath>
#include <map>

#include "agg.hpp"
#include "agg_device.cuh"
#include "jit.hpp"
#include "join.hpp"
#include "prims.hpp"

namespace prism {

namespace {

// PRISM_JOIN_SPLIT=1: the fused join -> aggregate over a Utf8 key reads
// match_rows_kernel's per-row match words instead of looking its keys up
// itself (measured: the same time per step on the 15M-key workload, so off)
bool join_split() {
  const char* e = std::getenv("PRISM_JOIN_SPLIT");
  return e && std::strcmp(e, "1") == 0;
}

bool join_key_words_on() {
  const char* e = std::getenv("PRISM_JOIN_KEY_WORDS");
  return !(e && std::strcmp(e, "0") == 0);
}

struct RowVals {
  double f[MAX_SRC];
  __int128 i[MAX_SRC];
  bool valid[MAX_SRC];
};

__device__ __forceinline__ void load_sources(const AggArgs& a, int64_t row, RowVals& v, uint32_t* err) {
  for (int s = 0; s < a.n_src; ++s) {
    const Src& sr = a.src[s];
    switch (sr.kind) {
      // inputs as arrow's cast to Float64 leaves them (hash_aggregate.rs:227-245)
      case S_COL_F64: v.f[s] = dcol_fval_cast(a.cols[sr.col], row); v.valid[s] = dcol_valid(a.cols[sr.col], row); break;
      case S_COL_INT: v.i[s] = dcol_ival_cast(a.cols[sr.col], row); v.valid[s] = dcol_valid(a.cols[sr.col], row); break;
      case S_COL_I128: v.i[s] = dcol_i128_cast(a.cols[sr.col], row); v.valid[s] = dcol_valid(a.cols[sr.col], row); break;
      case S_VALID: v.valid[s] = dcol_valid(a.cols[sr.col], row); break;
      case S_EXPR_F64: case S_EXPR_I128: {
        bool ovf = false;
        Val r = eval_expr(a.en, sr.begin, sr.end, a.pn, a.cl, a.cols, row, &ovf);
        if (ovf) atomicOr(err, DERR_RANGE);
        v.f[s] = r.f;
        v.i[s] = r.i;
        v.valid[s] = r.valid;
        break;
      }
    }
  }
}

__device__ __forceinline__ void apply_ops(const AggArgs& a, unsigned long long* acc, const RowVals& v, int64_t slot) {
  if (a.count_rows) atomicAdd(acc, 1ULL);
  for (int j = 0; j < a.n_ops; ++j) {
    const Op& o = a.op[j];
    if (o.kind == O_DISTINCT) continue;
    bool valid = v.valid[o.src];
    if (a.skip_nulls && !valid) continue;
    unsigned long long* w = acc + o.word;
    switch (o.kind) {
      case O_SUM_F64:
        if (a.wide)
          add_f64(a.gwide + ((size_t)slot * a.n_wide + o.distinct) * (WIDE_LIMBS + 1), v.f[o.src], WIDE_LO, a.err,
                  a.maxexp + j, WIDE_LIMBS);
        else
          add_f64(w, v.f[o.src], o.lo_exp, a.err, a.maxexp + j);
        break;
      case O_SUM_INT: add_i128_limbs(w, f64_cast_int((long long)v.i[o.src]), 2); break;
      case O_SUM_DEC: add_i128_limbs(w, v.i[o.src], 4); break;
      case O_MIN: {
        double d = v.f[o.src];
        if (!isnan(d)) atomicMin((long long*)w, (long long)total_key(d));
        break;
      }
      case O_MAX: {
        double d = v.f[o.src];
        if (!isnan(d)) atomicMax((long long*)w, (long long)total_key(d));
        break;
      }
      case O_NONNULL:
        if (valid) atomicAdd(w, 1ULL);
        break;
    }
  }
}

__device__ __forceinline__ uint64_t dist_value_id(const AggArgs& a, const Op& o, int64_t row, bool& ok) {
  const Src& sr = a.src[o.src];
  const DCol& c = a.cols[sr.col];
  ok = dcol_valid(c, row);
  if (!ok) return 0;
  switch (c.type) {
    case TY_F64: {  // distinct_value canonicalisation (hash_aggregate.rs:465-475)
      double d = static_cast<const double*>(c.values)[row];
      if (d == 0.0) return 0;
      if (isnan(d)) return 0x7ff8000000000000ULL;
      return (uint64_t)__double_as_longlong(d);
    }
    case TY_UTF8: case TY_DICT: {
      const uint8_t* p;
      int32_t n;
      dcol_str(c, row, p, n);
      return mix64(fx_str(0x9E3779B97F4A7C15ULL, p, n)) ^ (uint64_t)n;
    }
    case TY_DEC128: {
      const uint64_t* p = static_cast<const uint64_t*>(c.values) + 2 * row;
      return p[0] ^ mix64(p[1] + 0x632BE59BD9B4E019ULL);
    }
    case TY_F32: return (uint64_t)__float_as_uint(static_cast<const float*>(c.values)[row]);
    default: return (uint64_t)dcol_ival(c, row);
  }
}

// Inserts (group, value) into a distinct set; duplicates are ignored.
__device__ void distinct_insert(const DistinctTable& t, uint64_t g, uint64_t v, uint32_t* err) {
  uint64_t s = mix64(g * FIB ^ mix64(v)) & t.mask;
  if (g == GEMPTY && v == GEMPTY) v = GEMPTY - 1;  // keep the empty marker free
  for (uint64_t step = 0; step <= t.mask; ++step) {
    unsigned long long* p = t.slots + 2 * s;
    unsigned long long hi;
    unsigned long long lo = cas128(p, GEMPTY, GEMPTY, g, v, hi);
    if ((lo == GEMPTY && hi == GEMPTY) || (lo == g && hi == v)) return;
    s = (s + 1) & t.mask;
  }
  atomicOr(err, DERR_TABLE_FULL);
}

__device__ __forceinline__ uint64_t group_hash(const AggArgs& a, int64_t row) {
  uint64_t h = 0;
  for (int k = 0; k < a.n_gcols; ++k) h = fx_value(h, a.cols[a.gcol[k]], row);
  return h;
}

__device__ __forceinline__ int64_t dense_gid(const AggArgs& a, int64_t row) {
  int64_t g = 0;
  for (int k = 0; k < a.n_gcols; ++k) {
    const DCol& c = a.cols[a.gcol[k]];
    int64_t code = dcol_valid(c, row) ? dcol_ival(c, row) : a.dnull[k];
    g += code * a.dstride[k];
  }
  return g;
}

__device__ int64_t gfind(const AggArgs& a, uint64_t h) {
  if (h == GEMPTY) return (int64_t)a.gcap;
  uint64_t s = (h * FIB) >> a.gshift;
  for (uint64_t step = 0; step <= a.gmask; ++step) {
    unsigned long long cur = a.gkeys[s];
    if (cur == h) return (int64_t)s;
    if (cur == GEMPTY) return -1;
    s = (s + 1) & a.gmask;
  }
  return -1;
}

// Every word of a fresh group table: keys empty, first rows unset,
// accumulators at their initial values, counters zero.
__global__ void init_table_kernel(AggArgs a, int64_t nslots) {
  const int64_t words = nslots * a.W;
  const int64_t n = words > nslots ? words : nslots;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (i < nslots) {
      if (a.gkeys) a.gkeys[i] = GEMPTY;
      a.gfirst[i] = ~0ULL;
    }
    if (i < words) a.gacc[i] = a.winit[i % a.W];
    if (i < MAX_OPS) a.maxexp[i] = 0;
    if (i == 0 && a.gnew_count) *a.gnew_count = 0;
  }
}

// The aggregation kernel. Dynamic shared memory (hash mode):
//   skeys[SS] u64 | sfirst[SD] u64 | skeyof[SD] u64 | sacc[SD*W] u64 | sidx[SS] i32
// Dense mode: sfirst[G] | sacc[G*W] when G fits, else global atomics only.
__global__ void __launch_bounds__(512) agg_kernel(AggArgs a) {
  extern __shared__ unsigned long long smem[];
  __shared__ int s_count;
  const int SS = a.ss_log2 > 0 ? (1 << a.ss_log2) : 0;
  const bool dense = a.dense != 0;
  const int SD = dense ? (int)a.G : a.sd;
  const bool use_smem = a.use_smem != 0 && SD > 0;
  unsigned long long* skeys = smem;
  unsigned long long* sfirst = skeys + SS;
  unsigned long long* skeyof = sfirst + SD;
  unsigned long long* sacc = skeyof + (dense ? 0 : SD);
  int* sidx = reinterpret_cast<int*>(sacc + (size_t)SD * a.W);
  if (use_smem) {
    for (int i = threadIdx.x; i < SS; i += blockDim.x) { skeys[i] = GEMPTY; sidx[i] = -1; }
    for (int i = threadIdx.x; i < SD; i += blockDim.x) sfirst[i] = ~0ULL;
    for (int i = threadIdx.x; i < SD * a.W; i += blockDim.x) sacc[i] = a.winit[i % a.W];
  }
  if (threadIdx.x == 0) s_count = 0;
  __syncthreads();

  int64_t per = ceil_div_dev(a.n, gridDim.x);
  per = (per + 31) & ~int64_t(31);
  int64_t lo = (int64_t)blockIdx.x * per, hi = lo + per < a.n ? lo + per : a.n;
  RowVals v;
  for (int64_t row = lo + threadIdx.x; row < hi; row += blockDim.x) {
    if (a.has_filter) {
      bool pv;
      bool keep = eval_pred(a.pn, a.filter.begin, a.filter.len, a.cols, row, pv);
      if (!(keep && pv)) continue;
    }
    uint64_t grow = a.row_base + (uint64_t)row;
    int d = -1;
    uint64_t h = 0;
    if (dense) {
      int64_t gid = dense_gid(a, row);
      if (gid < 0 || gid >= a.G) { atomicOr(a.err, DERR_RANGE); continue; }
      d = (int)gid;
    } else {
      h = group_hash(a, row);
      if (use_smem && h != GEMPTY) {
        uint32_t s = (uint32_t)((h * FIB) >> (64 - a.ss_log2));
        for (int step = 0; step < SS; ++step) {
          unsigned long long cur = *(volatile unsigned long long*)&skeys[s];
          if (cur == GEMPTY) {
            unsigned long long prev = atomicCAS(&skeys[s], GEMPTY, h);
            if (prev == GEMPTY) {
              int nd = atomicAdd(&s_count, 1);
              if (nd < SD) { skeyof[nd] = h; sidx[s] = nd; }
              else sidx[s] = -2;  // overflow marker: this group goes global
              __threadfence_block();
              cur = h;
            } else {
              cur = prev;
            }
          }
          if (cur == h) {
            int x;
            uint32_t spins = 0;
            while ((x = *(volatile int*)&sidx[s]) == -1 && spins < SPIN_LIMIT) ++spins;
            if (x == -1) atomicOr(a.err, DERR_TIMEOUT);
            d = x >= 0 ? x : -1;
            break;
          }
          s = (s + 1) & (SS - 1);
        }
      }
    }
    unsigned long long* acc;
    int64_t gs = -1;
    if (d >= 0 && use_smem) {
      acc = sacc + (size_t)d * a.W;
      if (grow < sfirst[d]) atomicMin(&sfirst[d], grow);
    } else {
      gs = dense ? (int64_t)d : ginsert(a, h);
      if (gs < 0) continue;
      acc = a.gacc + (size_t)gs * a.W;
      if (grow < a.gfirst[gs]) atomicMin(&a.gfirst[gs], grow);
    }
    load_sources(a, row, v, a.err);
    apply_ops(a, acc, v, gs);
    // COUNT DISTINCT values go to their own sets keyed by (group, value)
    for (int j = 0; j < a.n_ops; ++j) {
      if (a.op[j].kind != O_DISTINCT) continue;
      bool ok;
      uint64_t vid = dist_value_id(a, a.op[j], row, ok);
      if (ok) distinct_insert(a.dt[a.op[j].distinct], dense ? (uint64_t)d : h, vid, a.err);
    }
  }
  __syncthreads();
  if (!use_smem) return;
  int used = dense ? SD : (s_count < SD ? s_count : SD);
  for (int d = threadIdx.x; d < used; d += blockDim.x) {
    if (sfirst[d] == ~0ULL) continue;  // no row of this CTA
    int64_t gs = dense ? d : ginsert(a, skeyof[d]);
    if (gs < 0) continue;
    atomicMin(&a.gfirst[gs], sfirst[d]);
    const unsigned long long* src = sacc + (size_t)d * a.W;
    unsigned long long* dst = a.gacc + (size_t)gs * a.W;
    for (int w = 0; w < a.W; ++w)
      if (src[w] != a.winit[w]) merge_word(dst + w, src[w], a.wkind[w]);
  }
}

// ----------------------------------------------------------- finalize ----
__global__ void collect_groups_kernel(const unsigned long long* gfirst, int64_t nslots, uint32_t* out_slots,
                                      unsigned long long* counter) {
  for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < nslots; s += (int64_t)gridDim.x * blockDim.x)
    if (gfirst[s] != ~0ULL) out_slots[atomicAdd(counter, 1ULL)] = (uint32_t)s;
}

__global__ void mark_first_kernel(const unsigned long long* gfirst, const uint32_t* slots, int64_t n, uint32_t* bits) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t r = gfirst[slots[i]];
    atomicOr(&bits[r >> 5], 1u << (r & 31));
  }
}

__global__ void word_popc32_kernel(const uint32_t* bits, int64_t nw, uint32_t* cnt) {
  for (int64_t w = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; w < nw; w += (int64_t)gridDim.x * blockDim.x)
    cnt[w] = __popc(bits[w]);
}

__global__ void place_groups_kernel(const unsigned long long* gfirst, const uint32_t* slots, int64_t n,
                                    const uint32_t* bits, const uint64_t* woff, uint32_t* ordered,
                                    unsigned long long* ordered_first) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t s = slots[i];
    uint64_t r = gfirst[s];
    uint64_t pos = woff[r >> 5] + __popc(bits[r >> 5] & ((1u << (r & 31)) - 1u));
    ordered[pos] = s;
    ordered_first[pos] = r;
  }
}

// Up to SMALL_GROUPS groups are put in first-seen order by one block: the
// groups' (first row, slot) pairs sorted in shared memory (bitonic, 64-bit
// order keys: a row index, or a fused join's (probe row << 32 | build row)).
// The candidates are the slots ginsert listed (plus the side slot when
// used), or, for dense ids, every slot with a row. out[0] = the group count,
// or ~0 when there are more groups than the block sorts (the general path
// then orders them). Dynamic shared memory: SMALL_GROUPS * 12 bytes.
constexpr int SMALL_GROUPS = 4096;
constexpr size_t SMALL_SMEM = SMALL_GROUPS * 12;
__global__ void __launch_bounds__(1024) small_order_kernel(const unsigned long long* gfirst, const uint32_t* gnew,
                                                           const unsigned long long* gnew_count, int64_t scan_n,
                                                           int64_t side, uint32_t* ordered, unsigned long long* firsts,
                                                           uint32_t* rows32, unsigned long long* out) {
  extern __shared__ unsigned long long okey[];  // [SMALL_GROUPS] order keys | [SMALL_GROUPS] u32 slots
  uint32_t* oslot = reinterpret_cast<uint32_t*>(okey + SMALL_GROUPS);
  __shared__ unsigned int cnt;
  const int tid = threadIdx.x;
  if (gnew) {
    const unsigned long long listed = *gnew_count;
    if (listed > (unsigned long long)(SMALL_GROUPS - 1)) {  // one entry left for the side slot
      if (tid == 0) *out = ~0ULL;
      return;
    }
    for (int i = tid; i < (int)listed; i += blockDim.x) {
      const uint32_t s = gnew[i];
      okey[i] = gfirst[s];
      oslot[i] = s;
    }
    if (tid == 0) {
      cnt = (unsigned int)listed;
      if (side >= 0 && gfirst[side] != ~0ULL) {
        okey[cnt] = gfirst[side];
        oslot[cnt] = (uint32_t)side;
        ++cnt;
      }
    }
  } else {
    if (tid == 0) cnt = 0;
    __syncthreads();
    for (int64_t s = tid; s < scan_n; s += blockDim.x)
      if (gfirst[s] != ~0ULL) {
        const unsigned int p = atomicAdd(&cnt, 1u);
        okey[p] = gfirst[s];
        oslot[p] = (uint32_t)s;
      }
  }
  __syncthreads();
  const int n = (int)cnt;
  if (n <= (int)blockDim.x) {
    // up to one key per thread: its rank is the number of smaller keys (the
    // keys are distinct), every thread reading the same key at once
    const unsigned long long mine = tid < n ? okey[tid] : 0ULL;
    const uint32_t slot = tid < n ? oslot[tid] : 0u;
    int rank = 0;
    for (int j = 0; j < n; ++j) rank += okey[j] < mine ? 1 : 0;
    if (tid < n) {
      ordered[rank] = slot;
      firsts[rank] = mine;
      rows32[rank] = (uint32_t)mine;
    }
    if (tid == 0) *out = (unsigned long long)n;
    return;
  }
  int m = 1;
  while (m < n) m <<= 1;
  for (int i = n + tid; i < m; i += blockDim.x) {
    okey[i] = ~0ULL;
    oslot[i] = 0xFFFFFFFFu;
  }
  __syncthreads();
  // order keys are distinct (one first row per group)
  for (int k = 2; k <= m; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = tid; i < m; i += blockDim.x) {
        const int ixj = i ^ j;
        if (ixj > i) {
          const unsigned long long x = okey[i], y = okey[ixj];
          if ((x > y) == ((i & k) == 0)) {
            okey[i] = y;
            okey[ixj] = x;
            const uint32_t t = oslot[i];
            oslot[i] = oslot[ixj];
            oslot[ixj] = t;
          }
        }
      }
      __syncthreads();
    }
  for (int i = tid; i < n; i += blockDim.x) {
    ordered[i] = oslot[i];
    firsts[i] = okey[i];
    rows32[i] = (uint32_t)okey[i];
  }
  if (tid == 0) *out = (unsigned long long)n;
}

// the probe and build rows of fused-join order keys (probe row << 32 | build row)
__global__ void split_join_rows_kernel(const unsigned long long* firsts, int64_t n, uint32_t* prow, uint32_t* brow) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    prow[i] = (uint32_t)(firsts[i] >> 32);
    brow[i] = (uint32_t)firsts[i];
  }
}

// exact big integer (signed 64-bit counters of 32-bit limbs, weight
// 2^(32k + lo_exp)) -> correctly rounded double; MAXL bounds n_limbs
template <int MAXL>
__device__ double limbs_to_double(const unsigned long long* acc, int n_limbs, int lo_exp) {
  // normalise to 32-bit digits with a signed top
  uint32_t dig[MAXL + 3];
  long long carry = 0;
  int nd = n_limbs + 3;
  for (int k = 0; k < nd; ++k) {
    __int128 v = (__int128)carry + (k < n_limbs ? (__int128)(long long)acc[k] : 0);
    dig[k] = (uint32_t)(unsigned long long)v;
    carry = (long long)(v >> 32);
  }
  bool neg = carry < 0;
  if (neg) {  // two's complement negate
    unsigned long long c = 1;
    for (int k = 0; k < nd; ++k) {
      unsigned long long t = (unsigned long long)(uint32_t)~dig[k] + c;
      dig[k] = (uint32_t)t;
      c = t >> 32;
    }
  }
  int kt = -1;
  for (int k = nd - 1; k >= 0; --k)
    if (dig[k]) { kt = k; break; }
  if (kt < 0) return 0.0;
  const int sh = __clz(dig[kt]);
  const int top = kt * 32 + 31 - sh;  // highest set bit
  // bits [top - 63, top] as m64 (top at bit 63), and whether any bit below is set
  unsigned __int128 x = ((unsigned __int128)dig[kt] << 64) | ((unsigned __int128)(kt >= 1 ? dig[kt - 1] : 0u) << 32) |
                        (kt >= 2 ? dig[kt - 2] : 0u);
  x <<= sh;
  const unsigned long long m64 = (unsigned long long)(x >> 32);
  bool below = (uint32_t)x != 0;
  for (int k = kt - 3; k >= 0 && !below; --k) below = dig[k] != 0;
  double r;
  if (top <= 52) {
    r = scalbn((double)(m64 >> (63 - top)), lo_exp);
  } else {
    unsigned long long m = m64 >> 11;  // bits [top - 52, top]
    const bool rb = (m64 >> 10) & 1;   // the bit below them
    const bool sticky = (m64 & 0x3FF) != 0 || below;
    if (rb && (sticky || (m & 1))) ++m;  // round half to even
    r = scalbn((double)m, top - 52 + lo_exp);
  }
  return neg ? -r : r;
}

__device__ __forceinline__ __int128 limbs_to_i128(const unsigned long long* acc, int n_limbs) {
  __int128 v = 0;
  for (int k = 0; k < n_limbs; ++k) v += (__int128)(long long)acc[k] << (32 * k);
  return v;
}

struct OutSpec {
  int32_t func;       // PRISM_AGG_*
  int32_t op;         // main op index (-1: group count)
  int32_t op_count;   // op of the non-null count (global AVG) or -1
  int32_t result;     // 0 f64, 1 i64, 2 dec128
  int32_t dec_scale;
  int32_t pad;
  void* out;
};

struct FinalArgs {
  const uint32_t* ordered;
  int64_t n;
  const unsigned long long* gacc;
  int32_t W;
  int32_t n_out;
  OutSpec out[32];
  Op op[MAX_OPS];
  const unsigned long long* dcount;  // [slot * 4 + table]
  int32_t wide;
  int32_t n_wide;
  const unsigned long long* gwide;
  int32_t grouped;                    // grouped path: MIN/MAX of all-NaN stay +-inf
  int64_t total_rows;
};

__global__ void finalize_kernel(FinalArgs f) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < f.n; i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t s = f.ordered[i];
    const unsigned long long* acc = f.gacc + (size_t)s * f.W;
    for (int k = 0; k < f.n_out; ++k) {
      const OutSpec& o = f.out[k];
      unsigned long long cnt = acc[0];
      if (o.op_count >= 0) cnt = acc[f.op[o.op_count].word];
      double r = 0;
      long long ri = 0;
      __int128 rd = 0;
      switch (o.func) {
        case PRISM_AGG_COUNT:
          ri = o.op < -1 ? f.total_rows : (long long)cnt;
          break;
        case PRISM_AGG_COUNT_DISTINCT:
          ri = (long long)f.dcount[(size_t)s * 4 + f.op[o.op].distinct];
          break;
        case PRISM_AGG_SUM: case PRISM_AGG_AVG: {
          const Op& op = f.op[o.op];
          const unsigned long long* w = acc + op.word;
          if (op.kind == O_SUM_F64) {
            int nl = LIMBS, lo = op.lo_exp;
            if (f.wide) {
              w = f.gwide + ((size_t)s * f.n_wide + op.distinct) * (WIDE_LIMBS + 1);
              nl = WIDE_LIMBS;
              lo = WIDE_LO;
            }
            unsigned long long fl = w[nl];
            if (fl & 1 || ((fl & 2) && (fl & 4))) r = __longlong_as_double(0x7ff8000000000000LL);
            else if (fl & 2) r = __longlong_as_double(0x7ff0000000000000LL);
            else if (fl & 4) r = __longlong_as_double((long long)0xfff0000000000000ULL);
            else if (f.wide) r = limbs_to_double<WIDE_LIMBS>(w, nl, lo);
            else r = limbs_to_double<LIMBS>(w, nl, lo);
          } else if (op.kind == O_SUM_INT) {
            r = limbs_to_double<2>(w, 2, 0);
          } else {  // O_SUM_DEC
            rd = limbs_to_i128(w, 4);
            double sc = 1.0;
            for (int q = 0; q < o.dec_scale; ++q) sc *= 10.0;
            r = limbs_to_double<4>(w, 4, 0) / sc;
          }
          if (o.func == PRISM_AGG_AVG) r = cnt > 0 ? r / (double)cnt : 0.0;
          break;
        }
        case PRISM_AGG_MIN: case PRISM_AGG_MAX: {
          const Op& op = f.op[o.op];
          long long key = (long long)acc[op.word];
          bool none = (o.func == PRISM_AGG_MIN) ? key == 0x7fffffffffffffffLL : key == (long long)0x8000000000000000ULL;
          if (cnt == 0) r = 0.0;
          else if (!none) r = from_total_key(key);
          else if (f.grouped) r = o.func == PRISM_AGG_MIN ? __longlong_as_double(0x7ff0000000000000LL)
                                                          : __longlong_as_double((long long)0xfff0000000000000ULL);
          else r = 0.0;
          break;
        }
      }
      if (o.result == 0) static_cast<double*>(o.out)[i] = r;
      else if (o.result == 1) static_cast<long long*>(o.out)[i] = ri;
      else {
        unsigned long long* p = static_cast<unsigned long long*>(o.out) + 2 * i;
        p[0] = (unsigned long long)rd;
        p[1] = (unsigned long long)(rd >> 64);
      }
    }
  }
}

__global__ void narrow_kernel(const unsigned long long* a, int64_t n, uint32_t* b) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = (uint32_t)a[i];
}

// distinct counting: every (group, value) entry adds one to its group
__global__ void distinct_count_kernel(AggArgs a, int table, unsigned long long* dcount) {
  const DistinctTable& t = a.dt[table];
  for (uint64_t e = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; e <= t.mask; e += (uint64_t)gridDim.x * blockDim.x) {
    unsigned long long g = t.slots[2 * e], v = t.slots[2 * e + 1];
    if (g == GEMPTY && v == GEMPTY) continue;
    int64_t s = a.dense ? (int64_t)g : gfind(a, g);
    if (s >= 0) atomicAdd(&dcount[(size_t)s * 4 + table], 1ULL);
  }
}

}  // namespace

// ---------------------------------------------------------------- host ----
namespace {

// register budget of a generated small-groups kernel: it holds TINY_R rows'
// operands per thread (a 128-bit integer and its null flag for integer sums,
// a double or key for the others)
bool tiny_fits_registers(const AggArgs& A) {
  int regs = 0;
  for (int j = 0; j < A.n_ops; ++j)
    regs += TINY_R * (A.op[j].kind == O_SUM_INT || A.op[j].kind == O_SUM_DEC ? 5 : A.op[j].kind == O_NONNULL ? 1 : 3);
  return regs <= 96;
}

// words per group of the small-groups kernel's accumulator columns
int tiny_group_words(const AggArgs& A) {
  int nw = TINY_FIRST_OP_WORD;
  for (int j = 0; j < A.n_ops; ++j) nw += tiny_words(A.op[j].kind);
  return nw;
}

bool int_like(int t) {
  return t == TY_I8 || t == TY_I16 || t == TY_I32 || t == TY_I64 || t == TY_U8 || t == TY_U16 || t == TY_U32 ||
         t == TY_BOOL;
}

struct ProjCol {  // one column of the (virtual) projected schema
  bool is_expr = false;
  int batch_col = -1;
  int expr = -1;
};

struct Plan {
  AggArgs args{};
  std::vector<OutSpec> outs;
  std::vector<int> out_result;
  std::vector<std::string> names;
  std::vector<int> out_types;  // TY_*
  std::vector<int> out_scale;
  int n_distinct = 0;
};

}  // namespace

static __global__ void concat_bits_kernel(const uint8_t* src, int64_t n, int64_t dst_off, uint32_t* dst) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    bool b = src == nullptr || ((src[i >> 3] >> (i & 7)) & 1);
    if (b) {
      int64_t j = dst_off + i;
      atomicOr(&dst[j >> 5], 1u << (j & 31));
    }
  }
}
static __global__ void concat_offsets_kernel(const int32_t* src, int64_t n, int32_t base, int64_t dst_data_off,
                                             int32_t* dst) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] = (int32_t)(src[i] - base + dst_data_off);
}

// Concatenation of one column's parts (same type) into a new column.
ColP concat_columns(Ctx& ctx, const std::vector<const Column*>& parts) {
  const Column& f = *parts[0];
  int64_t n = 0, bytes = 0;
  bool any_valid = false;
  for (auto* p : parts) {
    n += p->length;
    bytes += p->data_bytes;
    any_valid |= p->validity != nullptr;
    if (p->type != f.type) fail(PRISM_ERR_SCHEMA_MISMATCH, "batches disagree on column type");
    if (f.type == TY_DICT && p->dict_fingerprint != f.dict_fingerprint)
      fail(PRISM_ERR_UNSUPPORTED_AGGREGATION, "dictionary group keys with different dictionaries across batches");
  }
  ColP out;
  if (f.type == TY_UTF8) out = make_utf8_column(ctx, f.name, n, bytes, any_valid);
  else out = make_column(ctx, f.type == TY_DICT ? f.index_type : f.type, f.name, n, any_valid);
  out->type = f.type;
  out->index_type = f.index_type;
  out->nullable = f.nullable;
  out->precision = f.precision;
  out->scale = f.scale;
  out->dict = f.dict;
  out->dict_fingerprint = f.dict_fingerprint;
  if (any_valid) PRISM_CUDA(cudaMemsetAsync(out->validity, 0, (size_t)(n + 31) / 8 + 4, ctx.stream));
  if (f.type == TY_BOOL) PRISM_CUDA(cudaMemsetAsync(out->values, 0, (size_t)(n + 31) / 8 + 4, ctx.stream));
  int64_t off = 0, doff = 0;
  for (auto* p : parts) {
    int g = grid_for(ctx, std::max<int64_t>(p->length, 1), 256);
    if (any_valid && p->length) {
      concat_bits_kernel<<<g, 256, 0, ctx.stream>>>(p->validity, p->length, off, reinterpret_cast<uint32_t*>(out->validity));
      ctx.check_launch("concat_bits_kernel");
    }
    if (f.type == TY_UTF8) {
      concat_offsets_kernel<<<g, 256, 0, ctx.stream>>>(p->offsets, p->length, p->data_base, doff, out->offsets + off);
      ctx.check_launch("concat_offsets_kernel");
      if (p->data_bytes)
        PRISM_CUDA(cudaMemcpyAsync(out->data + doff, p->data, p->data_bytes, cudaMemcpyDeviceToDevice, ctx.stream));
      doff += p->data_bytes;
    } else if (f.type == TY_BOOL) {
      if (p->length) {
        concat_bits_kernel<<<g, 256, 0, ctx.stream>>>(static_cast<const uint8_t*>(p->values), p->length, off,
                                                      reinterpret_cast<uint32_t*>(out->values));
        ctx.check_launch("concat_bits_kernel(bool)");
      }
    } else if (f.type != TY_NULL) {
      int w = width_of(f.type == TY_DICT ? f.index_type : f.type);
      if (p->length)
        PRISM_CUDA(cudaMemcpyAsync(static_cast<uint8_t*>(out->values) + off * w, p->values, p->length * w,
                                   cudaMemcpyDeviceToDevice, ctx.stream));
    }
    off += p->length;
  }
  return out;
}

namespace {

int result_type(int func) {
  return (func == PRISM_AGG_COUNT || func == PRISM_AGG_COUNT_DISTINCT) ? TY_I64 : TY_F64;
}

}  // namespace

Batch aggregate(Ctx& ctx, const std::vector<const Batch*>& batches_in, const prism_agg_config& cfg,
                const prism_predicate* pred, const int32_t* cols, int n_cols, const prism_expr* exprs,
                int n_exprs, int arith_mode, bool fused, const AggTuning& tune, const JoinAggSpec* join) {
  // fused join: each probe batch is seen as the joined batch [probe columns,
  // build columns] with the probe batch's rows; build-side columns are read
  // at the matched build row inside the kernel
  const int n_probe_cols = join ? (int)batches_in.at(0)->cols.size() : -1;
  auto fused_fail = [](const std::string& why) {
    fail(PRISM_ERR_INVALID_ARGUMENT, why + " is not supported in the fused path");
  };
  std::vector<Batch> joined;
  std::vector<const Batch*> joined_ptrs;
  if (join) {
    if (!fused) fail(PRISM_ERR_INTERNAL, "fused join aggregation without a projection");
    if (!jit_enabled()) fused_fail("a join without run-time compilation");
    // build columns named like a probe column are `<name>_right` in the
    // joined schema, as the joined batch names them (hash_join.rs:436-447)
    std::vector<ColP> bcols;
    for (auto& c : join->table->build.cols) {
      bool clash = false;
      for (auto& pc : batches_in[0]->cols) clash |= pc->name == c->name;
      if (!clash) {
        bcols.push_back(c);
        continue;
      }
      auto r = std::make_shared<Column>(*c);
      r->name = c->name + "_right";
      bcols.push_back(r);
    }
    joined.reserve(batches_in.size());
    for (auto* p : batches_in) {
      Batch v;
      v.rows = p->rows;
      v.cols = p->cols;
      for (auto& c : bcols) v.cols.push_back(c);
      joined.push_back(std::move(v));
    }
    for (auto& v : joined) joined_ptrs.push_back(&v);
  }
  const std::vector<const Batch*>& batches = join ? joined_ptrs : batches_in;
  for (int i = 0; i < cfg.n_aggs; ++i)
    if (cfg.aggs[i].func < PRISM_AGG_SUM || cfg.aggs[i].func > PRISM_AGG_COUNT_DISTINCT)
      fail(PRISM_ERR_UNSUPPORTED_AGGREGATION, "unknown aggregate function");
  if (cfg.n_aggs > 32) fail(PRISM_ERR_INVALID_ARGUMENT, "at most 32 aggregates per call");
  if (cfg.n_group_by > MAX_GCOLS) fail(PRISM_ERR_INVALID_ARGUMENT, "at most 8 group-by columns");
  // EXACT also covers the materialized fallback of the fused call (fused =
  // false with the caller's mode); plain hash_aggregate passes F64
  const bool exact = arith_mode == PRISM_ARITH_EXACT;
  int64_t total_rows = 0;
  for (auto* b : batches) total_rows += b->rows;
  bool any_rows = total_rows > 0;
  // the accumulators are signed 64-bit counters of 32-bit limbs, added to
  // without carry normalisation: exact for up to 2^31 - 1 rows per call
  if (total_rows > (int64_t)INT32_MAX)
    fail(PRISM_ERR_INVALID_ARGUMENT, "aggregation input exceeds 2^31-1 rows per call");

  // projected schema description
  std::vector<ProjCol> proj;
  Program types;  // compiled against the first batch (types only)
  if (fused) {
    if (batches.empty()) fail(PRISM_ERR_INVALID_ARGUMENT, "fused aggregation needs at least one batch");
    for (int i = 0; i < n_cols; ++i) {
      if (cols[i] < 0 || cols[i] >= (int)batches[0]->cols.size()) fail(PRISM_ERR_INVALID_ARGUMENT, "projected column out of range");
      proj.push_back({false, cols[i], -1});
    }
    types = compile_program(*batches[0], pred, exprs, n_exprs, arith_mode);
    for (int e = 0; e < n_exprs; ++e) {
      const CompiledExpr& ce = types.exprs[e];
      if (ce.kind == EK_COLUMN) proj.push_back({false, ce.column, -1});
      else proj.push_back({true, -1, e});
    }
  } else if (!batches.empty()) {
    for (int i = 0; i < (int)batches[0]->cols.size(); ++i) proj.push_back({false, i, -1});
  }
  auto proj_type = [&](int idx) -> int {
    const ProjCol& pc = proj[idx];
    if (!pc.is_expr) return batches[0]->cols[pc.batch_col]->type;
    return types.exprs[pc.expr].out_type;
  };
  auto proj_name = [&](int idx) -> std::string {
    const ProjCol& pc = proj[idx];
    if (!pc.is_expr) return fused && idx >= n_cols ? "expr_" + std::to_string(pc.expr >= 0 ? pc.expr : idx - n_cols)
                                                   : batches[0]->cols[pc.batch_col]->name;
    return "expr_" + std::to_string(pc.expr);
  };

  const bool global = cfg.n_group_by == 0 && !exact;
  // ------------------------------------------------------- empty input --
  if (!any_rows) {
    Batch out;
    out.rows = 0;
    if (!batches.empty()) {
      for (int g = 0; g < cfg.n_group_by; ++g) {
        int idx = cfg.group_by[g];
        if (idx < 0 || idx >= (int)proj.size()) fail(PRISM_ERR_INVALID_ARGUMENT, "group-by column out of range");
        auto c = std::make_shared<Column>();
        if (!proj[idx].is_expr) {
          const Column& src = *batches[0]->cols[proj[idx].batch_col];
          c->type = src.type;
          c->index_type = src.index_type;
          c->dict = src.dict;
          c->name = src.name;
          c->nullable = src.nullable;
          c->precision = src.precision;
          c->scale = src.scale;
        } else {
          c->type = proj_type(idx);
          c->name = proj_name(idx);
        }
        if (c->type == TY_DICT && !c->dict) fail(PRISM_ERR_INTERNAL, "dictionary without values");
        out.cols.push_back(c);
      }
    } else if (cfg.n_group_by > 0) {
      // the reference builds the empty result against the aggregate fields only
      for (int g = 0; g < cfg.n_group_by; ++g) {
        int idx = cfg.group_by[g];
        if (idx < 0 || idx >= cfg.n_aggs) fail(PRISM_ERR_INVALID_ARGUMENT, "group-by column out of range");
        auto c = std::make_shared<Column>();
        c->type = result_type(cfg.aggs[idx].func);
        c->name = cfg.aggs[idx].output_name ? cfg.aggs[idx].output_name : "";
        out.cols.push_back(c);
      }
    }
    for (int i = 0; i < cfg.n_aggs; ++i) {
      auto c = std::make_shared<Column>();
      c->type = result_type(cfg.aggs[i].func);
      c->name = cfg.aggs[i].output_name ? cfg.aggs[i].output_name : "";
      out.cols.push_back(c);
    }
    return out;
  }

  // ------------------------------------------------------- plan the ops --
  const Batch& ref = **std::find_if(batches.begin(), batches.end(), [](const Batch* b) { return b->rows > 0; });
  for (int g = 0; g < cfg.n_group_by; ++g)
    if (cfg.group_by[g] < 0 || cfg.group_by[g] >= (int)proj.size()) fail(PRISM_ERR_INVALID_ARGUMENT, "group-by column out of range");
  for (int i = 0; i < cfg.n_aggs; ++i) {
    bool count_star_global = global && cfg.aggs[i].func == PRISM_AGG_COUNT && cfg.aggs[i].column >= (int)proj.size();
    if (!count_star_global && (cfg.aggs[i].column < 0 || cfg.aggs[i].column >= (int)proj.size()))
      fail(PRISM_ERR_INVALID_ARGUMENT, "aggregate column out of range");
  }
  for (int g = 0; g < cfg.n_group_by; ++g)
    if (proj[cfg.group_by[g]].is_expr) fail(PRISM_ERR_INVALID_ARGUMENT, "grouping by a computed expression is not supported in the fused path");

  // sources are defined against a per-batch program; record them symbolically
  struct SrcSym { int kind; int proj_idx; };
  std::vector<SrcSym> srcs;
  auto src_of = [&](int kind, int pidx) {
    for (size_t s = 0; s < srcs.size(); ++s)
      if (srcs[s].kind == kind && srcs[s].proj_idx == pidx) return (int)s;
    srcs.push_back({kind, pidx});
    if (srcs.size() > (size_t)MAX_SRC) fail(PRISM_ERR_INVALID_ARGUMENT, "too many distinct aggregate inputs");
    return (int)srcs.size() - 1;
  };
  Plan P;
  AggArgs& A = P.args;
  int W = 1;  // word 0: row count
  std::vector<unsigned long long> winit(1, 0);
  std::vector<int> wkind(1, W_ADD);
  auto add_words = [&](int n, unsigned long long init, int kind) {
    int w = W;
    for (int i = 0; i < n; ++i) { winit.push_back(init); wkind.push_back(kind); }
    W += n;
    return w;
  };
  auto new_op = [&](int kind, int src) -> int {
    for (int j = 0; j < A.n_ops; ++j)
      if (A.op[j].kind == kind && A.op[j].src == src) return j;
    if (A.n_ops >= MAX_OPS) fail(PRISM_ERR_INVALID_ARGUMENT, "too many aggregate accumulators");
    Op o{};
    o.kind = kind;
    o.src = src;
    o.lo_exp = -128;
    switch (kind) {
      case O_SUM_F64: o.word = add_words(LIMBS, 0, W_ADD); add_words(1, 0, W_OR); break;
      case O_SUM_INT: o.word = add_words(2, 0, W_ADD); break;
      case O_SUM_DEC: o.word = add_words(4, 0, W_ADD); break;
      case O_MIN: o.word = add_words(1, 0x7fffffffffffffffULL, W_MIN); break;
      case O_MAX: o.word = add_words(1, 0x8000000000000000ULL, W_MAX); break;
      case O_NONNULL: o.word = add_words(1, 0, W_ADD); break;
      case O_DISTINCT: o.word = 0; o.distinct = P.n_distinct++; break;
    }
    if (P.n_distinct > 4) fail(PRISM_ERR_INVALID_ARGUMENT, "at most 4 COUNT DISTINCT per call");
    A.op[A.n_ops] = o;
    return A.n_ops++;
  };
  for (int i = 0; i < cfg.n_aggs; ++i) {
    const prism_agg_expr& ag = cfg.aggs[i];
    OutSpec o{};
    o.func = ag.func;
    o.op = -1;
    o.op_count = -1;
    o.result = (ag.func == PRISM_AGG_COUNT || ag.func == PRISM_AGG_COUNT_DISTINCT) ? 1 : 0;
    int out_type = result_type(ag.func);
    int out_scale = 0;
    bool count_star_global = global && ag.func == PRISM_AGG_COUNT && ag.column >= (int)proj.size();
    int ty = count_star_global ? TY_NULL : proj_type(ag.column);
    bool numeric = int_like(ty) || ty == TY_U64 || ty == TY_F32 || ty == TY_F64 || ty == TY_DEC128;
    bool is_expr = !count_star_global && proj[ag.column].is_expr;
    int ek = is_expr ? types.exprs[proj[ag.column].expr].kind : -1;
    if (is_expr && ek != EK_F64 && ek != EK_DEC)
      fail(PRISM_ERR_INVALID_ARGUMENT, "aggregating a literal/cast/string expression is not supported in the fused path");
    switch (ag.func) {
      case PRISM_AGG_COUNT:
        if (count_star_global) o.op = -2;
        else if (global) o.op_count = new_op(O_NONNULL, src_of(S_VALID, ag.column));
        break;
      case PRISM_AGG_COUNT_DISTINCT:
        if (is_expr) fail(PRISM_ERR_INVALID_ARGUMENT, "COUNT DISTINCT of a computed expression is not supported");
        o.op = new_op(O_DISTINCT, src_of(S_VALID, ag.column));
        break;
      case PRISM_AGG_SUM: case PRISM_AGG_AVG: {
        if (!numeric && !is_expr)
          fail(PRISM_ERR_UNSUPPORTED_AGGREGATION, "numeric aggregate over a non-numeric column '" + proj_name(ag.column) + "'");
        int kind, sk;
        if (is_expr) {
          bool dec = ek == EK_DEC;
          kind = dec ? O_SUM_DEC : O_SUM_F64;
          sk = dec ? S_EXPR_I128 : S_EXPR_F64;
          if (dec) out_scale = types.exprs[proj[ag.column].expr].scale;
        } else if (ty == TY_DEC128 && exact) {
          kind = O_SUM_DEC;
          sk = S_COL_I128;
          out_scale = batches[0]->cols[proj[ag.column].batch_col]->scale;
        } else if (int_like(ty) || ty == TY_I64) {
          kind = O_SUM_INT;
          sk = S_COL_INT;
        } else {
          kind = O_SUM_F64;
          sk = S_COL_F64;
        }
        o.op = new_op(kind, src_of(sk, ag.column));
        o.dec_scale = out_scale;
        if (kind == O_SUM_DEC && ag.func == PRISM_AGG_SUM) { o.result = 2; out_type = TY_DEC128; }
        if (global) o.op_count = new_op(O_NONNULL, src_of(S_VALID, ag.column));
        break;
      }
      case PRISM_AGG_MIN: case PRISM_AGG_MAX: {
        if (!numeric && !is_expr)
          fail(PRISM_ERR_UNSUPPORTED_AGGREGATION, "numeric aggregate over a non-numeric column '" + proj_name(ag.column) + "'");
        int sk = is_expr ? S_EXPR_F64 : S_COL_F64;
        if (is_expr && ek == EK_DEC) fail(PRISM_ERR_INVALID_ARGUMENT, "MIN/MAX of an exact expression is not supported");
        o.op = new_op(ag.func == PRISM_AGG_MIN ? O_MIN : O_MAX, src_of(sk, ag.column));
        if (global) o.op_count = new_op(O_NONNULL, src_of(S_VALID, ag.column));
        break;
      }
    }
    P.outs.push_back(o);
    P.names.push_back(ag.output_name ? ag.output_name : "");
    P.out_types.push_back(out_type);
    P.out_scale.push_back(out_scale);
  }
  if (W > MAX_W) fail(PRISM_ERR_INVALID_ARGUMENT, "aggregate state exceeds 64 words per group");
  A.W = W;
  for (int w = 0; w < W; ++w) { A.winit[w] = winit[w]; A.wkind[w] = wkind[w]; }
  A.skip_nulls = global ? 1 : 0;
  A.count_rows = global ? 0 : 1;
  A.n_src = (int)srcs.size();

  // ----------------------------------------------------- group identity --
  bool dense = false;
  int64_t G = 1;
  std::vector<int> gbatch_cols;
  for (int g = 0; g < cfg.n_group_by; ++g) gbatch_cols.push_back(proj[cfg.group_by[g]].batch_col);
  if (join) {
    // hashed groups (no group columns: every row hashes to one group)
    for (auto& o : P.outs)
      if (o.op == -2) fused_fail("COUNT(*) over a join");
  } else if (cfg.n_group_by == 0) {
    dense = true;
    G = 1;
  } else {
    bool all_dict = true;
    for (int bc : gbatch_cols) {
      const Column& c = *ref.cols[bc];
      if (c.type != TY_DICT) { all_dict = false; break; }
      for (auto* b : batches)
        if (b->rows && b->cols[bc]->dict_fingerprint != c.dict_fingerprint) all_dict = false;
    }
    if (all_dict) {
      // one id per dictionary entry, plus one for null only when some batch
      // has nulls in the column (so null-free keys stay compact)
      std::vector<int64_t> card(cfg.n_group_by);
      int64_t prod = 1;
      for (int k = 0; k < cfg.n_group_by; ++k) {
        int bc = gbatch_cols[k];
        bool nulls = false;
        for (auto* b : batches)
          if (b->rows && b->cols[bc]->validity) nulls = true;
        card[k] = ref.cols[bc]->dict->length + (nulls ? 1 : 0);
        if (card[k] < 1 || prod * card[k] > 4096) { prod = -1; break; }
        prod *= card[k];
      }
      if (prod > 0) {
        dense = true;
        G = prod;
        int64_t stride = 1;
        for (int k = cfg.n_group_by - 1; k >= 0; --k) {
          const Column& c = *ref.cols[gbatch_cols[k]];
          A.dstride[k] = stride;
          A.dnull[k] = c.dict->length;
          stride *= card[k];
        }
      }
    }
  }
  A.dense = dense ? 1 : 0;
  A.G = G;

  // ---------------------------------------------------------- run it ----
  const int block = std::min(512, std::max(64, tune.block));
  int smem_optin = 0;
  PRISM_CUDA(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, ctx.device));
  size_t smem_budget = (size_t)std::min(smem_optin - 4096, 200 * 1024);
  int sd = 0, ss_log2 = 0;
  size_t smem = 0;
  if (dense) {
    smem = (size_t)G * 8 + (size_t)G * W * 8;
    if (smem > smem_budget) { smem = 0; }  // dense but too wide: global atomics only
  } else {
    sd = std::max(0, tune.smem_groups);
    while (sd > 0) {
      ss_log2 = 1;
      while ((1 << ss_log2) < 2 * sd) ++ss_log2;
      smem = (size_t)(1 << ss_log2) * 8 + (size_t)sd * 16 + (size_t)sd * W * 8 + (size_t)(1 << ss_log2) * 4;
      if (smem <= smem_budget) break;
      sd /= 2;
    }
    if (sd == 0) { ss_log2 = 0; smem = 0; }
  }
  A.sd = sd;
  A.ss_log2 = ss_log2;
  A.use_smem = smem > 0 ? 1 : 0;
  PRISM_CUDA(cudaFuncSetAttribute(agg_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(smem, 1)));

  // few dense groups: a generated kernel with per-thread register
  // accumulators (tiny_body), sized to the exact group and op counts
  bool any_f64 = false;
  for (int j = 0; j < A.n_ops; ++j) any_f64 |= A.op[j].kind == O_SUM_F64;
  bool tiny = dense && G <= 8 && P.n_distinct == 0 && A.n_ops >= 1 && A.n_ops <= 8 &&
              tiny_fits_registers(A) && (G + 1) * tiny_group_words(A) <= TINY_MAX_WORDS && jit_enabled();
  // hashed groups: a generated kernel whose per-block table slots own their
  // accumulator words (hash_body); the largest power-of-two table up to
  // 2 x smem_groups slots that fits the block's shared memory
  int hss_log2 = 0;
  size_t hsmem = 0;
  if (!dense && P.n_distinct == 0 && A.n_ops >= 1 && A.n_ops <= 8 && tiny_fits_registers(A) && jit_enabled()) {
    // a fused join waits on dependent loads per row: a smaller table (half
    // a block's share of the SM) keeps two blocks resident per SM
    const size_t hbudget = join ? (size_t)smem_optin / std::max(1, tune.join_min_blocks) - TINY_MAX_COLS * sizeof(DCol) - 1024
                                : (size_t)smem_optin - TINY_MAX_COLS * sizeof(DCol) - 1024;
    for (int l = join ? tune.join_table_log2 : 12; l >= 8; --l) {
      if ((1 << l) > 2 * std::max(128, tune.smem_groups)) continue;
      if (((size_t)(2 + W) * 8 << l) <= hbudget) {
        hss_log2 = l;
        hsmem = (size_t)(2 + W) * 8 << l;
        break;
      }
    }
  }
  if (join && !hss_log2) fused_fail("this aggregate list over a join");
  uint64_t gcap = dense ? (uint64_t)G : std::max<uint64_t>(1024, next_pow2((uint64_t)std::min<int64_t>(total_rows, 1 << 16) * 2));
  int dist_log2 = 0;
  // fused join: device views of each probe batch's key columns
  std::vector<MemP> jpk_mem;
  std::vector<const DCol*> jpk_dev;
  if (join) {
    if (total_rows >= (int64_t)UINT32_MAX) fused_fail("a join over 2^32 probe rows");
    if (join->table->has_dups) {
      // repeated build keys: a probe row can join several build rows, so
      // bound the joined rows (not the probe rows) by the accumulators' limit
      int64_t joined = 0;
      for (auto* pb : batches_in) joined += probe_count(ctx, *join->table, *pb, join->probe_keys, JoinTuning{});
      if (joined > (int64_t)INT32_MAX) fail(PRISM_ERR_INVALID_ARGUMENT, "aggregation input exceeds 2^31-1 joined rows per call");
    }
    for (auto* pb : batches_in) {
      std::vector<DCol> v;
      for (int k : join->probe_keys) v.push_back(pb->cols.at(k)->view());
      MemP m = ctx.alloc(v.size() * sizeof(DCol));
      ctx.h2d_staged(m->ptr, v.data(), v.size() * sizeof(DCol));
      jpk_dev.push_back(static_cast<const DCol*>(m->ptr));
      jpk_mem.push_back(m);
    }
  }
  for (int attempt = 0; attempt < 40; ++attempt) {
    MemP mkeys, mfirst, macc, mmax;
    uint64_t nslots = dense ? gcap : gcap + 1;
    A.gcap = gcap;
    A.gmask = dense ? 0 : gcap - 1;
    A.gshift = dense ? 0 : 64 - (63 - __builtin_clzll(gcap));
    A.gkeys = dense ? nullptr : ctx.alloc_t<unsigned long long>(nslots, mkeys);
    A.gfirst = ctx.alloc_t<unsigned long long>(nslots, mfirst);
    A.gacc = ctx.alloc_t<unsigned long long>(nslots * W, macc);
    A.maxexp = ctx.alloc_t<int>(MAX_OPS, mmax);
    MemP mwide;
    if (A.wide) {
      A.gwide = ctx.alloc_t<unsigned long long>(nslots * A.n_wide * (WIDE_LIMBS + 1), mwide);
      PRISM_CUDA(cudaMemsetAsync(A.gwide, 0, nslots * A.n_wide * (WIDE_LIMBS + 1) * 8, ctx.stream));
    }
    // hashed groups: ginsert lists the slots it creates (the small-groups
    // ordering reads that list instead of scanning the table)
    MemP mnew, mnewc, msmall;
    A.gnew = dense ? nullptr : ctx.alloc_t<uint32_t>(nslots, mnew);
    A.gnew_count = dense ? nullptr : ctx.alloc_t<unsigned long long>(1, mnewc);
    init_table_kernel<<<grid_for(ctx, (int64_t)(nslots * std::max(W, 1)), 256), 256, 0, ctx.stream>>>(A, (int64_t)nslots);
    ctx.check_launch("init_table_kernel");
    std::vector<MemP> dmem;
    for (int t = 0; t < P.n_distinct; ++t) {
      if (!dist_log2) dist_log2 = std::max(10, 64 - __builtin_clzll((uint64_t)std::max<int64_t>(total_rows, 1) * 2));
      uint64_t dcap = 1ULL << dist_log2;
      MemP md = ctx.alloc(dcap * 16);
      PRISM_CUDA(cudaMemsetAsync(md->ptr, 0xff, dcap * 16, ctx.stream));
      A.dt[t].slots = static_cast<unsigned long long*>(md->ptr);
      A.dt[t].mask = dcap - 1;
      dmem.push_back(md);
    }
    A.err = ctx.d_err;
    uint64_t row_base = 0;
    std::vector<Program> progs;
    progs.reserve(batches.size());
    std::vector<MemP> split_mem;  // per-batch match words of the split join, alive until the kernels ran
    for (auto* bp : batches) {
      const Batch& b = *bp;
      if (b.rows == 0) continue;
      // per-batch program: filter + expressions + source/group column slots
      progs.push_back(fused ? compile_program(b, pred, exprs, n_exprs, arith_mode) : Program{});
      Program& pg = progs.back();
      AggArgs a = A;
      a.n = b.rows;
      a.row_base = row_base;
      a.has_filter = fused && pg.has_filter;
      a.filter = pg.filter;
      for (int k = 0; k < cfg.n_group_by; ++k) a.gcol[k] = pg.slot_of(gbatch_cols[k]);
      a.n_gcols = cfg.n_group_by;
      for (size_t s = 0; s < srcs.size(); ++s) {
        const ProjCol& pc = proj[srcs[s].proj_idx < (int)proj.size() ? srcs[s].proj_idx : 0];
        Src sr{};
        sr.kind = srcs[s].kind;
        if (!pc.is_expr) {
          sr.col = pg.slot_of(pc.batch_col);
        } else {
          const CompiledExpr& ce = pg.exprs[pc.expr];
          sr.begin = ce.begin;
          sr.end = ce.end;
          sr.kind = ce.kind == EK_DEC ? S_EXPR_I128 : S_EXPR_F64;
          if (srcs[s].kind == S_VALID) sr.kind = S_EXPR_F64;
        }
        a.src[s] = sr;
      }
      int grid = (int)std::min<int64_t>(ceil_div(b.rows, block), (int64_t)ctx.sm_count * std::max(1, tune.blocks_per_sm));
      const void* jk = nullptr;
      if (tiny) {
        jk = jit_plan_kernel(pg, b, a, {(int64_t)G, any_f64 ? 1 : 0}, "prism_tiny_agg",
                             [&] { return jit_tiny_agg_source(pg, b, a, (int)G, any_f64); });
      }
      const void* hk = nullptr;
      if (join) {
        const JoinTable& t = *join->table;
        a.join = 1;
        a.jfast = t.int64_fast ? 1 : 0;
        a.jslots = t.slots ? static_cast<const ulonglong2*>(t.slots->ptr) : nullptr;
        a.jshift = 64 - t.log2cap;
        a.jmask = t.capacity - 1;
        a.jcap = t.capacity;
        a.jdup = t.dup_rows ? static_cast<const uint32_t*>(t.dup_rows->ptr) : nullptr;
        a.jn_dup = t.n_dup_rows;
        a.jdense = t.dense ? static_cast<const uint32_t*>(t.dense_rows->ptr) : nullptr;
        a.jdmin = t.dmin;
        a.jdrange = t.drange;
        a.jpk = jpk_dev[&b - &joined[0]];
        a.jbk = static_cast<const DCol*>(t.key_views_dev->ptr);
        a.jkrec = t.key_records ? static_cast<const ulonglong2*>(t.key_records->ptr) : nullptr;
        // the entries' lookup reads the probe key's bytes directly: a Utf8
        // (not dictionary) probe key
        const bool ent = t.key_entries && join->probe_keys.size() == 1 &&
                         b.cols[join->probe_keys[0]]->type == TY_UTF8;
        a.jent = ent ? static_cast<const ulonglong2*>(t.key_entries->ptr) : nullptr;
        a.jent_col = ent && t.entry_col >= 0 ? n_probe_cols + t.entry_col : -1;
        a.jmatch = nullptr;
        a.jinl = nullptr;
        a.jinl_w = 0;
        // PRISM_JOIN_KEY_WORDS=0: the probe key's bytes compared by the byte loops
        a.jkw = !ent && t.key_records && join_key_words_on() && join->probe_keys.size() == 1 &&
                        b.cols[join->probe_keys[0]]->type == TY_UTF8
                    ? 1
                    : 0;
        if (join_split() && join->probe_keys.size() == 1) {
          // split: the lookups by match_rows_kernel (many rows in flight),
          // then the fused kernel aggregates from its per-row match words
          MemP mm = ctx.alloc((size_t)b.rows * 4);
          int iw = 0;
          if (join->inline_col >= 0) {
            const Column& ic = *t.build.cols[join->inline_col];
            iw = width_of(ic.type == TY_DICT ? ic.index_type : ic.type);
          }
          MemP mi = iw ? ctx.alloc((size_t)b.rows * iw) : MemP();
          if (match_rows_utf8(ctx, t, *b.cols[join->probe_keys[0]], b.rows, join->inline_col,
                              static_cast<uint32_t*>(mm->ptr), mi ? mi->ptr : nullptr)) {
            a.jent = nullptr;  // the lookup is done; the kernel reads the match words
            a.jkw = 0;
            a.jmatch = static_cast<const uint32_t*>(mm->ptr);
            a.jinl = mi ? mi->ptr : nullptr;
            a.jinl_w = iw;
            a.jent_col = join->inline_col >= 0 ? n_probe_cols + join->inline_col : -1;
            split_mem.push_back(mm);
            if (mi) split_mem.push_back(mi);
          }
        }
        a.jnkeys = (int)join->probe_keys.size();
        a.n_cols = (int)pg.cols.size();
        if (A.wide) fused_fail("a Float64 sum beyond the 192-bit window over a join");
        JoinKernelShape shape;
        shape.block = tune.join_block;
        shape.min_blocks = tune.join_min_blocks;
        shape.rows = tune.join_rows;
        hk = jit_plan_kernel(pg, b, a, {n_probe_cols, shape.block, shape.min_blocks, shape.rows, shape.hash_block},
                             "prism_join_agg", [&] { return jit_hash_agg_source(pg, b, a, n_probe_cols, shape); });
        if (!hk) fused_fail("this projection over a join");
      } else if (!jk && hss_log2 && !A.wide) {
        a.n_cols = (int)pg.cols.size();
        JoinKernelShape shape;
        shape.hash_block = tune.hash_block;
        hk = jit_plan_kernel(pg, b, a, {-1, shape.block, shape.min_blocks, shape.rows, shape.hash_block},
                             "prism_hash_agg", [&] { return jit_hash_agg_source(pg, b, a, -1, shape); });
      }
      // the program's device copy: its upload waits for the stream (the
      // previous batch's kernel), so the kernel source above was generated
      // while that kernel ran
      upload_program(ctx, pg, b);
      a.pn = pg.d_pnodes;
      a.en = pg.d_enodes;
      a.cl = pg.d_clauses;
      a.cols = pg.d_cols;
      if (hk) {
        a.ss_log2 = hss_log2;
        PRISM_CUDA(cudaFuncSetAttribute(hk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)hsmem));
        int per_sm = 0;
        const int hblock = join ? tune.join_block : tune.hash_block;
        PRISM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, hk, hblock, hsmem));
        int hgrid = (int)std::min<int64_t>(ceil_div(b.rows, (int64_t)hblock * TINY_R * 4),
                                           (int64_t)ctx.sm_count * std::max(1, per_sm));
        void* params[] = {&a};
        KernelTimer kt(ctx, join ? "join_agg_jit" : "agg_hash_jit");
        PRISM_CUDA(cudaLaunchKernel(hk, dim3(hgrid), dim3(hblock), params, hsmem, ctx.stream));
      } else if (jk) {
        a.n_cols = (int)pg.cols.size();
        const int words = (int)(G + 1) * tiny_group_words(A), tblock = tiny_block(words);
        size_t tsmem = (size_t)words * tblock * 8;
        PRISM_CUDA(cudaFuncSetAttribute(jk, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)tsmem));
        // as many blocks as fit on every SM at once (registers and shared
        // memory decide); fewer for small inputs (each thread takes at
        // least 8 x TINY_R rows)
        int per_sm = 0;
        PRISM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, jk, tblock, tsmem));
        int tgrid = (int)std::min<int64_t>(ceil_div(b.rows, (int64_t)tblock * TINY_R * 8),
                                           (int64_t)ctx.sm_count * std::max(1, per_sm));
        void* params[] = {&a};
        KernelTimer kt(ctx, "agg_tiny_jit");
        PRISM_CUDA(cudaLaunchKernel(jk, dim3(tgrid), dim3(tblock), params, tsmem, ctx.stream));
      } else {
        KernelTimer kt(ctx, "agg_kernel");
        agg_kernel<<<grid, block, smem, ctx.stream>>>(a);
      }
      ctx.check_launch("agg_kernel");
      row_base += (uint64_t)b.rows;
    }
    // few groups: ordered by one block now, the count read back together
    // with the error word (one synchronisation)
    const bool small_try = total_rows < (int64_t)UINT32_MAX && (!dense || (int64_t)nslots <= SMALL_GROUPS);
    uint32_t* s_ordered = nullptr;
    uint32_t* s_rows = nullptr;
    unsigned long long* s_firsts = nullptr;
    unsigned long long* s_out = nullptr;
    MemP mso, msr, msf;
    if (small_try) {
      s_ordered = ctx.alloc_t<uint32_t>(SMALL_GROUPS, mso);
      s_rows = ctx.alloc_t<uint32_t>(SMALL_GROUPS, msr);
      s_firsts = ctx.alloc_t<unsigned long long>(SMALL_GROUPS, msf);
      s_out = ctx.alloc_t<unsigned long long>(1, msmall);
      PRISM_CUDA(cudaFuncSetAttribute(small_order_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMALL_SMEM));
      small_order_kernel<<<1, 1024, SMALL_SMEM, ctx.stream>>>(A.gfirst, A.gnew, A.gnew_count,
                                                              dense ? (int64_t)nslots : 0, dense ? -1 : (int64_t)gcap,
                                                              s_ordered, s_firsts, s_rows, s_out);
      ctx.check_launch("small_order_kernel");
    }
    // the group count into the context's page-locked words, read after the
    // error word's synchronisation (one round trip for both)
    unsigned long long* h_small = reinterpret_cast<unsigned long long*>(reinterpret_cast<char*>(ctx.h_err) + 64);
    if (small_try) PRISM_CUDA(cudaMemcpyAsync(h_small, s_out, 8, cudaMemcpyDeviceToHost, ctx.stream));
    uint32_t derr = ctx.take_device_errors();
    const unsigned long long small_n = small_try ? *h_small : ~0ULL;
    if (derr & DERR_TIMEOUT) fail(PRISM_ERR_TIMEOUT, "aggregation wait timed out");
    if (derr & DERR_CORRUPT) fail(PRISM_ERR_INTERNAL, "join table inconsistent (build rows changed while it was built?)");
    if (derr & DERR_TABLE_FULL) {
      if (P.n_distinct) dist_log2 += 1;
      if (!dense) gcap *= 2;
      continue;
    }
    if (derr & DERR_OVERFLOW) {
      // a Float64 value left the 192-bit window: accumulate every Float64
      // SUM over the whole double range instead (global accumulators)
      if (A.wide) fail(PRISM_ERR_INTERNAL, "Float64 sum overflow in wide mode");
      A.wide = 1;
      A.n_wide = 0;
      for (int j = 0; j < A.n_ops; ++j)
        if (A.op[j].kind == O_SUM_F64) A.op[j].distinct = A.n_wide++;
      A.use_smem = 0;
      smem = 0;
      tiny = false;
      continue;
    }
    if (derr & DERR_RANGE) fail(PRISM_ERR_EXECUTION, "decimal overflow in exact arithmetic");

    // ------------------------------------------------------ finalize ----
    MemP mdc;
    unsigned long long* dcount = nullptr;
    if (P.n_distinct) {
      dcount = ctx.alloc_t<unsigned long long>(nslots * 4, mdc);
      PRISM_CUDA(cudaMemsetAsync(dcount, 0, nslots * 32, ctx.stream));
      for (int t = 0; t < P.n_distinct; ++t) {
        distinct_count_kernel<<<grid_for(ctx, (int64_t)A.dt[t].mask + 1, 256), 256, 0, ctx.stream>>>(A, t, dcount);
        ctx.check_launch("distinct_count_kernel");
      }
    }
    int64_t G_out = 0;
    uint32_t* ordered = nullptr;
    uint32_t* rows32 = nullptr;  // first row of each output group (u32)
    MemP mslots, mcnt, mbits, mwc, mwo, mord, mof, mrow;
    MemP mjp, mjb;
    uint32_t* jprow = nullptr;  // fused join: first joined row's probe row (global) and build row per group
    uint32_t* jbrow = nullptr;
    if (join && !(small_try && small_n != ~0ULL)) fused_fail("more than 4,096 groups over a join");
    if (small_try && small_n != ~0ULL) {
      G_out = (int64_t)small_n;
      ordered = s_ordered;
      rows32 = s_rows;
      if (join) {
        jprow = ctx.alloc_t<uint32_t>((size_t)std::max<int64_t>(G_out, 1), mjp);
        jbrow = ctx.alloc_t<uint32_t>((size_t)std::max<int64_t>(G_out, 1), mjb);
        if (G_out) {
          split_join_rows_kernel<<<grid_for(ctx, G_out, 256), 256, 0, ctx.stream>>>(s_firsts, G_out, jprow, jbrow);
          ctx.check_launch("split_join_rows_kernel");
        }
      }
    } else {
      uint32_t* slots = ctx.alloc_t<uint32_t>(nslots, mslots);
      unsigned long long* counter = ctx.alloc_t<unsigned long long>(1, mcnt);
      PRISM_CUDA(cudaMemsetAsync(counter, 0, 8, ctx.stream));
      collect_groups_kernel<<<grid_for(ctx, (int64_t)nslots, 256), 256, 0, ctx.stream>>>(A.gfirst, (int64_t)nslots, slots,
                                                                                        counter);
      ctx.check_launch("collect_groups_kernel");
      unsigned long long ng = 0;
      PRISM_CUDA(cudaMemcpyAsync(&ng, counter, 8, cudaMemcpyDeviceToHost, ctx.stream));
      PRISM_CUDA(cudaStreamSynchronize(ctx.stream));
      G_out = (int64_t)ng;
      // first-seen order: rank of each group's first row among all first rows
      int64_t nw = ceil_div(total_rows, 32);
      uint32_t* bits = ctx.alloc_t<uint32_t>((size_t)nw, mbits);
      uint32_t* wc = ctx.alloc_t<uint32_t>((size_t)nw, mwc);
      uint64_t* wo = ctx.alloc_t<uint64_t>((size_t)nw, mwo);
      ordered = ctx.alloc_t<uint32_t>((size_t)std::max<int64_t>(G_out, 1), mord);
      unsigned long long* ofirst = ctx.alloc_t<unsigned long long>((size_t)std::max<int64_t>(G_out, 1), mof);
      PRISM_CUDA(cudaMemsetAsync(bits, 0, nw * 4, ctx.stream));
      if (G_out) {
        mark_first_kernel<<<grid_for(ctx, G_out, 256), 256, 0, ctx.stream>>>(A.gfirst, slots, G_out, bits);
        ctx.check_launch("mark_first_kernel");
        word_popc32_kernel<<<grid_for(ctx, nw, 256), 256, 0, ctx.stream>>>(bits, nw, wc);
        ctx.check_launch("word_popc32_kernel");
        scan_u32(ctx, wc, wo, nw);
        place_groups_kernel<<<grid_for(ctx, G_out, 256), 256, 0, ctx.stream>>>(A.gfirst, slots, G_out, bits, wo, ordered,
                                                                              ofirst);
        ctx.check_launch("place_groups_kernel");
      }
      if (cfg.n_group_by) {
        if (total_rows >= (int64_t)UINT32_MAX) fail(PRISM_ERR_INVALID_ARGUMENT, "aggregation input exceeds 2^32-1 rows");
        // narrow the first rows to u32 indices
        rows32 = ctx.alloc_t<uint32_t>((size_t)std::max<int64_t>(G_out, 1), mrow);
        if (G_out) {
          narrow_kernel<<<grid_for(ctx, G_out, 256), 256, 0, ctx.stream>>>(ofirst, G_out, rows32);
          ctx.check_launch("narrow_kernel");
        }
      }
    }
    Batch out;
    out.rows = G_out;
    // key columns: gather first rows (keys of multi-batch inputs are concatenated first)
    if (cfg.n_group_by) {
      for (int k = 0; k < cfg.n_group_by; ++k) {
        int bc = gbatch_cols[k];
        const Column& rc = *ref.cols[bc];
        ColP keycol;
        if (join && bc >= n_probe_cols) {  // build-side key: read at the build row
          keycol = take(ctx, *join->table->build.cols[bc - n_probe_cols], jbrow, nullptr, G_out, rc.name, rc.nullable);
        } else {
          std::vector<const Column*> parts;
          for (auto* b : batches)
            if (b->rows) parts.push_back(b->cols[bc].get());
          ColP src = parts.size() == 1
                         ? std::shared_ptr<Column>(std::shared_ptr<Column>{}, const_cast<Column*>(parts[0]))
                         : concat_columns(ctx, parts);
          keycol = take(ctx, *src, join ? jprow : rows32, nullptr, G_out, rc.name, rc.nullable);
        }
        if (fused && cfg.group_by[k] >= n_cols) keycol->name = proj_name(cfg.group_by[k]);
        out.cols.push_back(keycol);
      }
    }
    // aggregate columns
    FinalArgs F{};
    F.ordered = ordered;
    F.n = G_out;
    F.gacc = A.gacc;
    F.W = W;
    F.n_out = (int)P.outs.size();
    for (int j = 0; j < A.n_ops; ++j) F.op[j] = A.op[j];
    F.dcount = dcount;
    F.wide = A.wide;
    F.n_wide = A.n_wide;
    F.gwide = A.gwide;
    F.total_rows = total_rows;
    F.grouped = global ? 0 : 1;
    for (size_t k = 0; k < P.outs.size(); ++k) {
      int t = P.out_types[k];
      ColP c = make_column(ctx, t, P.names[k], G_out, false);
      c->nullable = true;
      if (t == TY_DEC128) { c->precision = 38; c->scale = P.out_scale[k]; }
      P.outs[k].out = c->values;
      F.out[k] = P.outs[k];
      out.cols.push_back(c);
    }
    if (G_out) {
      finalize_kernel<<<grid_for(ctx, G_out, 128), 128, 0, ctx.stream>>>(F);
      ctx.check_launch("finalize_kernel");
    }
    // the result is stream-ordered: the export (or the caller's next call on
    // this context) waits for it, so no synchronisation here
    return out;
  }
  fail(PRISM_ERR_TABLE_FULL, "aggregation table could not be sized");
}

}  // namespace prism
