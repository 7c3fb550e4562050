// agg_device.cuh — device-side state and accumulation code of the GROUP BY
// engine, shared by the ahead-of-time kernels (agg.cu) and the per-query
// kernels generated at run time (jit.cu), which compile this header with
// NVRTC. Accumulator semantics follow hash_aggregate
// (native/prism-executor/src/hash_aggregate.rs:174-447), made exact: integer
// SUMs in 128-bit limbs, Float64 SUMs in a fixed-point window rounded once,
// MIN/MAX by IEEE totalOrder.
#pragma once

#include "eval.cuh"
#include "join_device.cuh"

namespace prism {

constexpr int MAX_SRC = 16;
constexpr int MAX_OPS = 24;
constexpr int MAX_W = 64;
constexpr int MAX_GCOLS = 8;
constexpr int LIMBS = 6;  // f64 window: 6 x 32 bits
constexpr int WIDE_LIMBS = 68;  // 2^-1074 .. 2^1102
constexpr int WIDE_LO = -1074;

enum SrcKind : int32_t { S_COL_F64 = 0, S_COL_INT, S_COL_I128, S_EXPR_F64, S_EXPR_I128, S_VALID };
enum OpKind : int32_t { O_SUM_F64 = 0, O_SUM_INT, O_SUM_DEC, O_MIN, O_MAX, O_NONNULL, O_DISTINCT };
enum WordKind : int32_t { W_ADD = 0, W_MIN, W_MAX, W_OR };

struct Src {
  int32_t kind;
  int32_t col;          // program column slot
  int32_t begin, end;   // expression nodes
};
struct Op {
  int32_t kind;
  int32_t src;
  int32_t word;
  int32_t lo_exp;       // O_SUM_F64 window bottom exponent
  int32_t distinct;     // O_DISTINCT: table index
  int32_t pad;
};

struct DistinctTable {
  unsigned long long* slots;  // pairs (a, b)
  uint64_t mask;
};

struct AggArgs {
  int64_t n;
  uint64_t row_base;
  const PNode* pn;
  const ENode* en;
  const PRange* cl;
  const DCol* cols;
  int32_t has_filter;
  PRange filter;
  int32_t n_src;
  Src src[MAX_SRC];
  int32_t n_ops;
  Op op[MAX_OPS];
  int32_t W;
  unsigned long long winit[MAX_W];
  int32_t wkind[MAX_W];
  int32_t skip_nulls;
  int32_t count_rows;       // maintain word 0 (grouped path)
  // group identity
  int32_t n_gcols;
  int32_t gcol[MAX_GCOLS];
  int32_t dense;
  int64_t G;
  int64_t dstride[MAX_GCOLS];
  int64_t dnull[MAX_GCOLS];
  // shared-memory table geometry (hash mode)
  int32_t ss_log2;
  int32_t sd;
  int32_t use_smem;
  // few dense groups (tiny_body): number of program columns in `cols`
  int32_t n_cols;
  // global table
  unsigned long long* gkeys;
  unsigned long long* gfirst;
  unsigned long long* gacc;
  // fused join (join_body): each probe row looks up the build table and
  // every matched build row is aggregated as a joined row; the program
  // columns of the build side are read at the build row
  int32_t join;
  int32_t jfast;             // single Int64 key matched by raw value
  const ulonglong2* jslots;  // {key or row hash, cnt << 32 | row}; [jcap] = side slot
  int32_t jshift;
  uint64_t jmask;
  uint64_t jcap;
  const uint32_t* jdup;      // build rows of multi-row slots
  int64_t jn_dup;            // their count (a segment past it: DERR_CORRUPT)
  const uint32_t* jdense;    // dense mode: build row per key - jdmin
  int64_t jdmin;
  uint64_t jdrange;
  const DCol* jpk;           // probe key column views
  const DCol* jbk;           // build key column views
  const ulonglong2* jkrec;   // packed build keys (single Utf8 key), or null
  const ulonglong2* jent;    // slot entries (single Utf8 key), or null
  int32_t jent_col;          // joined column whose value the entries (or jinl) carry, or -1
  // split join -> aggregate: per probe row the match word written by
  // match_rows_kernel (verified build row, JOIN_NO_MATCH, or
  // JOIN_MATCH_SLOT | slot of several build rows) and the inlined value
  const uint32_t* jmatch;
  const void* jinl;
  int32_t jinl_w;            // 4 or 8 bytes per row, 0: none
  int32_t jkw;               // single Utf8 probe key against key records: compared as words
  int32_t jnkeys;
  uint32_t* gnew;                  // slots in creation order (ginsert appends), or null
  unsigned long long* gnew_count;  // length of gnew
  uint64_t gmask;
  int32_t gshift;
  uint64_t gcap;
  DistinctTable dt[4];
  uint32_t* err;
  int* maxexp;   // per op (O_SUM_F64 overflow diagnosis)
  // wide mode: Float64 sums over the whole double range (68 limbs from
  // 2^-1074), global accumulators only; used when a value overflowed the
  // 192-bit window
  int32_t wide;
  int32_t n_wide;
  unsigned long long* gwide;  // [slot][n_wide][WIDE_LIMBS + 1]
};

// ------------------------------------------------------------ accumulate --

__device__ __forceinline__ void atom_add(unsigned long long* p, unsigned long long v) {
  if (v) atomicAdd(p, v);
}

// Adds v to a 6-limb fixed-point accumulator whose bit 0 weighs 2^lo_exp
// (acc[6] collects NaN/+inf/-inf flags). A value with set bits above or
// below the window raises DERR_OVERFLOW (the caller reruns over the wide
// window from 2^-1074, which holds every double exactly), so no bit is lost.
__device__ inline void add_f64(unsigned long long* acc, double v, int lo_exp, uint32_t* err, int* maxexp, int nl = LIMBS) {
  uint64_t u = (uint64_t)__double_as_longlong(v);
  int be = (int)((u >> 52) & 0x7ff);
  uint64_t m = u & 0xFFFFFFFFFFFFFULL;
  if (be == 0x7ff) {
    atomicOr(acc + nl, m ? 1ULL : ((u >> 63) ? 4ULL : 2ULL));
    return;
  }
  if (be) m |= 1ULL << 52;
  else be = 1;
  if (!m) return;
  int pos = be - 1075 - lo_exp;
  if (pos < 0) {
    // set bits below 2^lo_exp: the window cannot hold the value exactly
    if (pos <= -64 || (m & ((1ULL << -pos) - 1))) {
      atomicOr(err, DERR_OVERFLOW);
      return;
    }
    m >>= -pos;
    pos = 0;
  }
  int k = pos >> 5, sh = pos & 31;
  unsigned __int128 x = (unsigned __int128)m << sh;
  uint32_t p0 = (uint32_t)x, p1 = (uint32_t)(x >> 32), p2 = (uint32_t)(x >> 64);
  if (k >= nl || (k + 1 >= nl && p1) || (k + 2 >= nl && p2)) {
    atomicOr(err, DERR_OVERFLOW);
    atomicMax(maxexp, be);
    return;
  }
  bool neg = u >> 63;
  unsigned long long q0 = neg ? (unsigned long long)(-(long long)p0) : p0;
  unsigned long long q1 = neg ? (unsigned long long)(-(long long)p1) : p1;
  unsigned long long q2 = neg ? (unsigned long long)(-(long long)p2) : p2;
  atom_add(acc + k, q0);
  if (k + 1 < nl) atom_add(acc + k + 1, q1);
  if (k + 2 < nl) atom_add(acc + k + 2, q2);
}

__device__ __forceinline__ void add_i128_limbs(unsigned long long* acc, __int128 v, int n_limbs) {
  // n_limbs 32-bit limbs, the top one signed
  for (int q = 0; q < n_limbs; ++q) {
    long long part;
    if (q == n_limbs - 1) part = (long long)(v >> (32 * q));
    else part = (long long)(uint32_t)(v >> (32 * q));
    atom_add(acc + q, (unsigned long long)part);
  }
}

__device__ __forceinline__ int64_t ceil_div_dev(int64_t a, int64_t b) { return (a + b - 1) / b; }

// An integer SUM operand as the reference sums it: its Float64 cast
// (hash_aggregate.rs:227-245 casts every input to Float64), as an exact
// integer. The identity for |v| < 2^53; above, v rounded to nearest even
// (2^63 - 1 rounds to 2^63, which only the 128-bit form holds).
__device__ __forceinline__ bool f64_exact_int(long long v) { return v > -(1LL << 53) && v < (1LL << 53); }
__device__ __forceinline__ __int128 f64_cast_int(long long v) {
  if (f64_exact_int(v)) return v;
  const double d = (double)v;
  if (d >= 9223372036854775808.0) return (__int128)1 << 63;
  return (__int128)(long long)d;
}

// ------------------------------------------------- global group table --
constexpr uint64_t GEMPTY = 0xFFFFFFFFFFFFFFFFULL;  // empty slot (a key hashing to it takes the side slot)
constexpr uint64_t FIB = 0x9E3779B97F4A7C15ULL;

// global open-addressing insert; returns the slot or -1 when full
__device__ inline int64_t ginsert(const AggArgs& a, uint64_t h) {
  if (h == GEMPTY) return (int64_t)a.gcap;  // side slot
  uint64_t s = (h * FIB) >> a.gshift;
  for (uint64_t step = 0; step <= a.gmask; ++step) {
    unsigned long long cur = *(volatile unsigned long long*)&a.gkeys[s];
    if (cur == h) return (int64_t)s;
    if (cur == GEMPTY) {
      unsigned long long prev = atomicCAS(&a.gkeys[s], GEMPTY, h);
      if (prev == GEMPTY) {  // created: listed once, by its creator
        if (a.gnew) a.gnew[atomicAdd(a.gnew_count, 1ULL)] = (uint32_t)s;
        return (int64_t)s;
      }
      if (prev == h) return (int64_t)s;
    }
    s = (s + 1) & a.gmask;
  }
  atomicOr(a.err, DERR_TABLE_FULL);
  return -1;
}

// folds a privatised accumulator word into the global one
__device__ __forceinline__ void merge_word(unsigned long long* dst, unsigned long long v, int kind) {
  switch (kind) {
    case W_ADD: atom_add(dst, v); break;
    case W_MIN: atomicMin((long long*)dst, (long long)v); break;
    case W_MAX: atomicMax((long long*)dst, (long long)v); break;
    case W_OR: if (v) atomicOr(dst, v); break;
  }
}

// ------------------------------------------------ few dense groups (<= 8) --
// The kernel body for GROUP BY with at most 8 dense groups (dictionary keys,
// or none). Every thread owns a private column of accumulators in shared
// memory, word w of thread t at tacc[w * TINY_BLOCK + t] (a warp's accesses
// never conflict, whatever groups its rows fall in). Per group: word 0 the
// row count, word 1 the first row seen, then each op's words (int64 partial
// of an integer sum, the two doubles of a double-double Float64 sum, a
// totalOrder MIN/MAX key, a non-null count). Slot G takes the rows the
// filter drops, so the row loop has no data-dependent branches: every row
// does one read-modify-write of its slot's words. An integer partial that
// would overflow spills exactly into the block's 128-bit accumulators.
// Threads stride over the rows so each warp loads 32 consecutive rows per
// step, TINY_R steps deep before using them (many loads in flight). At the
// end the block folds the columns (exact 128-bit integer sums, double-double
// Float64 sums) into the global words agg_kernel fills, so the same
// finalize kernels run.
//
// E supplies the row logic as code generated per query (jit.cu): E::Consts /
// E::load (per-thread constants read once), E::Row / E::fetch (a row's
// fixed-width column words, loaded first), E::keep (filter), E::gid (dense
// group id), E::values (every op's operand, with per-op flags asking for the
// exact recomputation E::slow or reporting an overflow), and the
// compile-time layout kKind[j] (op kinds), kWord[j] (first word of op j in
// a group), kNW (words per group), kI64[j] (op j's fast value fits int64),
// kSkipNulls.
constexpr int TINY_R = 2;        // rows in flight per thread
constexpr int TINY_MAX_COLS = 16;
// (G + 1) * kNW accumulator words per thread: up to 48 with 256-thread
// blocks, up to 96 with 128-thread blocks (96 KB of shared memory a block)
constexpr int TINY_MAX_WORDS = 96;
__host__ __device__ constexpr int tiny_block(int words) { return words <= 48 ? 256 : 128; }
constexpr int TINY_FIRST_OP_WORD = 2;

__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}

// result of a generated program's out-of-line 128-bit path
struct SlowVal {
  Val v;
  bool ovf;
};

// words an op occupies in a group's accumulator column
__host__ __device__ constexpr int tiny_words(int kind) { return kind == O_SUM_F64 ? 2 : 1; }

__host__ __device__ constexpr unsigned long long tiny_init(int kind) {
  return kind == O_MIN ? 0x7fffffffffffffffULL : kind == O_MAX ? 0x8000000000000000ULL : 0ULL;
}

// one row's contribution to its slot's words; FAST: the ops E::kI64 marks
// hold values that fit int64 (no 128-bit test)
template <class E, int G, int NOPS, bool F64, int BLOCK, bool FAST>
__device__ __forceinline__ void tiny_accumulate(const AggArgs& a, unsigned long long* col, int g, const Val* v,
                                                unsigned long long (*spill)[NOPS][4]) {
#pragma unroll
  for (int j = 0; j < NOPS; ++j) {
    const int kind = E::kKind[j];
    const Val& x = v[j];
    const bool use = !(E::kSkipNulls && !x.valid);
    unsigned long long* w = col + E::kWord[j] * BLOCK;
    if (kind == O_SUM_INT || kind == O_SUM_DEC) {
      const bool narrow = FAST && E::kI64[j];
      __int128 xi = use ? x.i : (__int128)0;
      long long x64 = narrow ? (use ? (long long)x.i : 0LL) : (long long)xi;
      // integer column: the value's Float64 cast (exact below 2^53: the
      // partial takes it; else the cast goes through the spill)
      bool fits = narrow || (__int128)x64 == xi;
      if (kind == O_SUM_INT && !f64_exact_int(x64)) {
        xi = f64_cast_int(x64);
        fits = false;
      }
      long long p = (long long)w[0];
      long long s = (long long)((unsigned long long)p + (unsigned long long)x64);
      if (fits && !(((p ^ s) & (x64 ^ s)) < 0)) {
        w[0] = (unsigned long long)s;
      } else {  // exact spill of partial + value; the partial restarts at 0
        if (g < G) add_i128_limbs(&spill[g][j][0], (__int128)p + xi, kind == O_SUM_INT ? 2 : 4);
        w[0] = 0;
      }
    } else if (kind == O_SUM_F64) {
      if (F64) {
        double xf = use ? x.f : 0.0;
        if (!isfinite(xf)) {  // NaN / inf: flag straight into the global accumulator
          if (g < G) {
            uint64_t u = (uint64_t)__double_as_longlong(xf);
            atomicOr(a.gacc + (size_t)g * a.W + a.op[j].word + LIMBS, isnan(xf) ? 1ULL : ((u >> 63) ? 4ULL : 2ULL));
          }
        } else {
          double s, e;
          two_sum(__longlong_as_double((long long)w[0]), xf, s, e);
          w[0] = (unsigned long long)__double_as_longlong(s);
          w[BLOCK] = (unsigned long long)__double_as_longlong(__longlong_as_double((long long)w[BLOCK]) + e);
        }
      }
    } else if (kind == O_MIN) {
      if (use && !isnan(x.f)) w[0] = (unsigned long long)min((long long)w[0], (long long)total_key(x.f));
    } else if (kind == O_MAX) {
      if (use && !isnan(x.f)) w[0] = (unsigned long long)max((long long)w[0], (long long)total_key(x.f));
    } else if (kind == O_NONNULL) {
      w[0] += x.valid ? 1ULL : 0ULL;
    }
  }
}

template <class E, int G, int NOPS, bool F64, int BLOCK>
__device__ __forceinline__ void tiny_body(const AggArgs& a) {
  constexpr int NW = E::kNW;
  constexpr int GS = G + 1;  // slot G: dropped rows
  extern __shared__ unsigned long long tacc[];  // [GS * NW][BLOCK]
  __shared__ unsigned long long spill[G][NOPS][4];  // exact overflow of integer partials
  __shared__ DCol scols[TINY_MAX_COLS];
  const int tid = threadIdx.x;
  const bool shared_cols = a.n_cols <= TINY_MAX_COLS;
  if (shared_cols && tid < a.n_cols) scols[tid] = a.cols[tid];
  for (int q = tid; q < G * NOPS * 4; q += BLOCK) (&spill[0][0][0])[q] = 0;
#pragma unroll
  for (int g = 0; g < GS; ++g) {
    tacc[(g * NW) * BLOCK + tid] = 0;
    tacc[(g * NW + 1) * BLOCK + tid] = ~0ULL;
#pragma unroll
    for (int j = 0; j < NOPS; ++j) {
      tacc[(g * NW + E::kWord[j]) * BLOCK + tid] = tiny_init(E::kKind[j]);
      if (tiny_words(E::kKind[j]) == 2) tacc[(g * NW + E::kWord[j] + 1) * BLOCK + tid] = 0;
    }
  }
  __syncthreads();
  const DCol* cols = shared_cols ? scols : a.cols;
  const typename E::Consts K = E::load(a);
  unsigned long long* my = tacc + tid;
  // row indices in E::idx_t: 32-bit when the batch has fewer than 2^31 rows
  // (cheaper address arithmetic), else 64-bit
  using I = typename E::idx_t;
  const I stride = (I)gridDim.x * BLOCK;
  const I n = (I)a.n, last = n - 1;
  bool err = false;
  unsigned seen = 0;  // slots this thread has met (slot G included: harmless)
  for (I base = (I)blockIdx.x * BLOCK + tid; base < n; base += stride * TINY_R) {
    int slot[TINY_R];
    unsigned flags[TINY_R];
    Val v[TINY_R][NOPS];
    typename E::Row rows[TINY_R];
    // phase 1: the fixed-width columns of all TINY_R rows are loaded first
    // (straight-line loads, all in flight together), then evaluated with
    // arithmetic only (no stores, atomics or calls)
#pragma unroll
    for (int r = 0; r < TINY_R; ++r) {
      I at = base + r * stride;
      I idx = at < last ? at : last;
      rows[r] = E::fetch(cols, idx, idx);  // rows past the end read the last row and are dropped
    }
#pragma unroll
    for (int r = 0; r < TINY_R; ++r) {
      I at = base + r * stride;
      I idx = at < last ? at : last;
      bool keep = at <= last && E::keep(a, K, cols, idx, idx, rows[r]);
      int g = E::gid(a, K, cols, idx, idx, rows[r]);
      bool bad = keep && (g < 0 || g >= G);
      err |= bad;
      slot[r] = (keep && !bad) ? g : G;
      flags[r] = 0;
      E::values(a, K, cols, idx, idx, rows[r], v[r], flags[r]);
    }
    // phase 2: the accumulators; rows with a flagged op first get its
    // 128-bit recomputation and take the general accumulate path, the others
    // the lean one (ops known to fit int64 there)
#pragma unroll
    for (int r = 0; r < TINY_R; ++r) {
      const int g = slot[r];
      const I at = base + r * stride;
      unsigned long long* col = my + (g * NW) * BLOCK;
      col[0] += 1;
      // a thread meets its rows in increasing order: the first row of a
      // group is the one seen while its bit is still clear
      const unsigned bit = 1u << g;
      if (!(seen & bit)) col[BLOCK] = a.row_base + (uint64_t)at;
      seen |= bit;
      if (g < G && flags[r]) {
        // every op of the row recomputed exactly (so the fast path's values
        // need only their 64-bit form kept)
        Val w[NOPS];
#pragma unroll
        for (int j = 0; j < NOPS; ++j) {
          SlowVal sv = E::slow(a, j, cols, at, at);
          w[j] = sv.v;
          err |= sv.ovf;
        }
        tiny_accumulate<E, G, NOPS, F64, BLOCK, false>(a, col, g, w, spill);
      } else {
        tiny_accumulate<E, G, NOPS, F64, BLOCK, true>(a, col, g, v[r], spill);
      }
    }
  }
  if (err) atomicOr(a.err, DERR_RANGE);
  __syncthreads();
  // fold the thread columns: one item per (group, count / first row / op)
  for (int q = tid; q < G * (NOPS + 2); q += BLOCK) {
    const int g = q / (NOPS + 2), jj = q % (NOPS + 2);
    unsigned long long* accg = a.gacc + (size_t)g * a.W;
    const unsigned long long* row = tacc + (size_t)(g * NW) * BLOCK;
    if (jj == 0) {
      unsigned long long c = 0;
      for (int t = 0; t < BLOCK; ++t) c += row[t];
      if (a.count_rows) atom_add(accg, c);
      continue;
    }
    if (jj == 1) {
      unsigned long long f = ~0ULL;
      for (int t = 0; t < BLOCK; ++t) f = min(f, row[BLOCK + t]);
      if (f != ~0ULL) atomicMin(&a.gfirst[g], f);
      continue;
    }
    const int j = jj - 2;
    int kind = 0, word = 0;
#pragma unroll
    for (int k = 0; k < NOPS; ++k)
      if (k == j) { kind = E::kKind[k]; word = E::kWord[k]; }
    const unsigned long long* w = row + (size_t)word * BLOCK;
    unsigned long long* gw = accg + a.op[j].word;
    if (kind == O_SUM_INT || kind == O_SUM_DEC) {
      __int128 s = 0;
      for (int t = 0; t < BLOCK; ++t) s += (__int128)(long long)w[t];
      for (int l = 0; l < 4; ++l) s += (__int128)(long long)spill[g][j][l] << (32 * l);
      add_i128_limbs(gw, s, kind == O_SUM_INT ? 2 : 4);
    } else if (kind == O_SUM_F64) {
      if (F64) {
        double h = 0, l = 0;
        for (int t = 0; t < BLOCK; ++t) {
          double s1, e1;
          two_sum(h, __longlong_as_double((long long)w[t]), s1, e1);
          e1 += l + __longlong_as_double((long long)w[t + BLOCK]);
          h = s1 + e1;
          l = e1 - (h - s1);
        }
        add_f64(gw, h, a.op[j].lo_exp, a.err, a.maxexp + j);  // both parts exactly into the window
        add_f64(gw, l, a.op[j].lo_exp, a.err, a.maxexp + j);
      }
    } else if (kind == O_MIN || kind == O_MAX) {
      long long m = (long long)tiny_init(kind);
      for (int t = 0; t < BLOCK; ++t) m = kind == O_MIN ? min(m, (long long)w[t]) : max(m, (long long)w[t]);
      if (m != (long long)tiny_init(kind)) {
        if (kind == O_MIN) atomicMin((long long*)gw, m);
        else atomicMax((long long*)gw, m);
      }
    } else if (kind == O_NONNULL) {
      unsigned long long c = 0;
      for (int t = 0; t < BLOCK; ++t) c += w[t];
      atom_add(gw, c);
    }
  }
}

// ---------------------------------------------- hashed groups (generated) --
// The kernel body for GROUP BY over hashed keys. Each block keeps a
// shared-memory open-addressing table of group hashes (the reference's
// FxHash identity, hash_aggregate.rs:483-504) whose slot s owns the
// accumulator words sacc[s * kW ...] in the global word layout (word 0 the
// row count, then each op's words at E::kWord[j]): a row finds or claims its
// slot with one compare-and-swap and updates the words with shared-memory
// atomics. A row whose key finds no slot within HASH_PROBES steps (or
// hashes to the empty marker) goes to the global table directly. At the end
// the block resolves each used slot's global slot once and folds its words
// in, one thread per (slot, word), so a warp's global atomics hit
// consecutive words. Rows are read TINY_R deep per thread (all loads of a
// step in flight before any is used), as in tiny_body.
//
// E supplies, besides the members tiny_body uses (keep, values, slow, Row,
// fetch, kKind, kI64, kSkipNulls), E::hash (the key columns' FxHash), kW
// (words per group, a.W), kWord (op j's first word, a.op[j].word) and
// kCountRows; initial values and merge kinds of the words are a.winit and
// a.wkind.
constexpr int HASH_PROBES = 32;

template <class E, int NOPS, bool FAST>
__device__ __forceinline__ void hash_accumulate(const AggArgs& a, unsigned long long* acc, const Val* v) {
  if (E::kCountRows) atomicAdd(acc, 1ULL);
#pragma unroll
  for (int j = 0; j < NOPS; ++j) {
    const int kind = E::kKind[j];
    const Val& x = v[j];
    if (E::kSkipNulls && !x.valid) continue;
    unsigned long long* w = acc + E::kWord[j];
    if (kind == O_SUM_F64) {
      add_f64(w, x.f, a.op[j].lo_exp, a.err, a.maxexp + j);
    } else if (kind == O_SUM_INT) {
      const long long q = (long long)x.i;
      if (q >= -(1LL << 32) && q < (1LL << 32)) {
        // one signed add into the low limb's counter: with at most 2^31 rows
        // per call its magnitude stays below 2^63
        atom_add(w, (unsigned long long)q);
      } else if (f64_exact_int(q)) {  // two 32-bit limbs of an int64 value, the top one signed
        atom_add(w, (unsigned long long)(uint32_t)q);
        atom_add(w + 1, (unsigned long long)(q >> 32));
      } else {
        add_i128_limbs(w, f64_cast_int(q), 2);
      }
    } else if (kind == O_SUM_DEC) {
      add_i128_limbs(w, x.i, 4);
    } else if (kind == O_MIN || kind == O_MAX) {
      if (!isnan(x.f)) {
        const long long k = (long long)total_key(x.f);
        const long long cur = (long long)*(volatile unsigned long long*)w;
        if (kind == O_MIN ? k < cur : k > cur) {  // most rows do not move the extreme: no atomic
          if (kind == O_MIN) atomicMin((long long*)w, k);
          else atomicMax((long long*)w, k);
        }
      }
    } else if (kind == O_NONNULL) {
      if (x.valid) atomicAdd(w, 1ULL);
    }
  }
}

// the block's table: skeys[SS] | sfirst[SS] | sacc[SS][kW] in dynamic
// shared memory
struct HashTable {
  unsigned long long* keys;
  unsigned long long* first;
  unsigned long long* acc;
  uint32_t mask;
  int shift;
};

template <class E>
__device__ __forceinline__ HashTable hash_table_init(const AggArgs& a, unsigned long long* smem, int tid, int block) {
  constexpr int W = E::kW;
  const int SS = 1 << a.ss_log2;
  HashTable t{smem, smem + SS, smem + 2 * SS, (uint32_t)SS - 1, 64 - a.ss_log2};
  for (int i = tid; i < SS; i += block) {
    t.keys[i] = GEMPTY;
    t.first[i] = ~0ULL;
  }
  for (int i = tid; i < SS * W; i += block) t.acc[i] = a.winit[i % W];
  return t;
}

// one (joined) row into its group: find or claim the key's slot, else the
// global table; `first` orders the rows (first-seen order of the groups)
template <class E, int NOPS>
__device__ __forceinline__ void hash_row_update(const AggArgs& a, const HashTable& t, uint64_t h, uint64_t first,
                                                const Val* v, unsigned flags, const DCol* cols,
                                                typename E::idx_t idx, typename E::idx_t bidx, bool& err) {
  constexpr int W = E::kW;
  int s = -1;
  if (h != GEMPTY) {
    uint32_t p = (uint32_t)((h * FIB) >> t.shift);
    for (int step = 0; step < HASH_PROBES; ++step) {
      unsigned long long cur = *(volatile unsigned long long*)&t.keys[p];
      if (cur == GEMPTY) {
        cur = atomicCAS(&t.keys[p], GEMPTY, h);
        if (cur == GEMPTY) cur = h;
      }
      if (cur == h) {
        s = (int)p;
        break;
      }
      p = (p + 1) & t.mask;
    }
  }
  unsigned long long* acc;
  if (s >= 0) {
    if (first < t.first[s]) atomicMin(&t.first[s], first);
    acc = t.acc + (size_t)s * W;
  } else {
    const int64_t gs = ginsert(a, h);
    if (gs < 0) return;
    if (first < a.gfirst[gs]) atomicMin(&a.gfirst[gs], first);
    acc = a.gacc + (size_t)gs * W;
  }
  if (flags) {
    // every op of the row recomputed exactly
    Val w[NOPS];
#pragma unroll
    for (int j = 0; j < NOPS; ++j) {
      SlowVal sv = E::slow(a, j, cols, idx, bidx);
      w[j] = sv.v;
      err |= sv.ovf;
    }
    hash_accumulate<E, NOPS, false>(a, acc, w);
  } else {
    hash_accumulate<E, NOPS, true>(a, acc, v);
  }
}

// folds the block's table into the global one: each used slot's global slot
// resolved once (kept in keys, -1: none), then one thread per (slot, word)
template <class E>
__device__ __forceinline__ void hash_table_merge(const AggArgs& a, const HashTable& t, int tid, int block) {
  constexpr int W = E::kW;
  const int SS = 1 << a.ss_log2;
  for (int i = tid; i < SS; i += block) {
    const unsigned long long k = t.keys[i];
    long long gs = -1;
    if (k != GEMPTY) {
      gs = ginsert(a, k);
      if (gs >= 0) atomicMin(&a.gfirst[gs], t.first[i]);
    }
    t.keys[i] = (unsigned long long)gs;
  }
  __syncthreads();
  for (int q = tid; q < SS * W; q += block) {
    const int i = q / W, w = q - i * W;
    const long long gs = (long long)t.keys[i];
    if (gs < 0) continue;
    const unsigned long long x = t.acc[q];
    if (x != a.winit[w]) merge_word(a.gacc + (size_t)gs * W + w, x, a.wkind[w]);
  }
}

template <class E, int NOPS, int BLOCK>
__device__ __forceinline__ void hash_body(const AggArgs& a) {
  extern __shared__ unsigned long long hsm[];
  __shared__ DCol scols[TINY_MAX_COLS];
  const int tid = threadIdx.x;
  const bool shared_cols = a.n_cols <= TINY_MAX_COLS;
  if (shared_cols && tid < a.n_cols) scols[tid] = a.cols[tid];
  const HashTable t = hash_table_init<E>(a, hsm, tid, BLOCK);
  __syncthreads();
  const DCol* cols = shared_cols ? scols : a.cols;
  const typename E::Consts K = E::load(a);
  using I = typename E::idx_t;
  const I stride = (I)gridDim.x * BLOCK;
  const I n = (I)a.n, last = n - 1;
  bool err = false;
  for (I base = (I)blockIdx.x * BLOCK + tid; base < n; base += stride * TINY_R) {
    typename E::Row rows[TINY_R];
    bool keep[TINY_R];
    uint64_t hs[TINY_R];
    unsigned flags[TINY_R];
    Val v[TINY_R][NOPS];
#pragma unroll
    for (int r = 0; r < TINY_R; ++r) {
      I at = base + r * stride;
      I idx = at < last ? at : last;
      rows[r] = E::fetch(cols, idx, idx);  // rows past the end read the last row and are dropped
    }
#pragma unroll
    for (int r = 0; r < TINY_R; ++r) {
      I at = base + r * stride;
      I idx = at < last ? at : last;
      keep[r] = at <= last && E::keep(a, K, cols, idx, idx, rows[r]);
      hs[r] = E::hash(a, K, cols, idx, idx, rows[r]);
      flags[r] = 0;
      E::values(a, K, cols, idx, idx, rows[r], v[r], flags[r]);
    }
#pragma unroll
    for (int r = 0; r < TINY_R; ++r) {
      if (!keep[r]) continue;
      const I at = base + r * stride;
      hash_row_update<E, NOPS>(a, t, hs[r], a.row_base + (uint64_t)at, v[r], flags[r], cols, at, at, err);
    }
  }
  if (err) atomicOr(a.err, DERR_RANGE);
  __syncthreads();
  hash_table_merge<E>(a, t, tid, BLOCK);
}

// The fused join -> aggregate body: R probe rows per thread and step, their
// keys looked up in the build table as the probe kernels do
// (join_device.cuh) with all R lookups in flight together, then for every
// row with one candidate its joined row's fixed-width columns fetched (again
// R at once) before the keys are compared; every matched build row, in
// ascending order, is aggregated as the joined row (probe row, build row)
// into the block's table. The order key of a joined row is
// (global probe row << 32 | build row), which sorts like the joined rows'
// positions (probe rows ascending, build rows ascending inside one).
// KW: a single Utf8 probe key against packed key records: the key's words
// read once, hashed and compared as words (no byte loops, no second read)
template <class E, int NOPS, int BLOCK, int R, bool ENT, bool MATCH = false, bool KW = false>
__device__ __forceinline__ void join_body(const AggArgs& a) {
  extern __shared__ unsigned long long hsm[];
  __shared__ DCol scols[TINY_MAX_COLS];
  const int tid = threadIdx.x;
  const bool shared_cols = a.n_cols <= TINY_MAX_COLS;
  if (shared_cols && tid < a.n_cols) scols[tid] = a.cols[tid];
  const HashTable t = hash_table_init<E>(a, hsm, tid, BLOCK);
  __syncthreads();
  const DCol* cols = shared_cols ? scols : a.cols;
  const typename E::Consts K = E::load(a);
  using I = typename E::idx_t;
  const I stride = (I)gridDim.x * BLOCK;
  const I n = (I)a.n;
  bool err = false;
  for (I base = (I)blockIdx.x * BLOCK + tid; base < n; base += stride * R) {
    uint32_t cand[R], cnt[R];
    uint64_t key[R];
    ulonglong2 e[R];
    uint64_t s[R];
    // slot entries (a single Utf8 probe key): the key's words read once,
    // hashed, then compared against the 64-byte entry; keq / inl hold each
    // single-row slot's comparison and inlined build value
    JoinKeyWords kw[ENT || KW ? R : 1];
    bool kw_ok[ENT || KW ? R : 1];
    bool keq[R];
    unsigned long long inl[ENT || MATCH ? R : 1];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const I idx = base + r * stride;
      cnt[r] = 0;
      cand[r] = JOIN_NO_MATCH;
      key[r] = 0;
      keq[r] = true;
      if constexpr (ENT || KW) {
        kw_ok[r] = idx < n && join_key_words(a.jpk[0], idx, kw[r]);
        if (kw_ok[r]) key[r] = join_words_hash(kw[r]);
        else if (idx < n) key[r] = join_key_hash(a.jpk, a.jnkeys, idx);
      } else if (!MATCH && idx < n) {
        key[r] = a.jfast ? (uint64_t)static_cast<const int64_t*>(a.jpk[0].values)[idx]
                         : join_key_hash(a.jpk, a.jnkeys, idx);
      }
    }
    if constexpr (MATCH) {
      // the lookup is done: one coalesced word per row (and its inlined
      // value); a slot of several build rows is expanded below
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const I idx = base + r * stride;
        inl[r] = 0;
        if (idx >= n) continue;
        const uint32_t m = __ldcs(a.jmatch + idx);
        if (m == JOIN_NO_MATCH) continue;
        if (m & JOIN_MATCH_SLOT) {
          const ulonglong2 sl = __ldg(a.jslots + (m & ~JOIN_MATCH_SLOT));
          cand[r] = (uint32_t)sl.y;
          cnt[r] = (uint32_t)(sl.y >> 32);
        } else {
          cand[r] = m;
          cnt[r] = 1;
          if (a.jinl_w == 8) inl[r] = __ldcs(static_cast<const unsigned long long*>(a.jinl) + idx);
          else if (a.jinl_w == 4) inl[r] = __ldcs(static_cast<const uint32_t*>(a.jinl) + idx);
        }
      }
    } else if constexpr (ENT) {
      ulonglong2 e1[R], e2[R], e3[R];
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const I idx = base + r * stride;
        s[r] = join_slot_of(key[r], a.jshift);
        e[r] = make_ulonglong2(JOIN_EMPTY, 0);
        if (idx < n) {
          const ulonglong2* p = a.jent + 4 * s[r];
          e[r] = __ldg(p);
          e1[r] = __ldg(p + 1);
          e2[r] = __ldg(p + 2);
          e3[r] = __ldg(p + 3);
        }
      }
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const I idx = base + r * stride;
        inl[r] = 0;
        if (idx >= n) continue;
        for (uint64_t steps = 0; e[r].x != key[r] && e[r].x != JOIN_EMPTY && steps <= a.jmask; ++steps) {
          s[r] = (s[r] + 1) & a.jmask;
          const ulonglong2* p = a.jent + 4 * s[r];
          e[r] = __ldg(p);
          e1[r] = __ldg(p + 1);
          e2[r] = __ldg(p + 2);
          e3[r] = __ldg(p + 3);
        }
        if (e[r].x == key[r]) {
          cand[r] = (uint32_t)e[r].y;
          cnt[r] = (uint32_t)(e[r].y >> 32);
          if (cnt[r] == 1) {
            // a long key on either side: compared against the columns
            keq[r] = kw_ok[r] && !(e1[r].x & JOIN_ENT_LONG) ? join_words_equal(kw[r], e1[r], e2[r], e3[r])
                                                             : join_rows_equal(a.jpk, a.jbk, 1, idx, cand[r]);
            inl[r] = e3[r].y;
          }
        }
      }
    } else if (a.jdense) {
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const I idx = base + r * stride;
        const uint64_t d = key[r] - (uint64_t)a.jdmin;
        const uint32_t row = (idx < n && d < a.jdrange) ? __ldg(a.jdense + d) : JOIN_NO_MATCH;
        if (row != JOIN_NO_MATCH) {
          cand[r] = row;
          cnt[r] = 1;
        }
      }
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const I idx = base + r * stride;
        s[r] = (a.jfast && key[r] == JOIN_EMPTY) ? a.jcap : join_slot_of(key[r], a.jshift);
        e[r] = idx < n ? __ldg(a.jslots + s[r]) : make_ulonglong2(JOIN_EMPTY, 0);
      }
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const I idx = base + r * stride;
        if (idx >= n) continue;
        for (uint64_t steps = 0; e[r].x != key[r] && e[r].x != JOIN_EMPTY && steps <= a.jmask; ++steps) {
          s[r] = (s[r] + 1) & a.jmask;
          e[r] = __ldg(a.jslots + s[r]);
        }
        if (e[r].x == key[r]) {
          cand[r] = (uint32_t)e[r].y;
          cnt[r] = (uint32_t)(e[r].y >> 32);
        }
      }
    }
    // single-candidate rows: the joined rows' columns, all R in flight
    typename E::Row rows[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const I idx = base + r * stride;
      if (cnt[r] == 1) {
        if constexpr (ENT || MATCH) rows[r] = E::fetch(cols, idx, (I)cand[r], inl[r], true);
        else rows[r] = E::fetch(cols, idx, (I)cand[r]);
      }
    }
    // packed build keys: every single-candidate row's key compared up front
    // (the R record loads in flight together, beside the fetches above)
    if constexpr (KW) {
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const I idx = base + r * stride;
        keq[r] = cnt[r] == 1 ? (kw_ok[r] ? join_words_rec_equal(kw[r], a.jkrec, cand[r])
                                         : join_rec_equal(a.jpk[0], idx, a.jkrec, cand[r]))
                             : true;
      }
    } else if constexpr (!ENT && !MATCH) {  // (match_rows_kernel verified its single-row matches)
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const I idx = base + r * stride;
        keq[r] = !a.jfast && a.jkrec && cnt[r] == 1 ? join_rec_equal(a.jpk[0], idx, a.jkrec, cand[r]) : true;
      }
    }
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const I idx = base + r * stride;
      if (cnt[r] > 1 && (int64_t)cand[r] + cnt[r] > a.jn_dup) {  // an inconsistent table
        atomicOr(a.err, DERR_CORRUPT);
        continue;
      }
      for (uint32_t j = 0; j < cnt[r]; ++j) {
        const uint32_t b = cnt[r] == 1 ? cand[r] : a.jdup[cand[r] + j];
        if (!a.jfast) {
          const bool eq = cnt[r] == 1 && (ENT || MATCH || a.jkrec) ? keq[r]
                          : a.jkrec                       ? join_rec_equal(a.jpk[0], idx, a.jkrec, b)
                                                          : join_rows_equal(a.jpk, a.jbk, a.jnkeys, idx, b);
          if (!eq) continue;
        }
        const I bidx = (I)b;
        const typename E::Row row = cnt[r] == 1 ? rows[r] : E::fetch(cols, idx, bidx);
        if (!E::keep(a, K, cols, idx, bidx, row)) continue;
        const uint64_t h = E::hash(a, K, cols, idx, bidx, row);
        unsigned flags = 0;
        Val v[NOPS];
        E::values(a, K, cols, idx, bidx, row, v, flags);
        hash_row_update<E, NOPS>(a, t, h, ((a.row_base + (uint64_t)idx) << 32) | b, v, flags, cols, idx, bidx, err);
      }
    }
  }
  if (err) atomicOr(a.err, DERR_RANGE);
  __syncthreads();
  hash_table_merge<E>(a, t, tid, BLOCK);
}

}  // namespace prism
