// agg_device.cuh — device-side state and accumulation code of the GROUP BY
// engine, shared by the ahead-of-time kernels (agg.cu) and the per-query
// kernels generated at run time (jit.cu), which compile this header with
// NVRTC. Accumulator semantics follow hash_aggregate
// (native/prism-executor/src/hash_aggregate.rs:174-447), made exact: integer
// SUMs in 128-bit limbs, Float64 SUMs in a fixed-point window rounded once,
// MIN/MAX by IEEE totalOrder.
#pragma once

#include "eval.cuh"

namespace prism {

constexpr int MAX_SRC = 8;
constexpr int MAX_OPS = 16;
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
// (acc[6] collects NaN/+inf/-inf flags). Bits below the window are dropped.
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
    if (pos <= -64) return;
    m >>= -pos;
    pos = 0;
    if (!m) return;
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

// ------------------------------------------------ few dense groups (<= 8) --
// The kernel body for GROUP BY with at most 8 dense groups (dictionary keys,
// or none). Each warp takes 32 consecutive rows per sub-step, TINY_R
// sub-steps at a time (coalesced loads of all of them first, so that many
// bytes are in flight), then folds the rows into the groups with warp-wide
// reductions: per group a ballot gives the row count, and a butterfly of
// shuffles sums / min-maxes the operands of the rows in that group. Lane 0
// keeps the warp's running totals in shared memory (exact 128-bit integer
// sums, double-double Float64 sums, totalOrder MIN/MAX keys, counts) and
// merges them into the global accumulators once at the end, into the same
// words agg_kernel fills, so the same finalize kernels run. Per row the
// cost is the row's own arithmetic plus a few instructions per group,
// instead of one read-modify-write per accumulator.
//
// E supplies the row logic as straight-line code generated per query
// (jit.cu): E::Consts / E::load (per-thread constants read once), E::keep
// (filter), E::gid (dense group id), E::kind (op kind of j), E::value (op
// j's operand).
constexpr int TINY_BLOCK = 256;  // 8 warps; two blocks per SM
constexpr int TINY_R = 4;        // 32-row sub-steps per warp step
constexpr int TINY_MAX_COLS = 16;

__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}

__device__ __forceinline__ long long warp_sum64(long long x) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) x += __shfl_xor_sync(0xffffffffu, x, d);
  return x;
}

__device__ __forceinline__ __int128 warp_sum128(__int128 x) {
  unsigned long long lo = (unsigned long long)x, hi = (unsigned long long)((unsigned __int128)x >> 64);
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    unsigned long long olo = __shfl_xor_sync(0xffffffffu, lo, d), ohi = __shfl_xor_sync(0xffffffffu, hi, d);
    unsigned long long s = lo + olo;
    hi = hi + ohi + (s < lo ? 1ULL : 0ULL);
    lo = s;
  }
  return (__int128)(((unsigned __int128)hi << 64) | lo);
}

// double-double sum across the warp (error-free two_sum at every step)
__device__ __forceinline__ void warp_sum_dd(double& h, double& l) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    double oh = __shfl_xor_sync(0xffffffffu, h, d), ol = __shfl_xor_sync(0xffffffffu, l, d), s, e;
    two_sum(h, oh, s, e);
    e += l + ol;
    h = s + e;
    l = e - (h - s);
  }
}

__device__ __forceinline__ long long warp_minmax64(long long x, bool is_min) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    long long o = __shfl_xor_sync(0xffffffffu, x, d);
    x = is_min ? min(x, o) : max(x, o);
  }
  return x;
}

// per-warp running totals of one (group, op): integer sums as (lo, hi) of a
// 128-bit value, Float64 sums as (hi, lo) doubles, MIN/MAX keys and
// non-null counts in w[0]
struct TinyAcc {
  unsigned long long w[2];
};

template <class E, int G, int NOPS, bool F64>
__device__ __forceinline__ void tiny_body(const AggArgs& a) {
  constexpr int WARPS = TINY_BLOCK / 32;
  __shared__ TinyAcc acc[WARPS][G][NOPS];
  __shared__ unsigned long long cnt[WARPS][G];
  __shared__ DCol scols[TINY_MAX_COLS];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const bool shared_cols = a.n_cols <= TINY_MAX_COLS;
  if (shared_cols && threadIdx.x < a.n_cols) scols[threadIdx.x] = a.cols[threadIdx.x];
  if (lane == 0) {
#pragma unroll
    for (int g = 0; g < G; ++g) {
      cnt[wid][g] = 0;
#pragma unroll
      for (int j = 0; j < NOPS; ++j) {
        int kind = E::kind(a, j);
        acc[wid][g][j].w[0] = kind == O_MIN ? 0x7fffffffffffffffULL : kind == O_MAX ? 0x8000000000000000ULL : 0ULL;
        acc[wid][g][j].w[1] = 0;
      }
    }
  }
  __syncthreads();
  const DCol* cols = shared_cols ? scols : a.cols;
  const typename E::Consts K = E::load(a);
  uint32_t seen = 0;  // groups this warp has met (rows arrive in increasing order)
  const int64_t gw = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t base = gw * 32 * TINY_R; base < a.n; base += nw * 32 * TINY_R) {
    int gid[TINY_R];
    Val v[TINY_R][NOPS];
#pragma unroll
    for (int r = 0; r < TINY_R; ++r) {
      int64_t idx = base + r * 32 + lane;
      bool keep = idx < a.n && E::keep(a, K, cols, idx);
      gid[r] = -1;
      if (keep) {
        int g = E::gid(a, K, cols, idx);
        if (g < 0 || g >= G) atomicOr(a.err, DERR_RANGE);
        else gid[r] = g;
      }
#pragma unroll
      for (int j = 0; j < NOPS; ++j) {
        if (gid[r] >= 0) {
          v[r][j] = E::value(a, K, j, cols, idx);
        } else {
          v[r][j].i = 0;
          v[r][j].f = 0;
          v[r][j].valid = false;
        }
      }
    }
#pragma unroll
    for (int r = 0; r < TINY_R; ++r) {
#pragma unroll
      for (int g = 0; g < G; ++g) {
        const unsigned m = __ballot_sync(0xffffffffu, gid[r] == g);
        if (m == 0) continue;  // warp-uniform
        const bool mine = gid[r] == g;
        if (lane == 0) {
          cnt[wid][g] += (unsigned long long)__popc(m);
          if (!((seen >> g) & 1u)) atomicMin(&a.gfirst[g], a.row_base + (uint64_t)(base + r * 32 + __ffs(m) - 1));
        }
        seen |= 1u << g;
#pragma unroll
        for (int j = 0; j < NOPS; ++j) {
          const int kind = E::kind(a, j);
          const Val& x = v[r][j];
          const bool use = mine && !(a.skip_nulls && !x.valid);
          TinyAcc& t = acc[wid][g][j];
          if (kind == O_SUM_INT || kind == O_SUM_DEC) {
            __int128 y = use ? x.i : (__int128)0;
            long long y64 = (long long)y;
            // 32 values below 2^57 in magnitude sum exactly in 64 bits
            bool small = (__int128)y64 == y && y64 > -(1LL << 57) && y64 < (1LL << 57);
            __int128 s = __all_sync(0xffffffffu, small) ? (__int128)warp_sum64(y64) : warp_sum128(y);
            if (lane == 0) {
              unsigned __int128 cur = ((unsigned __int128)t.w[1] << 64) | t.w[0];
              cur += (unsigned __int128)s;
              t.w[0] = (unsigned long long)cur;
              t.w[1] = (unsigned long long)(cur >> 64);
            }
          } else if (kind == O_SUM_F64) {
            if (F64) {
              double y = use ? x.f : 0.0;
              if (!isfinite(y)) {  // NaN / inf: flag straight into the global accumulator
                uint64_t u = (uint64_t)__double_as_longlong(y);
                atomicOr(a.gacc + (size_t)g * a.W + a.op[j].word + LIMBS, isnan(y) ? 1ULL : ((u >> 63) ? 4ULL : 2ULL));
                y = 0.0;
              }
              double h = y, l = 0.0;
              warp_sum_dd(h, l);
              if (lane == 0) {
                double th = __longlong_as_double((long long)t.w[0]), tl = __longlong_as_double((long long)t.w[1]);
                double s1, e1;
                two_sum(th, h, s1, e1);
                e1 += tl + l;
                double nh = s1 + e1;
                t.w[0] = (unsigned long long)__double_as_longlong(nh);
                t.w[1] = (unsigned long long)__double_as_longlong(e1 - (nh - s1));
              }
            }
          } else if (kind == O_MIN || kind == O_MAX) {
            const bool is_min = kind == O_MIN;
            long long key = (use && !isnan(x.f)) ? (long long)total_key(x.f)
                                                 : (is_min ? 0x7fffffffffffffffLL : (long long)0x8000000000000000ULL);
            key = warp_minmax64(key, is_min);
            if (lane == 0) t.w[0] = (unsigned long long)(is_min ? min((long long)t.w[0], key) : max((long long)t.w[0], key));
          } else if (kind == O_NONNULL) {
            unsigned mv = __ballot_sync(0xffffffffu, mine && x.valid);
            if (lane == 0) t.w[0] += (unsigned long long)__popc(mv);
          }
        }
      }
    }
  }
  __syncwarp();
  // lane 0 of each warp merges the warp's totals into the global words
  if (lane == 0) {
#pragma unroll
    for (int g = 0; g < G; ++g) {
      unsigned long long* accg = a.gacc + (size_t)g * a.W;
      if (a.count_rows) atom_add(accg, cnt[wid][g]);
#pragma unroll
      for (int j = 0; j < NOPS; ++j) {
        const int kind = E::kind(a, j);
        const TinyAcc& t = acc[wid][g][j];
        unsigned long long* w = accg + a.op[j].word;
        if (kind == O_SUM_INT || kind == O_SUM_DEC) {
          __int128 x = (__int128)(((unsigned __int128)t.w[1] << 64) | t.w[0]);
          add_i128_limbs(w, x, kind == O_SUM_INT ? 2 : 4);
        } else if (kind == O_SUM_F64) {
          if (F64) {  // both parts exactly into the fixed-point window
            add_f64(w, __longlong_as_double((long long)t.w[0]), a.op[j].lo_exp, a.err, a.maxexp + j);
            add_f64(w, __longlong_as_double((long long)t.w[1]), a.op[j].lo_exp, a.err, a.maxexp + j);
          }
        } else if (kind == O_MIN) {
          if ((long long)t.w[0] != 0x7fffffffffffffffLL) atomicMin((long long*)w, (long long)t.w[0]);
        } else if (kind == O_MAX) {
          if ((long long)t.w[0] != (long long)0x8000000000000000ULL) atomicMax((long long*)w, (long long)t.w[0]);
        } else if (kind == O_NONNULL) {
          atom_add(w, t.w[0]);
        }
      }
    }
  }
}

}  // namespace prism
