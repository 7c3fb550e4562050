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
  // few dense groups (tiny_body): input tiles staged into shared memory
  // (every program column fixed width, null-free, 16-byte aligned) or read
  // in place when n_stage == 0
  int32_t n_stage;
  int32_t stage_w[8];
  int32_t stage_off[8];
  int32_t stage_bytes;
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
// or none). Each thread keeps its own accumulators for every group in
// registers: integer-sum partials in int64 that spill exactly into the
// block's shared 128-bit accumulators when a row would overflow them,
// double-double Float64 partials, MIN/MAX totalOrder keys and row counts.
// Rows never contend on shared addresses; at the end each warp reduces with
// shuffles and one lane per warp merges into the block's and then the global
// exact accumulators (the same words agg_kernel fills, so the same finalize
// kernels run). Input tiles stream through a 3-stage shared-memory ring
// filled by cp.async (16-byte chunks, zero-filled tail), so the loads of the
// next tiles are in flight while the current one is evaluated.
//
// E supplies the row logic as straight-line code generated per query
// (jit.cu): E::Consts / E::load (per-thread constants read once), E::keep
// (filter), E::gid (dense group id), E::kind (op kind of j), E::value (op
// j's operand).
constexpr int TINY_BLOCK = 256;  // 8 warps, up to 255 registers a thread
constexpr int TINY_T = 2048;     // rows per tile
constexpr int TINY_STAGES = 3;
constexpr int TINY_MAX_COLS = 8;

__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gsrc, int src_bytes) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gsrc), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_2() { asm volatile("cp.async.wait_group 2;\n" ::: "memory"); }

__device__ __forceinline__ void two_sum(double a, double b, double& s, double& e) {
  s = a + b;
  double bb = s - a;
  e = (a - (s - bb)) + (b - bb);
}

// limbs of an integer-sum op: int64 inputs use 2 (low 32 bits, signed rest),
// 128-bit decimal inputs 4
__device__ __forceinline__ int int_limbs(int kind) { return kind == O_SUM_INT ? 2 : 4; }

// One row's contribution to a thread's accumulator of op j in group g.
template <bool F64>
__device__ __forceinline__ void tiny_apply(const AggArgs& a, int kind, long long& w0, long long& w1, const Val& v,
                                           int j, int g, unsigned long long* sacc) {
  if (a.skip_nulls && !v.valid) return;
  switch (kind) {
    case O_SUM_INT: case O_SUM_DEC: {
      long long x = (long long)v.i;
      long long r = (long long)((unsigned long long)w0 + (unsigned long long)x);
      bool fits = (__int128)x == v.i && !(((w0 ^ r) & (x ^ r)) < 0);
      if (fits) {
        w0 = r;
      } else {  // exact spill of partial + value, partial restarts at 0
        add_i128_limbs(sacc + (g * 8 + j) * 4, (__int128)w0 + v.i, int_limbs(kind));
        w0 = 0;
      }
      break;
    }
    case O_SUM_F64:
      if (F64) {
        if (!isfinite(v.f)) {  // NaN / inf: flag straight into the global accumulator
          uint64_t u = (uint64_t)__double_as_longlong(v.f);
          atomicOr(a.gacc + (size_t)g * a.W + a.op[j].word + LIMBS, isnan(v.f) ? 1ULL : ((u >> 63) ? 4ULL : 2ULL));
          break;
        }
        double s, e;
        two_sum(__longlong_as_double(w0), v.f, s, e);
        w0 = __double_as_longlong(s);
        w1 = __double_as_longlong(__longlong_as_double(w1) + e);
      }
      break;
    case O_MIN:
      if (!isnan(v.f)) w0 = min(w0, (long long)total_key(v.f));
      break;
    case O_MAX:
      if (!isnan(v.f)) w0 = max(w0, (long long)total_key(v.f));
      break;
    case O_NONNULL:
      w0 += v.valid ? 1 : 0;
      break;
  }
}

// issues the asynchronous copies of tile t into ring stage `stage` (always
// commits a group, empty past the last tile, so group counting stays uniform)
__device__ __forceinline__ void tiny_issue(const AggArgs& a, int64_t t, int stage, int64_t n_tiles,
                                           unsigned char* ring) {
  if (t < n_tiles) {
    int64_t r0 = t * TINY_T;
    int64_t rows = a.n - r0 < TINY_T ? a.n - r0 : TINY_T;
    unsigned char* sb = ring + (size_t)stage * a.stage_bytes;
    for (int k = 0; k < a.n_stage; ++k) {
      int w = a.stage_w[k];
      const unsigned char* src = static_cast<const unsigned char*>(a.cols[k].values) + r0 * w;
      unsigned char* dst = sb + a.stage_off[k];
      int bytes = (int)(rows * w);
      int chunks = (bytes + 15) >> 4;
      for (int c = threadIdx.x; c < chunks; c += blockDim.x) {
        int rem = bytes - (c << 4);
        cp_async16(dst + (c << 4), src + (c << 4), rem >= 16 ? 16 : rem);
      }
    }
  }
  cp_async_commit();
}

__device__ __forceinline__ long long shfl64(long long x, int d) { return __shfl_xor_sync(0xffffffffu, x, d); }

template <class E, int G, int NOPS, bool F64>
__device__ __forceinline__ void tiny_body(const AggArgs& a) {
  extern __shared__ __align__(16) unsigned char tiny_smem[];
  __shared__ unsigned long long sfirst[G];
  __shared__ unsigned long long sacc[G * 8 * 4];  // exact spill-over of integer sums
  __shared__ DCol shadow[TINY_STAGES][TINY_MAX_COLS];
  const bool staged = a.n_stage > 0;
  if (threadIdx.x < G) sfirst[threadIdx.x] = ~0ULL;
  for (int q = threadIdx.x; q < G * 8 * 4; q += blockDim.x) sacc[q] = 0;
  if (staged && threadIdx.x < TINY_STAGES * a.n_cols) {
    int st = threadIdx.x / a.n_cols, k = threadIdx.x % a.n_cols;
    DCol d = a.cols[k];
    d.values = tiny_smem + (size_t)st * a.stage_bytes + a.stage_off[k];
    shadow[st][k] = d;
  }
  uint32_t cnt[G];
  long long w0[G][NOPS], w1[G][F64 ? NOPS : 1];
#pragma unroll
  for (int g = 0; g < G; ++g) {
    cnt[g] = 0;
#pragma unroll
    for (int j = 0; j < NOPS; ++j) {
      int kind = E::kind(a, j);
      w0[g][j] = kind == O_MIN ? 0x7fffffffffffffffLL : kind == O_MAX ? (long long)0x8000000000000000ULL : 0LL;
      if (F64) w1[g][j] = 0;
    }
  }
  uint32_t seen = 0;
  const typename E::Consts K = E::load(a);
  __syncthreads();

  const int64_t n_tiles = (a.n + TINY_T - 1) / TINY_T;
  int64_t my = 0;  // k-th tile of this CTA: blockIdx.x + k * gridDim.x
  if (staged) {
    tiny_issue(a, blockIdx.x, 0, n_tiles, tiny_smem);
    tiny_issue(a, blockIdx.x + gridDim.x, 1, n_tiles, tiny_smem);
  }
  for (int64_t t = blockIdx.x; t < n_tiles; t += gridDim.x, ++my) {
    const int stage = (int)(my % TINY_STAGES);
    const DCol* cols = a.cols;
    int64_t r0 = t * TINY_T;
    int64_t base = r0;  // row index base passed to the row logic
    if (staged) {
      tiny_issue(a, t + 2 * (int64_t)gridDim.x, (int)((my + 2) % TINY_STAGES), n_tiles, tiny_smem);
      cp_async_wait_2();
      __syncthreads();
      cols = shadow[stage];
      base = 0;
    }
    int64_t rows = a.n - r0 < TINY_T ? a.n - r0 : TINY_T;
    for (int64_t i = threadIdx.x; i < rows; i += blockDim.x) {
      int64_t idx = base + i;
      if (!E::keep(a, K, cols, idx)) continue;
      int gid = E::gid(a, K, cols, idx);
      if (gid < 0 || gid >= G) {
        atomicOr(a.err, DERR_RANGE);
        continue;
      }
      uint64_t grow = a.row_base + (uint64_t)(r0 + i);
#pragma unroll
      for (int g = 0; g < G; ++g) {
        if (gid != g) continue;
        cnt[g] += 1;
        if (!((seen >> g) & 1u)) {
          seen |= 1u << g;
          atomicMin(&sfirst[g], grow);
        }
      }
      // one operand live at a time: evaluate op j's operand, fold it into
      // the row's group, move on
#pragma unroll
      for (int j = 0; j < NOPS; ++j) {
        Val v = E::value(a, K, j, cols, idx);
        int kind = E::kind(a, j);
#pragma unroll
        for (int g = 0; g < G; ++g)
          if (gid == g) tiny_apply<F64>(a, kind, w0[g][j], w1[g][F64 ? j : 0], v, j, g, sacc);
      }
    }
    if (staged) __syncthreads();  // the stage is refilled next iteration
  }
  if (staged) asm volatile("cp.async.wait_all;\n" ::: "memory");
  // warp reduction (integer partials widened to 128 bits), then lane 0
  // merges into the block's shared accumulators / the global words
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int g = 0; g < G; ++g) {
    unsigned long long c64 = cnt[g];
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) c64 += (unsigned long long)shfl64((long long)c64, d);
    unsigned long long* acc = a.gacc + (size_t)g * a.W;
    if (lane == 0 && a.count_rows) atom_add(acc, c64);
#pragma unroll
    for (int j = 0; j < NOPS; ++j) {
      int kind = E::kind(a, j);
      unsigned long long* w = acc + a.op[j].word;
      if (kind == O_SUM_INT || kind == O_SUM_DEC) {
        long long hi = w0[g][j] < 0 ? -1 : 0, lo = w0[g][j];
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
          long long olo = shfl64(lo, d), ohi = shfl64(hi, d);
          unsigned __int128 s = (((unsigned __int128)(unsigned long long)hi << 64) | (unsigned long long)lo) +
                                (((unsigned __int128)(unsigned long long)ohi << 64) | (unsigned long long)olo);
          lo = (long long)(unsigned long long)s;
          hi = (long long)(unsigned long long)(s >> 64);
        }
        if (lane == 0)
          add_i128_limbs(sacc + (g * 8 + j) * 4,
                         (__int128)(((unsigned __int128)(unsigned long long)hi << 64) | (unsigned long long)lo),
                         int_limbs(kind));
      } else if (kind == O_SUM_F64) {
        if (F64) {
          double h = __longlong_as_double(w0[g][j]), l = __longlong_as_double(w1[g][F64 ? j : 0]);
#pragma unroll
          for (int d = 16; d > 0; d >>= 1) {
            double oh = __shfl_xor_sync(0xffffffffu, h, d), ol = __shfl_xor_sync(0xffffffffu, l, d), s, e;
            two_sum(h, oh, s, e);
            e += l + ol;
            h = s + e;
            l = e - (h - s);
          }
          if (lane == 0) {  // both parts exactly into the fixed-point window
            add_f64(w, h, a.op[j].lo_exp, a.err, a.maxexp + j);
            add_f64(w, l, a.op[j].lo_exp, a.err, a.maxexp + j);
          }
        }
      } else {
        long long v = w0[g][j];
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
          long long o = shfl64(v, d);
          v = kind == O_MIN ? min(v, o) : kind == O_MAX ? max(v, o) : v + o;
        }
        if (lane == 0) {
          if (kind == O_MIN && v != 0x7fffffffffffffffLL) atomicMin((long long*)w, v);
          else if (kind == O_MAX && v != (long long)0x8000000000000000ULL) atomicMax((long long*)w, v);
          else if (kind == O_NONNULL) atom_add(w, (unsigned long long)v);
        }
      }
    }
  }
  __syncthreads();
  if (threadIdx.x < G && sfirst[threadIdx.x] != ~0ULL) atomicMin(&a.gfirst[threadIdx.x], sfirst[threadIdx.x]);
  // the block's exact integer sums into the global limbs
  for (int q = threadIdx.x; q < G * 8 * 4; q += blockDim.x) {
    int g = q / 32, j = (q / 4) % 8, limb = q % 4;
    if (j < NOPS) {
      int kind = E::kind(a, j);
      if ((kind == O_SUM_INT || kind == O_SUM_DEC) && limb < int_limbs(kind))
        atom_add(a.gacc + (size_t)g * a.W + a.op[j].word + limb, sacc[q]);
    }
  }
}

}  // namespace prism
