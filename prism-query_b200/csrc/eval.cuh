// eval.cuh — typed device programs for predicates and scalar expressions.
//
// The host compiles a prism_predicate / prism_expr (post-order trees) into a
// flat, statically typed program (plan.cpp); every thread of a warp runs the
// same node sequence, so the interpreter branches uniformly. Semantics follow
// the reference:
//   predicates  native/prism-executor/src/filter_project.rs:65-123, 346-404
//     (comparison result null when the column is null; AND/OR null when either
//      side is null; NOT keeps null; floats compare by IEEE totalOrder as
//      arrow-ord does)
//   expressions filter_project.rs:216-294 (F64: both operands cast to
//      Float64; EXACT: integer/decimal operands in 128-bit integers).
#pragma once

#include "common.cuh"

namespace prism {

enum POp : int32_t {
  P_LIT = 0,
  P_CMP_INT,   // integer-like column vs i64 literal
  P_CMP_F64,   // Float64 column vs f64 literal, totalOrder
  P_CMP_STR,   // Utf8 column vs bytes literal
  P_IS_NULL,
  P_IS_NOT_NULL,
  P_AND,
  P_OR,
  P_NOT,
  P_LIKE,
};
enum CmpOp : int32_t { C_EQ = 1, C_NE, C_LT, C_LE, C_GT, C_GE };

struct PNode {
  int32_t op;
  int32_t col;   // index into the program's column table
  int32_t cmp;   // CmpOp (P_CMP_*), case-insensitive flag (P_LIKE)
  int32_t slen;
  int64_t i;     // int literal / bool literal
  double f;      // f64 literal
  const uint8_t* s;  // device bytes (utf8 literal / LIKE pattern)
};

enum EOp : int32_t {
  E_COL_F64 = 0,  // push cast-to-f64 of column
  E_COL_I128,     // push exact integer/decimal of column
  E_LIT_F64,
  E_LIT_I128,
  E_ADD_F, E_SUB_F, E_MUL_F, E_DIV_F, E_NEG_F,
  E_ADD_I, E_SUB_I, E_MUL_I, E_NEG_I,
  E_I2F,          // int128 (scale = `col`) -> f64 value / 10^scale
  E_SCALE_I,      // multiply the top int128 by 10^`col`
  E_SELECT,       // IfThen over numeric branches: pops else (if any) then n thens
  E_F2I,          // f64 -> int128, truncating toward zero; NaN / outside Int64 -> null
};

struct ENode {
  int32_t op;
  int32_t col;        // column index / scale / n_clauses
  int32_t a;          // E_SELECT: has_else; E_COL_*: 1 = keep a null row's raw slot
                      // (a same-typed IfThen branch, which arrow does not cast)
  int32_t b;          // E_SELECT: first clause
  double f;
  int64_t lo, hi;     // i128 literal
};

struct PRange {
  int32_t begin, len;
};

constexpr int EVAL_STACK = 16;

struct Val {
  __int128 i;
  double f;
  bool valid;
};

__device__ __forceinline__ bool cmp_apply(int op, int c) {  // c = sign of (a - b)
  switch (op) {
    case C_EQ: return c == 0;
    case C_NE: return c != 0;
    case C_LT: return c < 0;
    case C_LE: return c <= 0;
    case C_GT: return c > 0;
    default: return c >= 0;
  }
}

__device__ __forceinline__ int bytes_cmp(const uint8_t* a, int32_t na, const uint8_t* b, int32_t nb) {
  int32_t n = na < nb ? na : nb;
  for (int32_t i = 0; i < n; ++i)
    if (a[i] != b[i]) return a[i] < b[i] ? -1 : 1;
  return na == nb ? 0 : (na < nb ? -1 : 1);
}

// SQL LIKE: '%' any run, '_' one UTF-8 code point, '\\' escapes the next
// character; iterative matcher with backtracking to the last '%'.
__device__ inline bool like_match(const uint8_t* s, int32_t ns, const uint8_t* p, int32_t np, bool ci) {
  auto low = [&](uint8_t c) -> uint8_t { return (ci && c >= 'A' && c <= 'Z') ? (uint8_t)(c + 32) : c; };
  auto cplen = [](uint8_t c) -> int32_t {
    if (c < 0x80) return 1;
    if ((c >> 5) == 6) return 2;
    if ((c >> 4) == 14) return 3;
    return 4;
  };
  int32_t si = 0, pi = 0, star_p = -1, star_s = 0;
  while (si < ns) {
    if (pi < np) {
      uint8_t pc = p[pi];
      if (pc == '%') { star_p = ++pi; star_s = si; continue; }
      if (pc == '_') { si += cplen(s[si]); ++pi; continue; }
      if (pc == '\\' && pi + 1 < np) {
        if (low(s[si]) == low(p[pi + 1])) { ++si; pi += 2; continue; }
      } else if (low(s[si]) == low(pc)) { ++si; ++pi; continue; }
    }
    if (star_p >= 0) {
      star_s += cplen(s[star_s]);
      si = star_s;
      pi = star_p;
      continue;
    }
    return false;
  }
  while (pi < np && p[pi] == '%') ++pi;
  return pi == np;
}

// Evaluates predicate nodes [begin, begin+len); returns value bit, sets valid.
__device__ inline bool eval_pred(const PNode* nodes, int begin, int len, const DCol* cols, int64_t row, bool& valid) {
  uint32_t vs = 0, ok = 0;  // bit stacks (depth <= 32)
  int sp = 0;
  for (int k = begin; k < begin + len; ++k) {
    const PNode& nd = nodes[k];
    bool v = false, va = true;
    switch (nd.op) {
      case P_LIT: v = nd.i != 0; break;
      case P_CMP_INT: {
        const DCol& c = cols[nd.col];
        va = dcol_valid(c, row);
        int64_t x = dcol_ival(c, row);
        v = cmp_apply(nd.cmp, x < nd.i ? -1 : (x > nd.i ? 1 : 0));
        break;
      }
      case P_CMP_F64: {
        const DCol& c = cols[nd.col];
        va = dcol_valid(c, row);
        int64_t x = total_key(static_cast<const double*>(c.values)[row]);
        int64_t y = total_key(nd.f);
        v = cmp_apply(nd.cmp, x < y ? -1 : (x > y ? 1 : 0));
        break;
      }
      case P_CMP_STR: {
        const DCol& c = cols[nd.col];
        va = dcol_valid(c, row);
        const uint8_t* p;
        int32_t n;
        dcol_str(c, row, p, n);
        v = cmp_apply(nd.cmp, bytes_cmp(p, n, nd.s, nd.slen));
        break;
      }
      case P_IS_NULL: v = !dcol_valid(cols[nd.col], row); break;
      case P_IS_NOT_NULL: v = dcol_valid(cols[nd.col], row); break;
      case P_LIKE: {
        const DCol& c = cols[nd.col];
        va = dcol_valid(c, row);
        const uint8_t* p;
        int32_t n;
        dcol_str(c, row, p, n);
        v = like_match(p, n, nd.s, nd.slen, nd.cmp != 0);
        break;
      }
      case P_AND: case P_OR: {
        bool rb = vs & 1, rv = ok & 1;
        bool lb = (vs >> 1) & 1, lv = (ok >> 1) & 1;
        vs >>= 2;
        ok >>= 2;
        sp -= 2;
        v = nd.op == P_AND ? (lb && rb) : (lb || rb);
        va = lv && rv;
        break;
      }
      case P_NOT: {
        bool b = vs & 1, bv = ok & 1;
        vs >>= 1;
        ok >>= 1;
        sp -= 1;
        v = !b;
        va = bv;
        break;
      }
    }
    vs = (vs << 1) | (v ? 1u : 0u);
    ok = (ok << 1) | (va ? 1u : 0u);
    ++sp;
  }
  valid = ok & 1;
  return vs & 1;
}

__device__ __forceinline__ __int128 pow10_i128(int k) {
  __int128 p = 1;
  for (int i = 0; i < k; ++i) p *= 10;
  return p;
}

// Overflow-checked 128-bit integer arithmetic (true when the exact result
// does not fit a signed 128-bit integer).
__device__ __forceinline__ bool add_ovf_i128(__int128 a, __int128 b, __int128& out) {
  out = (__int128)((unsigned __int128)a + (unsigned __int128)b);
  return ((a < 0) == (b < 0)) && ((out < 0) != (a < 0));
}
__device__ __forceinline__ bool sub_ovf_i128(__int128 a, __int128 b, __int128& out) {
  out = (__int128)((unsigned __int128)a - (unsigned __int128)b);
  return ((a < 0) != (b < 0)) && ((out < 0) != (a < 0));
}
__device__ __forceinline__ bool mul_ovf_i128(__int128 a, __int128 b, __int128& out) {
  bool neg = (a < 0) != (b < 0);
  unsigned __int128 ua = a < 0 ? (unsigned __int128)0 - (unsigned __int128)a : (unsigned __int128)a;
  unsigned __int128 ub = b < 0 ? (unsigned __int128)0 - (unsigned __int128)b : (unsigned __int128)b;
  unsigned long long ah = (unsigned long long)(ua >> 64), al = (unsigned long long)ua;
  unsigned long long bh = (unsigned long long)(ub >> 64), bl = (unsigned long long)ub;
  bool ovf = false;
  if (ah && bh) ovf = true;
  unsigned __int128 cross = (unsigned __int128)ah * bl + (unsigned __int128)al * bh;
  if (cross >> 64) ovf = true;
  unsigned __int128 lo = (unsigned __int128)al * bl;
  unsigned __int128 mag = lo + (cross << 64);
  if (mag < lo) ovf = true;
  unsigned __int128 lim = ((unsigned __int128)1 << 127) - (neg ? 0 : 1);
  if (mag > lim) ovf = true;
  out = neg ? (__int128)((unsigned __int128)0 - mag) : (__int128)mag;
  return ovf;
}

// Evaluates expression nodes [begin, end); clause predicates for E_SELECT come
// from `preds`/`clauses`. Sets *ovf on 128-bit overflow.
__device__ inline Val eval_expr(const ENode* nodes, int begin, int end, const PNode* preds, const PRange* clauses,
                                const DCol* cols, int64_t row, bool* ovf) {
  Val st[EVAL_STACK];
  int sp = 0;
  for (int k = begin; k < end; ++k) {
    const ENode& nd = nodes[k];
    switch (nd.op) {
      case E_COL_F64: {
        const DCol& c = cols[nd.col];
        st[sp].f = nd.a ? dcol_fval(c, row) : dcol_fval_cast(c, row);
        st[sp].valid = dcol_valid(c, row);
        ++sp;
        break;
      }
      case E_COL_I128: {
        const DCol& c = cols[nd.col];
        st[sp].i = nd.a ? dcol_i128(c, row) : dcol_i128_cast(c, row);
        st[sp].valid = dcol_valid(c, row);
        ++sp;
        break;
      }
      case E_LIT_F64: st[sp].f = nd.f; st[sp].valid = true; ++sp; break;
      case E_LIT_I128:
        st[sp].i = ((__int128)nd.hi << 64) | (unsigned __int128)(uint64_t)nd.lo;
        st[sp].valid = true;
        ++sp;
        break;
      case E_ADD_F: case E_SUB_F: case E_MUL_F: case E_DIV_F: {
        Val r = st[--sp];
        Val& l = st[sp - 1];
        double x = l.f, y = r.f;
        l.f = nd.op == E_ADD_F ? x + y : nd.op == E_SUB_F ? x - y : nd.op == E_MUL_F ? x * y : x / y;
        l.valid = l.valid && r.valid;
        break;
      }
      case E_NEG_F: st[sp - 1].f = -st[sp - 1].f; break;
      case E_ADD_I: case E_SUB_I: case E_MUL_I: {
        Val r = st[--sp];
        Val& l = st[sp - 1];
        __int128 o;
        bool bad;
        if (nd.op == E_ADD_I) bad = add_ovf_i128(l.i, r.i, o);
        else if (nd.op == E_SUB_I) bad = sub_ovf_i128(l.i, r.i, o);
        else bad = mul_ovf_i128(l.i, r.i, o);
        if (bad && l.valid && r.valid) *ovf = true;
        l.i = o;
        l.valid = l.valid && r.valid;
        break;
      }
      case E_NEG_I: st[sp - 1].i = -st[sp - 1].i; break;
      case E_I2F: {
        double s = 1.0;
        for (int q = 0; q < nd.col; ++q) s *= 10.0;
        st[sp - 1].f = (double)st[sp - 1].i / s;
        break;
      }
      case E_SCALE_I: {
        __int128 o;
        if (mul_ovf_i128(st[sp - 1].i, pow10_i128(nd.col), o) && st[sp - 1].valid) *ovf = true;
        st[sp - 1].i = o;
        break;
      }
      case E_F2I: {
        double x = st[sp - 1].f;
        double t = trunc(x);
        if (!st[sp - 1].valid) {
          st[sp - 1].i = 0;  // a cast leaves 0 in a null row's slot
        } else if (!(t >= -9.223372036854775808e18 && t < 9.223372036854775808e18)) {
          st[sp - 1].valid = false;
          st[sp - 1].i = 0;
        } else {
          st[sp - 1].i = (__int128)(long long)t;
        }
        break;
      }
      case E_SELECT: {
        int nc = nd.col, has_else = nd.a;
        int need = nc + has_else;
        Val res;
        if (has_else) res = st[sp - 1];
        else { res.valid = false; res.i = 0; res.f = 0; }
        int base = sp - need;
        for (int ci = nc - 1; ci >= 0; --ci) {
          bool pv;
          bool pt = eval_pred(preds, clauses[nd.b + ci].begin, clauses[nd.b + ci].len, cols, row, pv);
          if (pv && pt) res = st[base + ci];
        }
        sp = base;
        st[sp++] = res;
        break;
      }
    }
  }
  return st[0];
}

}  // namespace prism
