// filter_project.cu — predicate masks, ordered compaction and projections.
//
// evaluate_predicate (filter_project.rs:65-123) produces one Boolean column
// in a single pass over the referenced columns (the reference builds one
// BooleanArray per tree node). filter_batch (:126-135) keeps rows whose mask
// bit is true and valid, in order, via a popcount scan of the mask words.
// project_batch_with_exprs (:305-333) evaluates each expression in one pass.
#include "filter_project.hpp"
#include "prims.hpp"

namespace prism {

namespace {

// One warp evaluates 32 consecutive rows; ballots write whole mask words.
__global__ void predicate_kernel(const PNode* pn, PRange r, const DCol* cols, int64_t n, uint32_t* vals,
                                 uint32_t* valid) {
  int64_t total = (n + 31) & ~int64_t(31);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    bool v = false, ok = false;
    if (i < n) v = eval_pred(pn, r.begin, r.len, cols, i, ok);
    uint32_t wv = __ballot_sync(0xffffffffu, v);
    uint32_t wk = __ballot_sync(0xffffffffu, ok);
    if ((threadIdx.x & 31) == 0) {
      vals[i >> 5] = wv;
      valid[i >> 5] = wk;
    }
  }
}

__global__ void and_bits_kernel(const uint8_t* a, const uint8_t* b, int64_t nbytes, uint8_t* out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nbytes; i += (int64_t)gridDim.x * blockDim.x)
    out[i] = a[i] & (b ? b[i] : 0xff);
}

// Expression column: result kind 0 = f64, 1 = dec128, 2 = cast to fixed
// target (`out_type`) from the program's value (int128 or f64 domain).
__global__ void expr_kernel(const ENode* en, int begin, int end, const PNode* pn, const PRange* cl, const DCol* cols,
                            int64_t n, int kind, int out_type, int from_int, void* out, uint32_t* valid_words,
                            uint32_t* err) {
  int64_t total = (n + 31) & ~int64_t(31);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    bool ok = false;
    if (i < n) {
      bool ovf = false;
      Val v = eval_expr(en, begin, end, pn, cl, cols, i, &ovf);
      if (ovf) atomicOr(err, DERR_RANGE);
      ok = v.valid;
      // null rows keep the slot the reference leaves there: arithmetic fills
      // every slot from the operands' slots, casts leave 0, a same-typed
      // IfThen branch passes its raw slot through
      if (kind == 0) {
        static_cast<double*>(out)[i] = v.f;
      } else if (kind == 1) {
        __int128 x = v.i;
        unsigned long long* p = static_cast<unsigned long long*>(out) + 2 * i;
        p[0] = (unsigned long long)x;
        p[1] = (unsigned long long)(x >> 64);
      } else {
        // arrow safe cast into the target type: out-of-range -> null (slot 0)
        __int128 x;
        bool rep = true;
        if (from_int) x = v.i;
        else {
          double t = trunc(v.f);
          if (!(t >= -9.223372036854775808e18 && t < 9.223372036854775808e18)) rep = false;
          x = rep ? (__int128)(long long)t : 0;
        }
        if (out_type == TY_F32) {
          static_cast<float*>(out)[i] = (float)(from_int ? (double)v.i : v.f);
        } else {
          __int128 lo, hi;
          switch (out_type) {
            case TY_I8: lo = -128; hi = 127; break;
            case TY_I16: lo = -32768; hi = 32767; break;
            case TY_I32: case TY_DATE32: lo = INT32_MIN; hi = INT32_MAX; break;
            case TY_U8: lo = 0; hi = 255; break;
            case TY_U16: lo = 0; hi = 65535; break;
            case TY_U32: lo = 0; hi = UINT32_MAX; break;
            case TY_U64: lo = 0; hi = (__int128)UINT64_MAX; break;
            case TY_BOOL: lo = 0; hi = 1; break;
            default: lo = INT64_MIN; hi = INT64_MAX;
          }
          if (rep && (x < lo || x > hi)) {
            if (out_type == TY_BOOL) x = x != 0;  // numeric -> bool: non-zero is true
            else rep = false;
          }
          if (!rep) {
            x = 0;
            ok = false;
          }
          switch (out_type) {
            case TY_I8: case TY_U8: static_cast<int8_t*>(out)[i] = (int8_t)x; break;
            case TY_I16: case TY_U16: static_cast<int16_t*>(out)[i] = (int16_t)x; break;
            case TY_I32: case TY_U32: case TY_DATE32: static_cast<int32_t*>(out)[i] = (int32_t)x; break;
            case TY_BOOL: static_cast<uint8_t*>(out)[i] = (uint8_t)(x != 0); break;  // packed later
            default: static_cast<int64_t*>(out)[i] = (int64_t)x;
          }
        }
      }
    }
    uint32_t w = __ballot_sync(0xffffffffu, ok);
    if ((threadIdx.x & 31) == 0) valid_words[i >> 5] = w;
  }
}

// Utf8 IfThen: index of the chosen branch per row (n_clauses = else / null)
__global__ void str_select_kernel(const PNode* pn, const PRange* cl, int clause_begin, int n_clauses, const DCol* cols,
                                  int64_t n, int32_t* choice) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    int32_t c = n_clauses;
    for (int k = 0; k < n_clauses; ++k) {
      bool ok;
      bool v = eval_pred(pn, cl[clause_begin + k].begin, cl[clause_begin + k].len, cols, i, ok);
      if (ok && v) { c = k; break; }
    }
    choice[i] = c;
  }
}

struct StrBranch {
  const int32_t* offs;  // null for literal
  const uint8_t* data;  // data + offs[i] addresses row i (columns); literal bytes
  const uint8_t* valid;
  int32_t lit_len;
};
struct StrBranches {
  int32_t n;          // branches incl. else
  int32_t has_else;
  StrBranch b[17];
};

__device__ __forceinline__ bool branch_row(const StrBranches& s, int32_t c, int64_t i, const uint8_t*& p, int32_t& len) {
  if (c >= s.n) { p = nullptr; len = 0; return false; }
  const StrBranch& b = s.b[c];
  if (!b.offs) { p = b.data; len = b.lit_len; return true; }
  if (b.valid && !((b.valid[i >> 3] >> (i & 7)) & 1)) { p = nullptr; len = 0; return false; }
  p = b.data + b.offs[i];
  len = b.offs[i + 1] - b.offs[i];
  return true;
}

__global__ void str_select_len_kernel(StrBranches s, const int32_t* choice, int64_t n, uint32_t* len, uint32_t* vwords) {
  int64_t total = (n + 31) & ~int64_t(31);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < total; i += (int64_t)gridDim.x * blockDim.x) {
    bool ok = false;
    if (i < n) {
      int32_t c = choice[i];  // == n_clauses: the else branch, or null without one
      const uint8_t* p;
      int32_t l;
      ok = branch_row(s, c, i, p, l);
      len[i] = ok ? (uint32_t)l : 0u;
    }
    uint32_t w = __ballot_sync(0xffffffffu, ok);
    if ((threadIdx.x & 31) == 0) vwords[i >> 5] = w;
  }
}

__global__ void str_select_copy_kernel(StrBranches s, const int32_t* choice, int64_t n, const uint64_t* off,
                                       int32_t* out_offs, uint8_t* out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    out_offs[i] = (int32_t)off[i];
    int32_t c = choice[i];
    const uint8_t* p;
    int32_t l;
    if (!branch_row(s, c, i, p, l)) continue;
    for (int32_t k = 0; k < l; ++k) out[off[i] + k] = p[k];
  }
}

template <class T>
__global__ void fill_kernel(T* out, int64_t n, T v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) out[i] = v;
}

__global__ void fill_str_kernel(int32_t* offs, uint8_t* data, int64_t n, const uint8_t* lit, int32_t len) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= n; i += (int64_t)gridDim.x * blockDim.x) {
    offs[i] = (int32_t)(i * len);
    if (i < n)
      for (int32_t k = 0; k < len; ++k) data[i * len + k] = lit[k];
  }
}

}  // namespace

ColP evaluate_predicate(Ctx& ctx, const Batch& b, const prism_predicate& pred) {
  Program p = compile_program(b, &pred, nullptr, 0, PRISM_ARITH_F64);
  int64_t n = b.rows;
  ColP out = make_column(ctx, TY_BOOL, "mask", n, true);
  if (n > 0) {
    upload_program(ctx, p, b);
    predicate_kernel<<<grid_for(ctx, n, 256), 256, 0, ctx.stream>>>(p.d_pnodes, p.filter, p.d_cols, n,
                                                                      reinterpret_cast<uint32_t*>(out->values),
                                                                      reinterpret_cast<uint32_t*>(out->validity));
    ctx.check_launch("predicate_kernel");
    ctx.sync();  // the program buffer is released on return
  }
  return out;
}

MemP mask_rows(Ctx& ctx, const Column& mask, int64_t* count) {
  if (mask.type != TY_BOOL) fail(PRISM_ERR_INVALID_ARGUMENT, "filter mask must be a Boolean column");
  int64_t n = mask.length;
  const uint8_t* bits = static_cast<const uint8_t*>(mask.values);
  MemP tmp;
  if (mask.validity) {
    int64_t nbytes = (n + 7) / 8;
    uint8_t* t = ctx.alloc_t<uint8_t>((size_t)nbytes + 8, tmp);
    if (nbytes) {
      and_bits_kernel<<<grid_for(ctx, nbytes, 256), 256, 0, ctx.stream>>>(bits, mask.validity, nbytes, t);
      ctx.check_launch("and_bits_kernel");
    }
    bits = t;
  }
  MemP rows = compact_bits(ctx, bits, n, false, count);
  ctx.sync();
  return rows;
}

Batch filter_rows(Ctx& ctx, const Batch& b, const uint32_t* rows, int64_t n) {
  Batch out;
  out.rows = n;
  for (auto& c : b.cols) out.cols.push_back(filter_column(ctx, *c, rows, n));
  return out;
}

Batch filter_by_mask(Ctx& ctx, const Batch& b, const Column& mask) {
  if (mask.length != b.rows) fail(PRISM_ERR_INVALID_ARGUMENT, "mask length differs from the batch");
  int64_t n = 0;
  MemP rows = mask_rows(ctx, mask, &n);
  return filter_rows(ctx, b, static_cast<const uint32_t*>(rows->ptr), n);
}

Batch project(const Batch& b, const int32_t* cols, int n_cols) {
  Batch out;
  out.rows = b.rows;
  for (int i = 0; i < n_cols; ++i) {
    if (cols[i] < 0 || cols[i] >= (int)b.cols.size())
      fail(PRISM_ERR_INVALID_ARGUMENT, "column index " + std::to_string(cols[i]) + " out of range");
    out.cols.push_back(b.cols[cols[i]]);
  }
  return out;
}

static ColP literal_column(Ctx& ctx, const CompiledExpr& ce, int64_t n) {
  int g = grid_for(ctx, std::max<int64_t>(n, 1), 256);
  if (ce.out_type == TY_UTF8) {
    int64_t len = (int64_t)ce.literal_str.size();
    if (len * n > INT32_MAX) fail(PRISM_ERR_ARROW, "Utf8 literal column exceeds 2 GiB");
    ColP c = make_utf8_column(ctx, "", n, len * n, false);
    MemP ml = ctx.alloc(len + 1);
    PRISM_CUDA(cudaMemcpyAsync(ml->ptr, ce.literal_str.data(), len, cudaMemcpyHostToDevice, ctx.stream));
    fill_str_kernel<<<g, 256, 0, ctx.stream>>>(c->offsets, c->data, n, static_cast<uint8_t*>(ml->ptr), (int32_t)len);
    ctx.check_launch("fill_str_kernel");
    ctx.sync();
    return c;
  }
  ColP c = make_column(ctx, ce.out_type, "", n, false);
  if (n == 0) return c;
  switch (ce.out_type) {
    case TY_F64: fill_kernel<double><<<g, 256, 0, ctx.stream>>>((double*)c->values, n, ce.literal.f64); break;
    case TY_I64: fill_kernel<int64_t><<<g, 256, 0, ctx.stream>>>((int64_t*)c->values, n, ce.literal.i64); break;
    case TY_I32: case TY_DATE32: fill_kernel<int32_t><<<g, 256, 0, ctx.stream>>>((int32_t*)c->values, n, (int32_t)ce.literal.i64); break;
    case TY_BOOL: {
      uint32_t w = ce.literal.i64 ? 0xffffffffu : 0u;
      fill_kernel<uint32_t><<<g, 256, 0, ctx.stream>>>((uint32_t*)c->values, (n + 31) / 32, w);
      break;
    }
    default: fail(PRISM_ERR_INTERNAL, "literal type");
  }
  ctx.check_launch("fill_kernel");
  return c;
}

Batch project_with_exprs(Ctx& ctx, const Batch& b, const int32_t* cols, int n_cols, const prism_expr* exprs,
                         int n_exprs, int arith_mode) {
  Batch out = project(b, cols, n_cols);
  if (n_exprs == 0) return out;
  Program p = compile_program(b, nullptr, exprs, n_exprs, arith_mode);
  int64_t n = b.rows;
  upload_program(ctx, p, b);
  int g = grid_for(ctx, std::max<int64_t>(n, 1), 256);
  for (int e = 0; e < n_exprs; ++e) {
    const CompiledExpr& ce = p.exprs[e];
    std::string name = "expr_" + std::to_string(e);
    ColP c;
    switch (ce.kind) {
      case EK_COLUMN: {
        auto cc = std::make_shared<Column>(*b.cols[ce.column]);
        c = cc;
        break;
      }
      case EK_LITERAL:
        c = literal_column(ctx, ce, n);
        break;
      case EK_F64: case EK_DEC: case EK_CAST: {
        int kind = ce.kind == EK_F64 ? 0 : ce.kind == EK_DEC ? 1 : 2;
        int out_type = ce.kind == EK_F64 ? TY_F64 : ce.kind == EK_DEC ? TY_DEC128 : ce.out_type;
        int store_type = out_type == TY_BOOL ? TY_U8 : out_type;
        c = make_column(ctx, store_type, name, n, true);
        if (out_type == TY_DEC128) { c->precision = 38; c->scale = ce.scale; }
        // EK_CAST computes in the int128 domain unless the target is a float type
        int from_int = (ce.kind == EK_CAST && out_type != TY_F32) ? 1 : 0;
        if (n) {
          expr_kernel<<<g, 256, 0, ctx.stream>>>(p.d_enodes, ce.begin, ce.end, p.d_pnodes, p.d_clauses, p.d_cols, n, kind,
                                                  out_type, from_int, c->values, reinterpret_cast<uint32_t*>(c->validity),
                                                  ctx.d_err);
          ctx.check_launch("expr_kernel");
        }
        if (out_type == TY_BOOL) {  // pack bytes into a Boolean bitmap
          ColP bc = make_column(ctx, TY_BOOL, name, n, false);
          pack_bits(ctx, static_cast<uint8_t*>(c->values), n, static_cast<uint8_t*>(bc->values));
          bc->validity = c->validity;
          bc->owners.insert(bc->owners.end(), c->owners.begin(), c->owners.end());
          c = bc;
        }
        break;
      }
      case EK_STR_SELECT: {
        StrBranches sb{};
        int nb = (int)ce.branch_cols.size();
        if (nb > 17) fail(PRISM_ERR_INVALID_ARGUMENT, "at most 16 IfThen clauses for Utf8 branches");
        sb.n = nb;
        sb.has_else = ce.sel_has_else;
        std::vector<MemP> lits;
        for (int k = 0; k < nb; ++k) {
          if (ce.branch_cols[k] >= 0) {
            const Column& bc = *b.cols[ce.branch_cols[k]];
            sb.b[k].offs = bc.offsets;
            sb.b[k].data = bc.data - bc.data_base;
            sb.b[k].valid = bc.validity;
          } else {
            const std::string& s = ce.branch_lits[k];
            MemP ml = ctx.alloc(s.size() + 1);
            PRISM_CUDA(cudaMemcpyAsync(ml->ptr, s.data(), s.size(), cudaMemcpyHostToDevice, ctx.stream));
            sb.b[k].data = static_cast<uint8_t*>(ml->ptr);
            sb.b[k].lit_len = (int32_t)s.size();
            lits.push_back(ml);
          }
        }
        MemP mch, mlen, moff, mv;
        int32_t* choice = ctx.alloc_t<int32_t>((size_t)std::max<int64_t>(n, 1), mch);
        uint32_t* len = ctx.alloc_t<uint32_t>((size_t)std::max<int64_t>(n, 1), mlen);
        uint64_t* off = ctx.alloc_t<uint64_t>((size_t)std::max<int64_t>(n, 1), moff);
        uint32_t* vw = ctx.alloc_t<uint32_t>((size_t)(n + 31) / 32 + 2, mv);
        uint64_t total = 0;
        if (n) {
          str_select_kernel<<<g, 256, 0, ctx.stream>>>(p.d_pnodes, p.d_clauses, ce.sel_clause_begin, ce.sel_n_clauses,
                                                        p.d_cols, n, choice);
          ctx.check_launch("str_select_kernel");
          str_select_len_kernel<<<g, 256, 0, ctx.stream>>>(sb, choice, n, len, vw);
          ctx.check_launch("str_select_len_kernel");
          total = scan_u32(ctx, len, off, n);
        }
        if (total > (uint64_t)INT32_MAX) fail(PRISM_ERR_ARROW, "Utf8 output exceeds 2 GiB");
        c = make_utf8_column(ctx, name, n, (int64_t)total, false);
        c->validity = reinterpret_cast<uint8_t*>(vw);
        c->owners.push_back(mv);
        if (n) {
          str_select_copy_kernel<<<g, 256, 0, ctx.stream>>>(sb, choice, n, off, c->offsets, c->data);
          ctx.check_launch("str_select_copy_kernel");
        }
        PRISM_CUDA(cudaMemcpyAsync(c->offsets + n, &total, 4, cudaMemcpyHostToDevice, ctx.stream));
        ctx.sync();
        break;
      }
    }
    c->name = name;
    c->nullable = true;
    out.cols.push_back(c);
  }
  uint32_t derr = ctx.take_device_errors();
  if (derr & DERR_RANGE) fail(PRISM_ERR_EXECUTION, "decimal overflow in exact arithmetic");
  return out;
}

}  // namespace prism
