// api.cpp — the extern "C" entry points of include/prism_gpu.h.
//
// Every entry point catches failures and returns a status code (the library
// never aborts); the message is kept on the context for prism_last_error().
#include <algorithm>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <functional>

#include "agg.hpp"
#include "arrow_io.hpp"
#include "exchange.hpp"
#include "parquet.hpp"
#include "filter_project.hpp"
#include "jit.hpp"
#include "join.hpp"
#include "prims.hpp"
#include "sort.hpp"
#include "tuning.hpp"

using namespace prism;

namespace {

thread_local std::string t_err;  // errors before a context exists

int run(prism_ctx* ctx, const std::function<void()>& fn) {
  if (!ctx) return PRISM_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::recursive_mutex> lk(ctx->impl.mu);
  try {
    fn();
    return PRISM_OK;
  } catch (const Failure& f) {
    ctx->impl.last_error = f.msg;
    cudaGetLastError();
    return f.code;
  } catch (const std::bad_alloc&) {
    ctx->impl.last_error = "host allocation failed";
    return PRISM_ERR_NO_MEMORY;
  } catch (const std::exception& e) {
    ctx->impl.last_error = e.what();
    return PRISM_ERR_INTERNAL;
  }
}

prism_batch* wrap(prism_ctx* ctx, Batch b) {
  auto* out = new prism_batch();
  out->impl = std::move(b);
  out->ctx = ctx;
  return out;
}

const Batch& B(const prism_batch* b) {
  if (!b) fail(PRISM_ERR_INVALID_ARGUMENT, "null batch");
  return b->impl;
}

std::vector<int> ints(const int32_t* p, int n) {
  if (n > 0 && !p) fail(PRISM_ERR_INVALID_ARGUMENT, "null column list");
  return std::vector<int>(p, p + std::max(0, n));
}

// PRISM_JOIN_DENSE=0 keeps single Int64 keys in the hash table (dense mode off)
// PRISM_JOIN_PARTITION=0|1 turns the radix-partitioned build / probe off or
// on (default: on once the hash slots outgrow L2)
JoinTuning join_tuning() {
  JoinTuning t{};
  const char* d = std::getenv("PRISM_JOIN_DENSE");
  if (d && (std::strcmp(d, "0") == 0 || std::strcmp(d, "1") == 0)) {
    t.dense = d[0] == '1';
    t.fixed |= JoinTuning::FIX_DENSE;
  }
  // PRISM_JOIN_DENSE_PAIRS=0|1: dense tables without / with {row, value} pairs
  const char* dp = std::getenv("PRISM_JOIN_DENSE_PAIRS");
  if (dp && (std::strcmp(dp, "0") == 0 || std::strcmp(dp, "1") == 0)) t.dense_pairs = dp[0] == '1';
  // PRISM_JOIN_KEY_RECORDS=0: Utf8 keys compared through the build column, not packed records
  const char* kr = std::getenv("PRISM_JOIN_KEY_RECORDS");
  if (kr && std::strcmp(kr, "0") == 0) t.key_records = false;
  // PRISM_JOIN_KEY_ENTRIES=1: the fused join -> aggregate over a Utf8 key
  // looks up 64-byte slot entries instead of hash slots and row records
  const char* ke = std::getenv("PRISM_JOIN_KEY_ENTRIES");
  if (ke && (std::strcmp(ke, "0") == 0 || std::strcmp(ke, "1") == 0)) t.key_entries = ke[0] == '1';
  const char* p = std::getenv("PRISM_JOIN_PARTITION");
  if (p && (std::strcmp(p, "0") == 0 || std::strcmp(p, "1") == 0)) {
    t.partition = p[0] - '0';
    t.fixed |= JoinTuning::FIX_PARTITION;
  }
  return t;
}
// the environment's settings, then the tuning table's record for the build
// side's shape class
JoinTuning join_tuning_for(const Batch& build, const std::vector<int>& keys) {
  JoinTuning t = join_tuning();
  apply_join_tuning(join_shape(build, keys), t);
  return t;
}
JoinTuning join_tuning_for(const JoinTable& t) { return join_tuning_for(t.build, t.key_cols); }
// PRISM_JOIN_AGG_SHAPE=block,min_blocks,rows,table_log2 sets the fused join
// -> aggregate kernel's shape (block 128-1024 in powers of two, min_blocks
// 1-8, rows 1, 2, 4 or 8, block table of at most 2^table_log2 slots, 8-12)
AggTuning agg_tuning() {
  AggTuning t{};
  const char* d = std::getenv("PRISM_JOIN_AGG_SHAPE");
  int b = 0, m = 0, r = 0, l = 0;
  if (d && std::sscanf(d, "%d,%d,%d,%d", &b, &m, &r, &l) == 4 && (b == 128 || b == 256 || b == 512 || b == 1024) &&
      m >= 1 && m <= 8 && (r == 1 || r == 2 || r == 4 || r == 8) && l >= 8 && l <= 12) {
    t.join_block = b;
    t.join_min_blocks = m;
    t.join_rows = r;
    t.join_table_log2 = l;
    t.fixed |= AggTuning::FIX_JOIN_SHAPE;
  }
  // PRISM_HASH_AGG_BLOCK=256|512|1024: threads per block of the hashed-groups kernel
  const char* hb = std::getenv("PRISM_HASH_AGG_BLOCK");
  if (hb && (std::atoi(hb) == 256 || std::atoi(hb) == 512 || std::atoi(hb) == 1024)) {
    t.hash_block = std::atoi(hb);
    t.fixed |= AggTuning::FIX_HASH_BLOCK;
  }
  return t;
}
// the environment's settings, then the tuning table's record for `rows` input rows
AggTuning agg_tuning_for(int64_t rows) {
  AggTuning t = agg_tuning();
  apply_agg_tuning(rows, t);
  return t;
}
int64_t total_rows(const std::vector<const Batch*>& bs) {
  int64_t n = 0;
  for (auto* b : bs) n += b->rows;
  return n;
}

// PRISM_JOIN_AGG_FUSED=0 materializes the joined rows before aggregating
bool join_agg_fused() {
  const char* d = std::getenv("PRISM_JOIN_AGG_FUSED");
  return !(d && std::strcmp(d, "0") == 0);
}

std::string right_name(const Batch& probe, const std::string& nm) {
  for (auto& c : probe.cols)
    if (c->name == nm) return nm + "_right";
  return nm;
}

__global__ void fill_u32_kernel(uint32_t* p, int64_t n, uint32_t v) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) p[i] = v;
}
// bits [0, n_valid) set, [n_valid, n) clear, whole words
__global__ void prefix_bits_kernel(uint32_t* w, int64_t n, int64_t n_valid) {
  int64_t nw = (n + 31) / 32;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nw; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t lo = i * 32;
    uint32_t v;
    if (lo + 32 <= n_valid) v = 0xffffffffu;
    else if (lo >= n_valid) v = 0u;
    else v = (1u << (n_valid - lo)) - 1u;
    w[i] = v;
  }
}
// bits [0, n_null) clear, [n_null, n) set
__global__ void suffix_bits_kernel(uint32_t* w, int64_t n, int64_t n_null) {
  int64_t nw = (n + 31) / 32;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nw; i += (int64_t)gridDim.x * blockDim.x) {
    int64_t lo = i * 32;
    uint32_t v;
    if (lo + 32 <= n_null) v = 0u;
    else if (lo >= n_null) v = 0xffffffffu;
    else v = ~((1u << (n_null - lo)) - 1u);
    w[i] = v;
  }
}

struct IndexVec {
  MemP mem;
  uint32_t* ptr = nullptr;
  MemP vmem;
  uint8_t* valid = nullptr;  // null: all valid
  int64_t n = 0;
};

// concatenates index pieces: (ptr, n) or a constant fill (ptr null)
IndexVec concat_idx(Ctx& ctx, const std::vector<std::pair<const uint32_t*, int64_t>>& parts, uint32_t fill) {
  IndexVec v;
  for (auto& p : parts) v.n += p.second;
  v.ptr = ctx.alloc_t<uint32_t>((size_t)std::max<int64_t>(v.n, 1), v.mem);
  int64_t off = 0;
  for (auto& p : parts) {
    if (p.second == 0) continue;
    if (p.first) PRISM_CUDA(cudaMemcpyAsync(v.ptr + off, p.first, p.second * 4, cudaMemcpyDeviceToDevice, ctx.stream));
    else {
      fill_u32_kernel<<<grid_for(ctx, p.second, 256), 256, 0, ctx.stream>>>(v.ptr + off, p.second, fill);
      ctx.check_launch("fill_u32_kernel");
    }
    off += p.second;
  }
  return v;
}

Batch assemble(Ctx& ctx, const Batch& probe, const IndexVec& pi, const Batch& build, const IndexVec& bi, int mode) {
  Batch out;
  out.rows = pi.n;
  for (auto& c : probe.cols)
    out.cols.push_back(take(ctx, *c, pi.ptr, pi.valid, pi.n, c->name, mode == 0 ? c->nullable : true));
  for (auto& c : build.cols) {
    std::string nm = right_name(probe, c->name);
    bool nullable = c->nullable;
    if (mode == 2 && nm != c->name) nullable = true;
    out.cols.push_back(take(ctx, *c, bi.ptr, bi.valid, bi.n, nm, nullable));
  }
  return out;
}

IndexVec as_vec(const MemP& m, int64_t n) {
  IndexVec v;
  v.mem = m;
  v.ptr = m ? static_cast<uint32_t*>(m->ptr) : nullptr;
  v.n = n;
  return v;
}

MemP matched_bits(Ctx& ctx, const uint32_t* idx, int64_t n_idx, int64_t n_rows) {
  MemP m = ctx.alloc((size_t)(n_rows + 31) / 32 * 4 + 8);
  PRISM_CUDA(cudaMemsetAsync(m->ptr, 0, (size_t)(n_rows + 31) / 32 * 4 + 8, ctx.stream));
  scatter_bits(ctx, idx, n_idx, static_cast<uint8_t*>(m->ptr));
  return m;
}

// hash_join / per-batch assembly of hash_join_probe_chunked
// (native/prism-executor/src/hash_join.rs:206-282, 312-365)
Batch join_one(Ctx& ctx, const Batch& probe, const Batch& build, const JoinTable& t, const std::vector<int>& pk,
               int join_type, bool chunked) {
  std::vector<ProbeGather> none;
  ProbeResult pr = probe_join_table(ctx, t, probe, pk, true, true, none, -1, join_tuning_for(t));
  int64_t n = pr.matches;
  IndexVec pi = as_vec(pr.probe_idx, n), bi = as_vec(pr.build_idx, n);
  switch (join_type) {
    case PRISM_JOIN_INNER:
      return assemble(ctx, probe, pi, build, bi, 0);
    case PRISM_JOIN_LEFT: {
      // left_join_indices (hash_join.rs:455-483): unmatched probe rows pair
      // with build index 0, i.e. they carry build row 0's values
      MemP mb = matched_bits(ctx, pi.ptr, n, probe.rows);
      int64_t nu = 0;
      MemP un = compact_bits(ctx, static_cast<uint8_t*>(mb->ptr), probe.rows, true, &nu);
      if (nu > 0 && build.rows == 0)
        fail(PRISM_ERR_JOIN, "left join of unmatched probe rows against an empty build side "
                             "(the reference indexes build row 0)");
      IndexVec p2 = concat_idx(ctx, {{pi.ptr, n}, {static_cast<uint32_t*>(un->ptr), nu}}, 0);
      IndexVec b2 = concat_idx(ctx, {{bi.ptr, n}, {nullptr, nu}}, 0);
      return assemble(ctx, probe, p2, build, b2, 0);
    }
    case PRISM_JOIN_LEFT_SEMI: case PRISM_JOIN_LEFT_ANTI: {
      MemP mb = matched_bits(ctx, pi.ptr, n, probe.rows);
      int64_t nk = 0;
      MemP rows = compact_bits(ctx, static_cast<uint8_t*>(mb->ptr), probe.rows, join_type == PRISM_JOIN_LEFT_ANTI, &nk);
      Batch out = filter_rows(ctx, probe, static_cast<uint32_t*>(rows->ptr), nk);
      return out;
    }
    case PRISM_JOIN_RIGHT: case PRISM_JOIN_FULL: {
      if (chunked) return assemble(ctx, probe, pi, build, bi, 0);  // hash_join.rs:261-270
      MemP bm = matched_bits(ctx, bi.ptr, n, build.rows);
      int64_t nub = 0;
      MemP unb = compact_bits(ctx, static_cast<uint8_t*>(bm->ptr), build.rows, true, &nub);
      int64_t nup = 0;
      MemP unp;
      if (join_type == PRISM_JOIN_FULL) {
        MemP pm = matched_bits(ctx, pi.ptr, n, probe.rows);
        unp = compact_bits(ctx, static_cast<uint8_t*>(pm->ptr), probe.rows, true, &nup);
        // non-nullable, non-renamed build fields would receive nulls: arrow-rs
        // RecordBatch::try_new rejects that batch in the reference
        if (nup > 0)
          for (auto& c : build.cols)
            if (!c->nullable && right_name(probe, c->name) == c->name)
              fail(PRISM_ERR_ARROW, "Invalid argument error: Column '" + c->name +
                                        "' is declared as non-nullable but contains null values");
      }
      // probe indices: matched, unmatched probe (FULL), null for unmatched build
      IndexVec p2 = concat_idx(ctx, {{pi.ptr, n}, {unp ? static_cast<uint32_t*>(unp->ptr) : nullptr, nup}, {nullptr, nub}}, 0);
      p2.vmem = ctx.alloc((size_t)(p2.n + 31) / 32 * 4 + 8);
      p2.valid = static_cast<uint8_t*>(p2.vmem->ptr);
      prefix_bits_kernel<<<grid_for(ctx, (p2.n + 31) / 32 + 1, 256), 256, 0, ctx.stream>>>(
          reinterpret_cast<uint32_t*>(p2.valid), p2.n, n + nup);
      ctx.check_launch("prefix_bits_kernel");
      IndexVec b2 = concat_idx(ctx, {{bi.ptr, n}, {nullptr, nup}, {static_cast<uint32_t*>(unb->ptr), nub}}, 0);
      if (join_type == PRISM_JOIN_FULL && nup > 0) {
        // build indices null for the unmatched probe rows [n, n + nup)
        b2.vmem = ctx.alloc((size_t)(b2.n + 31) / 32 * 4 + 8);
        b2.valid = static_cast<uint8_t*>(b2.vmem->ptr);
        // set all, then clear [n, n+nup): compose prefix [0,n) with suffix [n+nup, end)
        MemP tmp1 = ctx.alloc((size_t)(b2.n + 31) / 32 * 4 + 8), tmp2 = ctx.alloc((size_t)(b2.n + 31) / 32 * 4 + 8);
        int g = grid_for(ctx, (b2.n + 31) / 32 + 1, 256);
        prefix_bits_kernel<<<g, 256, 0, ctx.stream>>>(static_cast<uint32_t*>(tmp1->ptr), b2.n, n);
        suffix_bits_kernel<<<g, 256, 0, ctx.stream>>>(static_cast<uint32_t*>(tmp2->ptr), b2.n, n + nup);
        ctx.check_launch("bits_kernel");
        // or the two masks
        std::vector<uint32_t> h1((size_t)(b2.n + 31) / 32), h2(h1.size());
        PRISM_CUDA(cudaMemcpyAsync(h1.data(), tmp1->ptr, h1.size() * 4, cudaMemcpyDeviceToHost, ctx.stream));
        PRISM_CUDA(cudaMemcpyAsync(h2.data(), tmp2->ptr, h2.size() * 4, cudaMemcpyDeviceToHost, ctx.stream));
        PRISM_CUDA(cudaStreamSynchronize(ctx.stream));
        for (size_t i = 0; i < h1.size(); ++i) h1[i] |= h2[i];
        PRISM_CUDA(cudaMemcpyAsync(b2.valid, h1.data(), h1.size() * 4, cudaMemcpyHostToDevice, ctx.stream));
        PRISM_CUDA(cudaStreamSynchronize(ctx.stream));
      }
      return assemble(ctx, probe, p2, build, b2, join_type == PRISM_JOIN_FULL ? 2 : 1);
    }
  }
  fail(PRISM_ERR_INVALID_ARGUMENT, "unknown join type");
}

std::string joined_name(const Batch& probe, const Batch& build, int col) {
  int np = (int)probe.cols.size();
  if (col < np) return probe.cols[col]->name;
  return right_name(probe, build.cols[col - np]->name);
}

// join_project: probe `probe` against `t` and gather `oc` of the joined
// schema (probe columns, then build columns; PRISM_COL_* for row indices).
Batch join_project_impl(Ctx& x, const JoinTable& t, const Batch& probe, const std::vector<int>& pk,
                        const std::vector<int>& oc, uint32_t flags) {
  if (flags & ~(uint32_t)PRISM_JOIN_ANY_ORDER) fail(PRISM_ERR_INVALID_ARGUMENT, "unknown join_project flags");
  const Batch& build = t.build;
  int np = (int)probe.cols.size(), nb = (int)build.cols.size();
  for (int col : oc)
    if (col < PRISM_COL_BUILD_ROW_INDEX || col >= np + nb) fail(PRISM_ERR_INVALID_ARGUMENT, "joined column out of range");
  // gather fixed-width null-free columns inside the probe kernel
  bool fusable = (int)oc.size() <= 6;
  int n_gather = 0;
  for (int col : oc) {
    if (col < 0) continue;
    const Column& src = col < np ? *probe.cols[col] : *build.cols[col - np];
    int w = width_of(src.type);
    if (src.validity || (w != 4 && w != 8) || src.type == TY_DICT) fusable = false;
    ++n_gather;
  }
  if (n_gather > 4) fusable = false;
  int64_t cap = match_upper_bound(t, probe.rows);
  if (cap < 0) cap = probe_count(x, t, probe, pk, join_tuning_for(t));
  bool want_p = !fusable, want_b = !fusable;
  for (int col : oc) {
    if (col == PRISM_COL_PROBE_ROW_INDEX) want_p = true;
    if (col == PRISM_COL_BUILD_ROW_INDEX) want_b = true;
  }
  std::vector<ProbeGather> gathers;
  std::vector<ColP> gcols;
  if (fusable) {
    for (int col : oc) {
      if (col < 0) continue;
      const Column& src = col < np ? *probe.cols[col] : *build.cols[col - np];
      ColP dst = make_column(x, src.type, joined_name(probe, build, col), cap, false);
      dst->nullable = src.nullable;
      dst->precision = src.precision;
      dst->scale = src.scale;
      gathers.push_back({col < np ? 0 : 1, src.values, width_of(src.type), dst->values});
      gcols.push_back(dst);
    }
  }
  ProbeResult r = probe_join_table(x, t, probe, pk, want_p, want_b, gathers, cap, join_tuning_for(t),
                                   (flags & PRISM_JOIN_ANY_ORDER) != 0);
  Batch res;
  res.rows = r.matches;
  size_t gi = 0;
  for (int col : oc) {
    if (col == PRISM_COL_PROBE_ROW_INDEX) {
      res.cols.push_back(u32_column(x, "probe_idx", r.probe_idx, static_cast<uint32_t*>(r.probe_idx->ptr), r.matches));
    } else if (col == PRISM_COL_BUILD_ROW_INDEX) {
      res.cols.push_back(u32_column(x, "build_idx", r.build_idx, static_cast<uint32_t*>(r.build_idx->ptr), r.matches));
    } else if (fusable) {
      ColP g = gcols[gi++];
      g->length = r.matches;
      res.cols.push_back(g);
    } else {
      const Column& src = col < np ? *probe.cols[col] : *build.cols[col - np];
      const uint32_t* idx = static_cast<const uint32_t*>(col < np ? r.probe_idx->ptr : r.build_idx->ptr);
      res.cols.push_back(take(x, src, idx, nullptr, r.matches, joined_name(probe, build, col), src.nullable));
    }
  }
  return res;
}

// try_execute_fused_join_aggregate (executor.rs:333-458): the fused kernel
// (lookup, projection and aggregation of the joined rows in one kernel per
// probe batch) under `tune`, or the materialising path for shapes it does not
// take.
Batch join_aggregate_impl(Ctx& x, const std::vector<const Batch*>& probes, const Batch& bb, const std::vector<int>& pk,
                          const std::vector<int>& bk, const int32_t* cols, int32_t n_cols, const prism_expr* exprs,
                          int32_t n_exprs, const prism_agg_config* agg, const AggTuning& tune) {
  for (const Batch* p : probes) check_join_keys(*p, pk, bb, bk);
  JoinTuning jt = join_tuning_for(bb, bk);
  // a single Utf8 key looked up through slot entries by the fused kernel:
  // they replace the row records
  const bool entries = join_agg_fused() && jt.key_entries && bk.size() == 1 && bb.cols[bk[0]]->type == TY_UTF8;
  if (entries) jt.key_records = false;
  auto t = build_join_table(x, bb, bk, jt);
  // joined columns referenced by the projection (executor.rs:474-551)
  const Batch& p0 = *probes[0];
  int np = (int)p0.cols.size(), total = np + (int)bb.cols.size();
  std::vector<bool> need(total, false);
  for (int i = 0; i < n_cols; ++i) {
    if (cols[i] < 0 || cols[i] >= total) fail(PRISM_ERR_INVALID_ARGUMENT, "joined column out of range");
    need[cols[i]] = true;
  }
  for (int e = 0; e < n_exprs; ++e) {
    for (int k = 0; k < exprs[e].n_nodes; ++k)
      if (exprs[e].nodes[k].op == PRISM_EXPR_COLUMN) {
        int col = exprs[e].nodes[k].column;
        if (col < 0 || col >= total) fail(PRISM_ERR_INVALID_ARGUMENT, "joined column out of range");
        need[col] = true;
      }
    for (int k = 0; k < exprs[e].n_preds; ++k) {
      int op = exprs[e].preds[k].op;
      if (op != PRISM_PRED_LITERAL && op != PRISM_PRED_AND && op != PRISM_PRED_OR && op != PRISM_PRED_NOT) {
        int col = exprs[e].preds[k].column;
        if (col < 0 || col >= total) fail(PRISM_ERR_INVALID_ARGUMENT, "joined column out of range");
        need[col] = true;
      }
    }
  }
  // the first referenced build column of fixed width 4 or 8 without nulls
  // rides with the lookup (in the slot entries, or per probe row from the
  // split lookup) and is read from there for single-row slots
  int inl = -1;
  for (int c = 0; c < (int)bb.cols.size() && inl < 0; ++c) {
    const Column& col = *bb.cols[c];
    const int w = width_of(col.type == TY_DICT ? col.index_type : col.type);
    if (need[np + c] && !col.validity && col.type != TY_BOOL && (w == 4 || w == 8)) inl = c;
  }
  if (entries) build_key_entries(x, *t, inl);
  if (join_agg_fused()) {
    // one kernel per probe batch: lookup, projection and aggregation of
    // the joined rows without materializing them
    JoinAggSpec js;
    js.table = t.get();
    js.probe_keys = pk;
    js.inline_col = inl;
    try {
      return aggregate(x, probes, *agg, nullptr, cols, n_cols, exprs, n_exprs, PRISM_ARITH_F64, true, tune, &js);
    } catch (const Failure& f) {
      if (f.code != PRISM_ERR_INVALID_ARGUMENT || f.msg.find("fused path") == std::string::npos) throw;
    }
  }
  std::vector<Batch> projected;
  for (const Batch* pbp : probes) {
    const Batch& pb = *pbp;
    std::vector<ProbeGather> none;
    ProbeResult r = probe_join_table(x, *t, pb, pk, true, true, none, -1, join_tuning_for(*t));
    if (r.matches == 0 && !projected.empty()) continue;
    Batch joined;
    joined.rows = r.matches;
    for (int col = 0; col < total; ++col) {
      if (!need[col]) {
        auto z = std::make_shared<Column>();
        z->type = TY_NULL;
        z->length = r.matches;
        joined.cols.push_back(z);
        continue;
      }
      const Column& src = col < np ? *pb.cols[col] : *bb.cols[col - np];
      const uint32_t* idx = static_cast<const uint32_t*>(col < np ? r.probe_idx->ptr : r.build_idx->ptr);
      joined.cols.push_back(take(x, src, idx, nullptr, r.matches, joined_name(pb, bb, col), src.nullable));
    }
    projected.push_back(project_with_exprs(x, joined, cols, n_cols, exprs, n_exprs, PRISM_ARITH_F64));
  }
  std::vector<const Batch*> ps;
  for (auto& p : projected)
    if (p.rows > 0 || projected.size() == 1) ps.push_back(&p);
  return aggregate(x, ps, *agg, nullptr, nullptr, 0, nullptr, 0, PRISM_ARITH_F64, false, agg_tuning_for(total_rows(ps)));
}

}  // namespace

extern "C" {

const char* prism_version(void) { return "prism-gpu 0.1 (sm_100a)"; }

int prism_ctx_create(int device, uint64_t budget, prism_ctx** out) {
  if (!out) return PRISM_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  auto* c = new prism_ctx();
  Ctx& x = c->impl;
  try {
    PRISM_CUDA(cudaSetDevice(device));
    x.device = device;
    PRISM_CUDA(cudaStreamCreateWithFlags(&x.own_stream, cudaStreamNonBlocking));
    x.stream = x.own_stream;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    PRISM_CUDA(cudaMemPoolCreate(&x.pool, &props));
    uint64_t thr = UINT64_MAX;
    PRISM_CUDA(cudaMemPoolSetAttribute(x.pool, cudaMemPoolAttrReleaseThreshold, &thr));
    size_t free_b = 0, total_b = 0;
    PRISM_CUDA(cudaMemGetInfo(&free_b, &total_b));
    x.budget = budget ? budget : (uint64_t)(free_b * 0.9);
    PRISM_CUDA(cudaDeviceGetAttribute(&x.sm_count, cudaDevAttrMultiProcessorCount, device));
    int l2 = 0;
    PRISM_CUDA(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, device));
    if (l2 > 0) x.l2_bytes = l2;
    PRISM_CUDA(cudaMalloc(&x.d_err, 64));
    PRISM_CUDA(cudaMemset(x.d_err, 0, 64));
    PRISM_CUDA(cudaMallocHost(&x.h_err, 128));
    // the staging ring is optional: without it staged copies wait for the stream
    constexpr size_t STAGE = (size_t)1 << 20;
    if (cudaMallocHost(&x.h_stage, STAGE) == cudaSuccess &&
        cudaEventCreateWithFlags(&x.stage_ev, cudaEventDisableTiming) == cudaSuccess) {
      x.stage_cap = STAGE;
    } else {
      cudaGetLastError();
      if (x.h_stage) cudaFreeHost(x.h_stage);
      x.h_stage = nullptr;
      x.stage_ev = nullptr;
    }
  } catch (const Failure& f) {
    t_err = f.msg;
    if (x.pool) cudaMemPoolDestroy(x.pool);
    if (x.own_stream) cudaStreamDestroy(x.own_stream);
    delete c;
    cudaGetLastError();
    return f.code;
  }
  *out = c;
  return PRISM_OK;
}

void prism_ctx_destroy(prism_ctx* c) {
  if (!c) return;
  Ctx& x = c->impl;
  cudaStreamSynchronize(x.stream);
  x.clear_timings();
  for (auto e : x.event_pool) cudaEventDestroy(e);
  for (auto& [fn, g] : x.probe_graphs) {
    if (g.exec) cudaGraphExecDestroy(g.exec);
    if (g.graph) cudaGraphDestroy(g.graph);
  }
  x.probe_graphs.clear();
  if (x.d_err) cudaFree(x.d_err);
  if (x.h_err) cudaFreeHost(x.h_err);
  if (x.h_stage) cudaFreeHost(x.h_stage);
  if (x.stage_ev) cudaEventDestroy(x.stage_ev);
  if (x.pool) cudaMemPoolDestroy(x.pool);
  if (x.own_stream) cudaStreamDestroy(x.own_stream);
  delete c;
}

const char* prism_last_error(const prism_ctx* c) { return c ? c->impl.last_error.c_str() : t_err.c_str(); }

int prism_ctx_set_stream(prism_ctx* c, void* s) {
  return run(c, [&] {
    PRISM_CUDA(cudaStreamSynchronize(c->impl.stream));
    c->impl.stream = s ? static_cast<cudaStream_t>(s) : c->impl.own_stream;
  });
}

int prism_ctx_synchronize(prism_ctx* c) { return run(c, [&] { c->impl.sync(); }); }
uint64_t prism_ctx_bytes_in_use(const prism_ctx* c) { return c ? c->impl.in_use.load() : 0; }

int prism_ctx_set_profiling(prism_ctx* c, int enable) {
  return run(c, [&] {
    c->impl.sync();
    c->impl.clear_timings();
    c->impl.profiling = enable != 0;
  });
}

int prism_ctx_kernel_stats(prism_ctx* c, const char* name, uint64_t* launches, double* total_ms) {
  return run(c, [&] {
    if (!name || !launches || !total_ms) fail(PRISM_ERR_INVALID_ARGUMENT, "null arguments");
    c->impl.sync();
    *launches = 0;
    *total_ms = 0;
    auto it = c->impl.timings.find(name);
    if (it == c->impl.timings.end()) return;
    for (auto& pr : it->second) {
      float ms = 0;
      PRISM_CUDA(cudaEventElapsedTime(&ms, pr.first, pr.second));
      *total_ms += ms;
      *launches += 1;
    }
  });
}

int prism_jit_stats(int32_t* enabled, int64_t* compiles, double* total_ms) {
  if (enabled) *enabled = prism::jit_enabled() ? 1 : 0;
  prism::jit_stats(compiles, total_ms);
  return PRISM_OK;
}
uint64_t prism_ctx_kernel_launches(const prism_ctx* c) { return c ? c->impl.launches.load() : 0; }

// ------------------------------------------------------------- batches ---
int prism_batch_import(prism_ctx* c, const ArrowArray* a, const ArrowSchema* s, prism_batch** out) {
  return run(c, [&] {
    if (!out) fail(PRISM_ERR_INVALID_ARGUMENT, "null output");
    *out = wrap(c, import_batch(c->impl, a, s, false));
  });
}

int prism_batch_import_device(prism_ctx* c, const ArrowDeviceArray* a, const ArrowSchema* s, prism_batch** out) {
  return run(c, [&] {
    if (!out) fail(PRISM_ERR_INVALID_ARGUMENT, "null output");
    *out = wrap(c, import_device_batch(c->impl, a, s));
  });
}

int prism_batch_export(prism_ctx* c, const prism_batch* b, ArrowArray* a, ArrowSchema* s) {
  return run(c, [&] { export_batch(c->impl, B(b), a, s); });
}

int64_t prism_batch_num_rows(const prism_batch* b) { return b ? b->impl.rows : -1; }
int32_t prism_batch_num_columns(const prism_batch* b) { return b ? (int32_t)b->impl.cols.size() : -1; }
int prism_batch_column_device(const prism_batch* b, int32_t col, const void** values, const uint8_t** validity,
                              int32_t* width) {
  if (!b || col < 0 || col >= (int32_t)b->impl.cols.size()) return PRISM_ERR_INVALID_ARGUMENT;
  const Column& c = *b->impl.cols[col];
  if (values) *values = c.type == TY_UTF8 ? static_cast<const void*>(c.offsets) : c.values;
  if (validity) *validity = c.validity;
  if (width) *width = width_of(c.type == TY_DICT ? c.index_type : c.type);
  return PRISM_OK;
}
void prism_batch_free(prism_batch* b) {
  if (!b) return;
  if (b->ctx) {
    std::lock_guard<std::recursive_mutex> lk(b->ctx->impl.mu);
    delete b;
  } else {
    delete b;
  }
}

// ---------------------------------------------------------------- join ---
int prism_hash_table_build(prism_ctx* c, const prism_batch* build, const int32_t* keys, int32_t n, prism_hash_table** out) {
  return run(c, [&] {
    if (!out) fail(PRISM_ERR_INVALID_ARGUMENT, "null output");
    auto* h = new prism_hash_table();
    h->ctx = c;
    try {
      const std::vector<int> kv = ints(keys, n);
      h->t = build_join_table(c->impl, B(build), kv, join_tuning_for(B(build), kv));
    } catch (...) {
      delete h;
      throw;
    }
    *out = h;
  });
}

int prism_hash_table_probe(prism_ctx* c, const prism_hash_table* t, const prism_batch* probe, const int32_t* keys,
                           int32_t n, prism_batch** out) {
  return run(c, [&] {
    if (!t || !out) fail(PRISM_ERR_INVALID_ARGUMENT, "null table/output");
    std::vector<ProbeGather> none;
    ProbeResult r = probe_join_table(c->impl, *t->t, B(probe), ints(keys, n), true, true, none, -1, join_tuning_for(*t->t));
    Batch b;
    b.rows = r.matches;
    b.cols.push_back(u32_column(c->impl, "probe_idx", r.probe_idx, static_cast<uint32_t*>(r.probe_idx->ptr), r.matches));
    b.cols.push_back(u32_column(c->impl, "build_idx", r.build_idx, static_cast<uint32_t*>(r.build_idx->ptr), r.matches));
    *out = wrap(c, std::move(b));
  });
}

int64_t prism_hash_table_num_rows(const prism_hash_table* t) { return t ? t->t->build.rows : -1; }
int prism_hash_table_has_duplicates(const prism_hash_table* t) { return t && t->t->has_dups ? 1 : 0; }
int prism_hash_table_layout(const prism_hash_table* t) {
  if (!t || !t->t) return -1;
  return t->t->dense ? PRISM_TABLE_DENSE : PRISM_TABLE_HASH;
}
void prism_hash_table_free(prism_hash_table* t) {
  if (!t) return;
  if (t->ctx) {
    std::lock_guard<std::recursive_mutex> lk(t->ctx->impl.mu);
    delete t;
  } else {
    delete t;
  }
}

int prism_join_project(prism_ctx* c, const prism_hash_table* tab, const prism_batch* probe_b, const int32_t* probe_keys,
                       int32_t n_keys, const int32_t* out_cols, int32_t n_out, prism_batch** out) {
  return prism_join_project_ex(c, tab, probe_b, probe_keys, n_keys, out_cols, n_out, 0u, out);
}

int prism_join_project_ex(prism_ctx* c, const prism_hash_table* tab, const prism_batch* probe_b,
                          const int32_t* probe_keys, int32_t n_keys, const int32_t* out_cols, int32_t n_out,
                          uint32_t flags, prism_batch** out) {
  return run(c, [&] {
    if (!tab || !tab->t || !out) fail(PRISM_ERR_INVALID_ARGUMENT, "null table/output");
    Batch res = join_project_impl(c->impl, *tab->t, B(probe_b), ints(probe_keys, n_keys), ints(out_cols, n_out), flags);
    c->impl.sync();
    *out = wrap(c, std::move(res));
  });
}

int prism_join_project_arrow(prism_ctx* c, const prism_hash_table* tab, const ArrowArray* probe_a,
                             const ArrowSchema* probe_s, const int32_t* probe_keys, int32_t n_keys,
                             const int32_t* out_cols, int32_t n_out, uint32_t flags, ArrowArray* out,
                             ArrowSchema* out_schema) {
  return run(c, [&] {
    if (!tab || !tab->t || !out || !out_schema) fail(PRISM_ERR_INVALID_ARGUMENT, "null table/output");
    Ctx& x = c->impl;
    const JoinTable& t = *tab->t;
    std::vector<int> pk = ints(probe_keys, n_keys), oc = ints(out_cols, n_out);
    std::vector<HostView> hv = host_view(probe_a, probe_s);
    const int np = (int)hv.size(), nb = (int)t.build.cols.size();
    const int64_t n = probe_a->length;
    for (int col : oc)
      if (col < PRISM_COL_BUILD_ROW_INDEX || col >= np + nb) fail(PRISM_ERR_INVALID_ARGUMENT, "joined column out of range");
    // Streamed when every match has one row (unique Int64 build keys) and the
    // probe key and every gathered column are fixed-width without nulls:
    // the probe rows go up in chunks, and chunk i+1's upload, chunk i's probe
    // and chunk i-1's download run at once (uploads and downloads use the
    // link's two directions). Anything else: one upload, probe, download.
    bool stream = t.int64_fast && !t.has_dups && pk.size() == 1 && pk[0] >= 0 && pk[0] < np &&
                  hv[pk[0]].meta->type == TY_I64 && hv[pk[0]].values && oc.size() <= 6;
    int n_gather = 0;
    for (int col : oc) {
      if (col < 0) continue;
      ++n_gather;
      if (col < np) {
        const HostView& h = hv[col];
        const int w = width_of(h.meta->type);
        if (!h.values || h.null_count != 0 || (w != 4 && w != 8) || h.meta->type == TY_DICT) stream = false;
      } else {
        const Column& src = *t.build.cols[col - np];
        const int w = width_of(src.type);
        if (src.validity || (w != 4 && w != 8) || src.type == TY_DICT) stream = false;
      }
    }
    if (n_gather > 4) stream = false;
    if (!stream || n == 0) {
      Batch probe = import_batch(x, probe_a, probe_s, false);
      Batch res = join_project_impl(x, t, probe, pk, oc, flags);
      export_batch(x, res, out, out_schema);
      return;
    }
    Batch pmeta;  // the probe schema (metadata only)
    pmeta.rows = n;
    for (auto& h : hv) pmeta.cols.push_back(h.meta);
    check_join_keys(pmeta, pk, t.build, t.key_cols);
    const bool any = (flags & PRISM_JOIN_ANY_ORDER) != 0;
    if (flags & ~(uint32_t)PRISM_JOIN_ANY_ORDER) fail(PRISM_ERR_INVALID_ARGUMENT, "unknown join_project flags");
    constexpr int64_t CH = (int64_t)1 << 23;  // probe rows per chunk (a multiple of every probe tile)
    const int64_t nchunks = (n + CH - 1) / CH;
    // probe columns to upload (the key first), with their staging slots
    std::vector<int> up{pk[0]};
    for (int col : oc)
      if (col >= 0 && col < np && std::find(up.begin(), up.end(), col) == up.end()) up.push_back(col);
    std::vector<MemP> in_mem[2];
    for (int sl = 0; sl < 2; ++sl)
      for (int col : up) in_mem[sl].push_back(x.alloc((size_t)std::min(CH, n) * width_of(hv[col].meta->type) + 16));
    // outputs: host columns sized for every probe row, device staging per slot
    std::vector<HostOutCol> hcols;
    std::vector<int> ow;
    for (int col : oc) {
      ColP m = std::make_shared<Column>();
      if (col == PRISM_COL_PROBE_ROW_INDEX || col == PRISM_COL_BUILD_ROW_INDEX) {
        m->type = TY_U32;
        m->name = col == PRISM_COL_PROBE_ROW_INDEX ? "probe_idx" : "build_idx";
        m->nullable = false;
      } else {
        const Column& src = col < np ? *hv[col].meta : *t.build.cols[col - np];
        m->type = src.type;
        m->name = joined_name(pmeta, t.build, col);
        m->nullable = src.nullable;
        m->precision = src.precision;
        m->scale = src.scale;
      }
      ow.push_back(width_of(m->type));
      hcols.push_back(host_out_column(m, (size_t)n * ow.back()));
    }
    std::vector<MemP> out_mem[2];
    for (int sl = 0; sl < 2; ++sl)
      for (size_t k = 0; k < oc.size(); ++k)
        if (oc[k] >= 0) out_mem[sl].push_back(x.alloc((size_t)std::min(CH, n) * ow[k] + 16));
    cudaStream_t s_in = nullptr, s_out = nullptr;
    cudaEvent_t ev_in[2] = {}, ev_used[2] = {}, ev_probed[2] = {}, ev_out[2] = {};
    ProbeResult held[2];
    auto cleanup = [&] {
      if (s_in) cudaStreamSynchronize(s_in);
      if (s_out) cudaStreamSynchronize(s_out);
      cudaStreamSynchronize(x.stream);
      for (auto* e : {ev_in, ev_used, ev_probed, ev_out})
        for (int sl = 0; sl < 2; ++sl)
          if (e[sl]) cudaEventDestroy(e[sl]);
      if (s_in) cudaStreamDestroy(s_in);
      if (s_out) cudaStreamDestroy(s_out);
    };
    int64_t total = 0;
    try {
      PRISM_CUDA(cudaStreamCreateWithFlags(&s_in, cudaStreamNonBlocking));
      PRISM_CUDA(cudaStreamCreateWithFlags(&s_out, cudaStreamNonBlocking));
      for (auto* e : {ev_in, ev_used, ev_probed, ev_out})
        for (int sl = 0; sl < 2; ++sl) PRISM_CUDA(cudaEventCreateWithFlags(&e[sl], cudaEventDisableTiming));
      // the staging and output buffers were allocated on the context's stream
      PRISM_CUDA(cudaEventRecord(ev_used[0], x.stream));
      PRISM_CUDA(cudaStreamWaitEvent(s_in, ev_used[0], 0));
      auto upload = [&](int64_t i) {
        const int sl = (int)(i & 1);
        const int64_t lo = i * CH, rows = std::min(CH, n - lo);
        if (i >= 2) PRISM_CUDA(cudaStreamWaitEvent(s_in, ev_used[sl], 0));  // chunk i-2's probe read the slot
        for (size_t u = 0; u < up.size(); ++u) {
          const int w = width_of(hv[up[u]].meta->type);
          PRISM_CUDA(cudaMemcpyAsync(in_mem[sl][u]->ptr, static_cast<const uint8_t*>(hv[up[u]].values) + lo * w,
                                     (size_t)rows * w, cudaMemcpyHostToDevice, s_in));
        }
        PRISM_CUDA(cudaEventRecord(ev_in[sl], s_in));
      };
      upload(0);
      for (int64_t i = 0; i < nchunks; ++i) {
        const int sl = (int)(i & 1);
        const int64_t lo = i * CH, rows = std::min(CH, n - lo);
        if (i + 1 < nchunks) upload(i + 1);
        PRISM_CUDA(cudaStreamWaitEvent(x.stream, ev_in[sl], 0));
        if (i >= 2) PRISM_CUDA(cudaStreamWaitEvent(x.stream, ev_out[sl], 0));  // chunk i-2's download left the slot
        held[sl] = ProbeResult{};  // chunk i-2's index arrays: freed after its download (ordered above)
        Batch chunk;
        chunk.rows = rows;
        for (int j = 0; j < np; ++j) {
          auto col = std::make_shared<Column>(*hv[j].meta);
          col->length = rows;
          auto it = std::find(up.begin(), up.end(), j);
          col->values = it == up.end() ? nullptr : in_mem[sl][it - up.begin()]->ptr;
          chunk.cols.push_back(col);
        }
        std::vector<ProbeGather> gathers;
        bool want_p = false, want_b = false;
        size_t g = 0;
        for (int col : oc) {
          if (col == PRISM_COL_PROBE_ROW_INDEX) want_p = true;
          else if (col == PRISM_COL_BUILD_ROW_INDEX) want_b = true;
          else {
            const Column& src = col < np ? *chunk.cols[col] : *t.build.cols[col - np];
            gathers.push_back({col < np ? 0 : 1, src.values, width_of(src.type), out_mem[sl][g++]->ptr});
          }
        }
        held[sl] = probe_join_table(x, t, chunk, pk, want_p, want_b, gathers, rows, join_tuning_for(t), any, lo);
        const int64_t m = held[sl].matches;
        PRISM_CUDA(cudaEventRecord(ev_used[sl], x.stream));
        PRISM_CUDA(cudaEventRecord(ev_probed[sl], x.stream));
        PRISM_CUDA(cudaStreamWaitEvent(s_out, ev_probed[sl], 0));
        g = 0;
        for (size_t k = 0; k < oc.size(); ++k) {
          const void* src = oc[k] == PRISM_COL_PROBE_ROW_INDEX   ? held[sl].probe_idx->ptr
                            : oc[k] == PRISM_COL_BUILD_ROW_INDEX ? held[sl].build_idx->ptr
                                                                 : out_mem[sl][g++]->ptr;
          if (m)
            PRISM_CUDA(cudaMemcpyAsync(static_cast<uint8_t*>(hcols[k].values) + (size_t)total * ow[k], src,
                                       (size_t)m * ow[k], cudaMemcpyDeviceToHost, s_out));
        }
        PRISM_CUDA(cudaEventRecord(ev_out[sl], s_out));
        total += m;
      }
      PRISM_CUDA(cudaStreamSynchronize(s_out));
    } catch (...) {
      cleanup();
      throw;
    }
    cleanup();
    export_host_columns(hcols, total, out, out_schema);
  });
}

int prism_hash_join(prism_ctx* c, const prism_batch* probe, const prism_batch* build, const prism_join_config* cfg,
                    prism_batch** out) {
  return run(c, [&] {
    if (!cfg || !out) fail(PRISM_ERR_INVALID_ARGUMENT, "null config/output");
    std::vector<int> pk = ints(cfg->probe_keys, cfg->n_keys), bk = ints(cfg->build_keys, cfg->n_keys);
    check_join_keys(B(probe), pk, B(build), bk);
    auto t = build_join_table(c->impl, B(build), bk, join_tuning_for(B(build), bk));
    Batch r = join_one(c->impl, B(probe), B(build), *t, pk, cfg->join_type, false);
    c->impl.sync();
    *out = wrap(c, std::move(r));
  });
}

int prism_probe_matches_chunked(prism_ctx* c, const prism_batch* const* probes, int32_t n_probes, const prism_batch* build,
                                const int32_t* probe_keys, const int32_t* build_keys, int32_t n_keys, prism_batch** out) {
  return run(c, [&] {
    if (!out || (n_probes > 0 && !probes)) fail(PRISM_ERR_INVALID_ARGUMENT, "null probes/output");
    std::vector<int> pk = ints(probe_keys, n_keys), bk = ints(build_keys, n_keys);
    for (int i = 0; i < n_probes; ++i) check_join_keys(B(probes[i]), pk, B(build), bk);
    auto t = build_join_table(c->impl, B(build), bk, join_tuning_for(B(build), bk));
    std::vector<prism_batch*> res;
    try {
      for (int i = 0; i < n_probes; ++i) {
        std::vector<ProbeGather> none;
        ProbeResult r = probe_join_table(c->impl, *t, B(probes[i]), pk, true, true, none, -1, join_tuning_for(*t));
        Batch b;
        b.rows = r.matches;
        b.cols.push_back(u32_column(c->impl, "probe_idx", r.probe_idx, static_cast<uint32_t*>(r.probe_idx->ptr), r.matches));
        b.cols.push_back(u32_column(c->impl, "build_idx", r.build_idx, static_cast<uint32_t*>(r.build_idx->ptr), r.matches));
        res.push_back(wrap(c, std::move(b)));
      }
    } catch (...) {
      for (auto* r : res) delete r;
      throw;
    }
    for (int i = 0; i < n_probes; ++i) out[i] = res[i];
  });
}

int prism_hash_join_probe_chunked(prism_ctx* c, const prism_batch* const* probes, int32_t n_probes,
                                  const prism_batch* build, const prism_join_config* cfg, prism_batch** out,
                                  int32_t* n_out) {
  return run(c, [&] {
    if (!cfg || !out || !n_out) fail(PRISM_ERR_INVALID_ARGUMENT, "null config/output");
    std::vector<int> pk = ints(cfg->probe_keys, cfg->n_keys), bk = ints(cfg->build_keys, cfg->n_keys);
    for (int i = 0; i < n_probes; ++i) check_join_keys(B(probes[i]), pk, B(build), bk);
    auto t = build_join_table(c->impl, B(build), bk, join_tuning_for(B(build), bk));
    std::vector<prism_batch*> res;
    try {
      for (int i = 0; i < n_probes; ++i) {
        Batch r = join_one(c->impl, B(probes[i]), B(build), *t, pk, cfg->join_type, true);
        if (r.rows > 0) res.push_back(wrap(c, std::move(r)));
      }
      c->impl.sync();
    } catch (...) {
      for (auto* r : res) delete r;
      throw;
    }
    for (size_t i = 0; i < res.size(); ++i) out[i] = res[i];
    *n_out = (int32_t)res.size();
  });
}

// ----------------------------------------------------------- aggregate ---
int prism_hash_aggregate_batches(prism_ctx* c, const prism_batch* const* batches, int32_t n, const prism_agg_config* cfg,
                                 prism_batch** out) {
  return run(c, [&] {
    if (!cfg || !out || (n > 0 && !batches)) fail(PRISM_ERR_INVALID_ARGUMENT, "null config/batches/output");
    std::vector<const Batch*> bs;
    for (int i = 0; i < n; ++i) bs.push_back(&B(batches[i]));
    *out = wrap(c, aggregate(c->impl, bs, *cfg, nullptr, nullptr, 0, nullptr, 0, PRISM_ARITH_F64, false,
                             agg_tuning_for(total_rows(bs))));
  });
}

int prism_hash_aggregate(prism_ctx* c, const prism_batch* batch, const prism_agg_config* cfg, prism_batch** out) {
  const prism_batch* one[1] = {batch};
  return prism_hash_aggregate_batches(c, one, 1, cfg, out);
}

// -------------------------------------------------------- filter/project -
int prism_evaluate_predicate(prism_ctx* c, const prism_batch* b, const prism_predicate* p, prism_batch** out) {
  return run(c, [&] {
    if (!p || !out) fail(PRISM_ERR_INVALID_ARGUMENT, "null predicate/output");
    Batch r;
    r.rows = B(b).rows;
    r.cols.push_back(evaluate_predicate(c->impl, B(b), *p));
    *out = wrap(c, std::move(r));
  });
}

int prism_filter_batch(prism_ctx* c, const prism_batch* b, const prism_batch* mask, prism_batch** out) {
  return run(c, [&] {
    if (!out) fail(PRISM_ERR_INVALID_ARGUMENT, "null output");
    const Batch& m = B(mask);
    if (m.cols.size() != 1) fail(PRISM_ERR_INVALID_ARGUMENT, "mask must be a one-column Boolean batch");
    *out = wrap(c, filter_by_mask(c->impl, B(b), *m.cols[0]));
  });
}

int prism_project_batch(prism_ctx* c, const prism_batch* b, const int32_t* cols, int32_t n, prism_batch** out) {
  return run(c, [&] {
    if (!out || (n > 0 && !cols)) fail(PRISM_ERR_INVALID_ARGUMENT, "null columns/output");
    *out = wrap(c, project(B(b), cols, n));
  });
}

int prism_filter_and_project(prism_ctx* c, const prism_batch* b, const prism_predicate* p, const int32_t* cols, int32_t n,
                             prism_batch** out) {
  return run(c, [&] {
    if (!out || (n > 0 && !cols)) fail(PRISM_ERR_INVALID_ARGUMENT, "null columns/output");
    Batch f = B(b);
    if (p) {
      ColP m = evaluate_predicate(c->impl, f, *p);
      f = filter_by_mask(c->impl, f, *m);
    }
    *out = wrap(c, n == 0 ? f : project(f, cols, n));
  });
}

int prism_evaluate_scalar_expr(prism_ctx* c, const prism_batch* b, const prism_expr* e, int32_t mode, prism_batch** out) {
  return run(c, [&] {
    if (!e || !out) fail(PRISM_ERR_INVALID_ARGUMENT, "null expression/output");
    Batch r = project_with_exprs(c->impl, B(b), nullptr, 0, e, 1, mode);
    *out = wrap(c, std::move(r));
  });
}

int prism_project_batch_with_exprs(prism_ctx* c, const prism_batch* b, const int32_t* cols, int32_t n,
                                   const prism_expr* exprs, int32_t n_exprs, int32_t mode, prism_batch** out) {
  return run(c, [&] {
    if (!out || (n > 0 && !cols) || (n_exprs > 0 && !exprs)) fail(PRISM_ERR_INVALID_ARGUMENT, "null arguments");
    *out = wrap(c, project_with_exprs(c->impl, B(b), cols, n, exprs, n_exprs, mode));
  });
}

// --------------------------------------------------------------- fused ---
int prism_filter_project_aggregate(prism_ctx* c, const prism_batch* const* batches, int32_t n, const prism_predicate* p,
                                   const int32_t* cols, int32_t n_cols, const prism_expr* exprs, int32_t n_exprs,
                                   int32_t mode, const prism_agg_config* agg, prism_batch** out) {
  return run(c, [&] {
    if (!agg || !out || (n > 0 && !batches)) fail(PRISM_ERR_INVALID_ARGUMENT, "null arguments");
    std::vector<const Batch*> bs;
    for (int i = 0; i < n; ++i) bs.push_back(&B(batches[i]));
    try {
      *out = wrap(c, aggregate(c->impl, bs, *agg, p, cols, n_cols, exprs, n_exprs, mode, true, agg_tuning_for(total_rows(bs))));
      return;
    } catch (const Failure& f) {
      if (f.code != PRISM_ERR_INVALID_ARGUMENT || f.msg.find("fused path") == std::string::npos) throw;
    }
    // shapes the one-pass kernel does not take: filter, project, then aggregate
    std::vector<Batch> mats;
    for (auto* b : bs) {
      Batch f = *b;
      if (p) {
        ColP m = evaluate_predicate(c->impl, f, *p);
        f = filter_by_mask(c->impl, f, *m);
      }
      mats.push_back(project_with_exprs(c->impl, f, cols, n_cols, exprs, n_exprs, mode));
    }
    std::vector<const Batch*> ms;
    for (auto& m : mats) ms.push_back(&m);
    *out = wrap(c, aggregate(c->impl, ms, *agg, nullptr, nullptr, 0, nullptr, 0, mode, false, agg_tuning_for(total_rows(ms))));
  });
}

int prism_join_aggregate(prism_ctx* c, const prism_batch* const* probes, int32_t n_probes, const prism_batch* build,
                         const int32_t* probe_keys, const int32_t* build_keys, int32_t n_keys, const int32_t* cols,
                         int32_t n_cols, const prism_expr* exprs, int32_t n_exprs, const prism_agg_config* agg,
                         prism_batch** out) {
  return run(c, [&] {
    if (!agg || !out || n_probes <= 0 || !probes) fail(PRISM_ERR_INVALID_ARGUMENT, "null arguments");
    std::vector<int> pk = ints(probe_keys, n_keys), bk = ints(build_keys, n_keys);
    std::vector<const Batch*> pbs;
    for (int i = 0; i < n_probes; ++i) pbs.push_back(&B(probes[i]));
    const Batch& bb = B(build);
    AggTuning tune = agg_tuning();
    apply_join_agg_tuning(join_shape(bb, bk), tune);
    *out = wrap(c, join_aggregate_impl(c->impl, pbs, bb, pk, bk, cols, n_cols, exprs, n_exprs, agg, tune));
  });
}

// ----------------------------------------------------------- autotuner --
namespace {

// Times `fn` on the context's stream with CUDA events: one warm-up run, then
// the median of `reps` runs (milliseconds).
double time_ms(Ctx& x, int reps, const std::function<void()>& fn) {
  fn();
  x.sync();
  cudaEvent_t a, b;
  PRISM_CUDA(cudaEventCreate(&a));
  PRISM_CUDA(cudaEventCreate(&b));
  std::vector<double> t;
  for (int i = 0; i < reps; ++i) {
    PRISM_CUDA(cudaEventRecord(a, x.stream));
    fn();
    PRISM_CUDA(cudaEventRecord(b, x.stream));
    PRISM_CUDA(cudaEventSynchronize(b));
    float ms = 0;
    PRISM_CUDA(cudaEventElapsedTime(&ms, a, b));
    t.push_back(ms);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  std::sort(t.begin(), t.end());
  return t[t.size() / 2];
}

void put_result(prism_tune_result* r, const std::vector<std::string>& desc, const std::vector<double>& ms, int best) {
  if (!r) return;
  *r = prism_tune_result{};
  r->n_candidates = (int32_t)std::min<size_t>(desc.size(), PRISM_TUNE_MAX_CANDIDATES);
  r->best = best;
  for (int i = 0; i < r->n_candidates; ++i) {
    r->ms[i] = ms[i];
    std::snprintf(r->desc[i], sizeof r->desc[i], "%s", desc[i].c_str());
  }
}

std::string join_desc(const JoinTuning& t) {
  char b[64];
  if (t.dense) std::snprintf(b, sizeof b, "dense rows");
  else if (t.partition > 0) std::snprintf(b, sizeof b, "hash lf=%.2f partitioned 2^%d", t.load_factor, t.partition_bits);
  else std::snprintf(b, sizeof b, "hash lf=%.2f streamed", t.load_factor);
  return b;
}

}  // namespace

int prism_tune_join(prism_ctx* c, const prism_batch* build, const prism_batch* probe, const int32_t* build_keys,
                    const int32_t* probe_keys, int32_t n_keys, uint32_t flags, prism_tune_result* result) {
  return run(c, [&] {
    if (flags & ~(uint32_t)PRISM_JOIN_ANY_ORDER) fail(PRISM_ERR_INVALID_ARGUMENT, "unknown join flags");
    Ctx& x = c->impl;
    const Batch& bb = B(build);
    const Batch& pb = B(probe);
    std::vector<int> bk = ints(build_keys, n_keys), pk = ints(probe_keys, n_keys);
    check_join_keys(pb, pk, bb, bk);
    const JoinShape shape = join_shape(bb, bk);
    const bool any = (flags & PRISM_JOIN_ANY_ORDER) != 0;
    // candidates: the dense row table (unique compact Int64 keys), hash slots
    // at two load factors, and for Int64 keys the radix-partitioned build and
    // probe at two fan-outs
    std::vector<JoinTuning> cand;
    auto mk = [](bool dense, double lf, int part, int bits) {
      JoinTuning t;
      t.dense = dense;
      t.load_factor = lf;
      t.partition = part;
      t.partition_bits = bits;
      return t;
    };
    if (shape.key_kind == 0) cand.push_back(mk(true, 0.5, 0, 8));
    for (double lf : {0.5, 0.7}) {
      cand.push_back(mk(false, lf, 0, 8));
      if (shape.key_kind == 1 || any) {  // general keys: the partitioned build alone
        cand.push_back(mk(false, lf, 1, 8));
        cand.push_back(mk(false, lf, 1, 6));
      }
    }
    std::vector<double> ms;
    std::vector<std::string> desc;
    std::vector<JoinTuning> kept;
    int best = -1;
    for (const JoinTuning& jt : cand) {
      bool dense_taken = false;
      const double t = time_ms(x, 3, [&] {
        auto tab = build_join_table(x, bb, bk, jt);
        dense_taken = tab->dense;
        std::vector<ProbeGather> none;
        probe_join_table(x, *tab, pb, pk, true, true, none, -1, jt, any);
      });
      if (jt.dense && !dense_taken) continue;  // the keys do not allow the dense table
      ms.push_back(t);
      desc.push_back(join_desc(jt));
      kept.push_back(jt);
      if (best < 0 || t < ms[best]) best = (int)ms.size() - 1;
    }
    record_join_tuning(shape, kept[best]);
    put_result(result, desc, ms, best);
  });
}

int prism_tune_join_aggregate(prism_ctx* c, const prism_batch* const* probes, int32_t n_probes, const prism_batch* build,
                              const int32_t* probe_keys, const int32_t* build_keys, int32_t n_keys, const int32_t* cols,
                              int32_t n_cols, const prism_expr* exprs, int32_t n_exprs, const prism_agg_config* agg,
                              prism_tune_result* result) {
  return run(c, [&] {
    if (!agg || n_probes <= 0 || !probes) fail(PRISM_ERR_INVALID_ARGUMENT, "null arguments");
    Ctx& x = c->impl;
    std::vector<int> pk = ints(probe_keys, n_keys), bk = ints(build_keys, n_keys);
    std::vector<const Batch*> pbs;
    for (int i = 0; i < n_probes; ++i) pbs.push_back(&B(probes[i]));
    const Batch& bb = B(build);
    // fused kernel shapes: (threads per block, blocks per SM, probe rows in
    // flight per thread, log2 of the block's group-table slots)
    const int shapes[][4] = {{512, 3, 2, 9}, {512, 2, 2, 10}, {1024, 1, 2, 9}, {256, 6, 2, 9},
                             {512, 4, 1, 9}, {512, 3, 4, 9},  {256, 4, 4, 9},  {1024, 2, 1, 8}};
    std::vector<double> ms;
    std::vector<std::string> desc;
    std::vector<AggTuning> tried;
    int best = -1;
    for (auto& sh : shapes) {
      AggTuning t = agg_tuning();
      t.join_block = sh[0];
      t.join_min_blocks = sh[1];
      t.join_rows = sh[2];
      t.join_table_log2 = sh[3];
      const double v = time_ms(x, 2, [&] {
        join_aggregate_impl(x, pbs, bb, pk, bk, cols, n_cols, exprs, n_exprs, agg, t);
      });
      char d[64];
      std::snprintf(d, sizeof d, "block %d x %d/SM, %d rows, 2^%d slots", sh[0], sh[1], sh[2], sh[3]);
      ms.push_back(v);
      desc.push_back(d);
      tried.push_back(t);
      if (best < 0 || v < ms[best]) best = (int)ms.size() - 1;
    }
    record_join_agg_tuning(join_shape(bb, bk), tried[best]);
    put_result(result, desc, ms, best);
  });
}

int prism_tune_hash_aggregate(prism_ctx* c, const prism_batch* const* batches, int32_t n, const prism_agg_config* cfg,
                              prism_tune_result* result) {
  return run(c, [&] {
    if (!cfg || n < 0 || (n > 0 && !batches)) fail(PRISM_ERR_INVALID_ARGUMENT, "null arguments");
    Ctx& x = c->impl;
    std::vector<const Batch*> bs;
    for (int i = 0; i < n; ++i) bs.push_back(&B(batches[i]));
    std::vector<double> ms;
    std::vector<std::string> desc;
    std::vector<AggTuning> tried;
    int best = -1;
    for (int block : {256, 512, 1024}) {
      AggTuning t = agg_tuning();
      t.hash_block = block;
      const double v = time_ms(x, 3, [&] {
        aggregate(x, bs, *cfg, nullptr, nullptr, 0, nullptr, 0, PRISM_ARITH_F64, false, t);
      });
      ms.push_back(v);
      desc.push_back("hashed groups block " + std::to_string(block));
      tried.push_back(t);
      if (best < 0 || v < ms[best]) best = (int)ms.size() - 1;
    }
    record_agg_tuning(total_rows(bs), tried[best]);
    put_result(result, desc, ms, best);
  });
}

int prism_tuning_save(const char* path) {
  try {
    if (!path) fail(PRISM_ERR_INVALID_ARGUMENT, "null path");
    tuning_save(path);
    return PRISM_OK;
  } catch (const Failure& f) {
    t_err = f.msg;
    return f.code;
  }
}

int prism_tuning_load(const char* path) {
  try {
    if (!path) fail(PRISM_ERR_INVALID_ARGUMENT, "null path");
    tuning_load(path);
    return PRISM_OK;
  } catch (const Failure& f) {
    t_err = f.msg;
    return f.code;
  }
}

void prism_tuning_clear(void) { tuning_clear(); }

int64_t prism_tuning_dump(char* buf, int64_t capacity) {
  const std::string d = tuning_dump();
  if (buf && capacity > 0) {
    const size_t n = std::min<size_t>(d.size(), (size_t)capacity - 1);
    std::memcpy(buf, d.data(), n);
    buf[n] = 0;
  }
  return (int64_t)d.size();
}

// ------------------------------------------------------------------ sort --
int prism_sort_batch(prism_ctx* c, const prism_batch* b, const prism_sort_key* keys, int32_t n_keys, int64_t limit,
                     prism_batch** out) {
  return run(c, [&] {
    if (!out || (n_keys > 0 && !keys) || n_keys < 0) fail(PRISM_ERR_INVALID_ARGUMENT, "null arguments");
    *out = wrap(c, sort_batch(c->impl, B(b), keys, n_keys, limit));
  });
}

// ---------------------------------------------------------------- parquet --
static ParquetScanArgs scan_args(const prism_parquet_scan_config* cfg) {
    if (!cfg || (cfg->n_uris > 0 && !cfg->uris) || cfg->n_uris < 0 ||
        (cfg->n_projection > 0 && !cfg->projection) || cfg->n_projection < 0)
      fail(PRISM_ERR_INVALID_ARGUMENT, "null scan config");
    ParquetScanArgs a;
    for (int i = 0; i < cfg->n_uris; ++i) {
      if (!cfg->uris[i]) fail(PRISM_ERR_INVALID_ARGUMENT, "null URI");
      a.uris.push_back(cfg->uris[i]);
    }
    a.predicate = cfg->predicate;
    a.has_projection = cfg->projection != nullptr;
    if (a.has_projection) a.projection.assign(cfg->projection, cfg->projection + cfg->n_projection);
    a.batch_size = cfg->batch_size;
    a.skip_expand = cfg->skip_expand != 0;
    if (cfg->target_schema) {
      // ParquetScanConfig.target_schema (parquet_scan.rs:45-50): a struct schema
      const ArrowSchema* ts = cfg->target_schema;
      if (!ts->format || std::string(ts->format) != "+s" || (ts->n_children > 0 && !ts->children))
        fail(PRISM_ERR_INVALID_ARGUMENT, "target_schema must be a struct schema (format '+s')");
      a.has_target = true;
      for (int64_t i = 0; i < ts->n_children; ++i) {
        const ArrowSchema* f = ts->children[i];
        TargetField t;
        t.name = f->name ? f->name : "";
        t.nullable = (f->flags & ARROW_FLAG_NULLABLE) != 0;
        if (f->dictionary || !arrow_format_type(f->format, t.type, t.precision, t.scale) || t.type == TY_NULL)
          fail(PRISM_ERR_INVALID_ARGUMENT, "target_schema field '" + t.name + "' has a type the engine does not hold");
        a.target.push_back(t);
      }
    }
    return a;
}

static void batch_array(prism_ctx* c, std::vector<Batch>& bs, prism_batch*** out, int32_t* n_out) {
  auto** arr = static_cast<prism_batch**>(std::malloc(sizeof(prism_batch*) * std::max<size_t>(bs.size(), 1)));
  if (!arr) fail(PRISM_ERR_NO_MEMORY, "host allocation failed");
  for (size_t i = 0; i < bs.size(); ++i) arr[i] = wrap(c, std::move(bs[i]));
  *out = arr;
  *n_out = (int32_t)bs.size();
}

static void put_stats(const ParquetScanStats& st, prism_parquet_scan_stats* stats) {
  if (stats)
    *stats = {st.files, st.row_groups, st.row_groups_skipped, st.pages, st.compressed_bytes, st.inflated_bytes,
              st.decoded_bytes};
}

int prism_parquet_scan(prism_ctx* c, const prism_parquet_scan_config* cfg, prism_batch*** out, int32_t* n_out,
                       prism_parquet_scan_stats* stats) {
  return run(c, [&] {
    if (!out || !n_out) fail(PRISM_ERR_INVALID_ARGUMENT, "null output");
    *out = nullptr;
    *n_out = 0;
    ParquetScanStats st;
    std::vector<Batch> bs = parquet_scan(c->impl, scan_args(cfg), &st);
    put_stats(st, stats);
    batch_array(c, bs, out, n_out);
  });
}

struct prism_parquet_prepared {
  std::shared_ptr<prism::ParquetPrepared> impl;
};

int prism_parquet_prepare(prism_ctx* c, const prism_parquet_scan_config* cfg, prism_parquet_prepared** out,
                          prism_parquet_scan_stats* stats) {
  return run(c, [&] {
    if (!out) fail(PRISM_ERR_INVALID_ARGUMENT, "null output");
    ParquetScanStats st;
    auto p = parquet_prepare(c->impl, scan_args(cfg), &st);
    put_stats(st, stats);
    *out = new prism_parquet_prepared{std::move(p)};
  });
}

int prism_parquet_decode(prism_ctx* c, const prism_parquet_prepared* p, prism_batch*** out, int32_t* n_out,
                         prism_parquet_scan_stats* stats) {
  return run(c, [&] {
    if (!p || !out || !n_out) fail(PRISM_ERR_INVALID_ARGUMENT, "null prepared scan/output");
    *out = nullptr;
    *n_out = 0;
    ParquetScanStats st;
    std::vector<Batch> bs = parquet_decode(c->impl, *p->impl, &st);
    put_stats(st, stats);
    batch_array(c, bs, out, n_out);
  });
}

int64_t prism_parquet_prepared_rows(const prism_parquet_prepared* p) { return p ? parquet_prepared_rows(*p->impl) : -1; }
int64_t prism_parquet_prepared_bytes(const prism_parquet_prepared* p) { return p ? parquet_prepared_bytes(*p->impl) : -1; }
void prism_parquet_prepared_free(prism_parquet_prepared* p) { delete p; }

int prism_parquet_row_count(const char* const* uris, int32_t n, const prism_predicate* pred, int64_t* count) {
  try {
    if (!count || n < 0 || (n > 0 && !uris)) fail(PRISM_ERR_INVALID_ARGUMENT, "null arguments");
    std::vector<std::string> u;
    for (int i = 0; i < n; ++i) {
      if (!uris[i]) fail(PRISM_ERR_INVALID_ARGUMENT, "null URI");
      u.push_back(uris[i]);
    }
    *count = parquet_row_count(u, pred);
    return PRISM_OK;
  } catch (const Failure& f) {
    t_err = f.msg;
    return f.code;
  } catch (const std::exception& e) {
    t_err = e.what();
    return PRISM_ERR_INTERNAL;
  }
}

void prism_free_array(void* a) { std::free(a); }

// ------------------------------------------- distributed aggregation --
int prism_expand_worker_aggregates(const prism_agg_config* original, prism_agg_expr* out_aggs, int32_t capacity,
                                   int32_t* n_out) {
  try {
    if (!original || !n_out) fail(PRISM_ERR_INVALID_ARGUMENT, "null config/output");
    const WorkerAggs w = expand_worker_aggregates(*original);
    *n_out = (int32_t)w.aggs.size();
    if ((int32_t)w.aggs.size() > capacity || (!out_aggs && !w.aggs.empty()))
      fail(PRISM_ERR_INVALID_ARGUMENT, "worker aggregate list longer than the output capacity");
    for (size_t i = 0; i < w.aggs.size(); ++i) out_aggs[i] = w.aggs[i];
    return PRISM_OK;
  } catch (const Failure& f) {
    t_err = f.msg;
    return f.code;
  }
}

int prism_batch_packed_size(const prism_batch* b, uint64_t* size) {
  try {
    if (!size) fail(PRISM_ERR_INVALID_ARGUMENT, "null output");
    *size = packed_size(B(b));
    return PRISM_OK;
  } catch (const Failure& f) {
    t_err = f.msg;
    return f.code;
  }
}

int prism_batch_pack(prism_ctx* c, const prism_batch* b, void* dst, uint64_t capacity) {
  return run(c, [&] { pack_batch(c->impl, B(b), dst, capacity); });
}

int prism_batch_unpack(prism_ctx* c, const void* src, uint64_t size, prism_batch** out) {
  return run(c, [&] {
    if (!out) fail(PRISM_ERR_INVALID_ARGUMENT, "null output");
    *out = wrap(c, unpack_batch(c->impl, src, size));
  });
}

int prism_arrow_packed_size(const ArrowArray* a, const ArrowSchema* s, uint64_t* size) {
  try {
    if (!size) fail(PRISM_ERR_INVALID_ARGUMENT, "null output");
    std::vector<std::shared_ptr<std::vector<uint8_t>>> keep;
    *size = packed_size(host_batch(a, s, keep));
    return PRISM_OK;
  } catch (const Failure& f) {
    t_err = f.msg;
    return f.code;
  }
}

int prism_arrow_pack(const ArrowArray* a, const ArrowSchema* s, void* dst, uint64_t capacity) {
  try {
    std::vector<std::shared_ptr<std::vector<uint8_t>>> keep;
    pack_host(host_batch(a, s, keep), dst, capacity);
    return PRISM_OK;
  } catch (const Failure& f) {
    t_err = f.msg;
    return f.code;
  }
}

int prism_arrow_unpack(const void* src, uint64_t size, ArrowArray* out, ArrowSchema* out_schema) {
  try {
    std::shared_ptr<std::vector<uint8_t>> payload;
    Batch b = unpack_host(src, size, payload);
    export_host_batch(b, payload, out, out_schema);
    return PRISM_OK;
  } catch (const Failure& f) {
    t_err = f.msg;
    return f.code;
  } catch (const std::bad_alloc&) {
    t_err = "host allocation failed";
    return PRISM_ERR_NO_MEMORY;
  }
}

int prism_merge_partial_aggregates(prism_ctx* c, const prism_batch* const* partials, int32_t n,
                                   const prism_agg_config* original, prism_batch** out) {
  return run(c, [&] {
    if (!original || !out || n < 0 || (n > 0 && !partials)) fail(PRISM_ERR_INVALID_ARGUMENT, "null config/partials/output");
    std::vector<const Batch*> ps;
    for (int i = 0; i < n; ++i) ps.push_back(&B(partials[i]));
    *out = wrap(c, merge_partial_aggregates(c->impl, ps, *original, agg_tuning()));
  });
}

// ------------------------------------------------------- arrow wrappers --
int prism_sort_batch_arrow(prism_ctx* c, const ArrowArray* batch, const ArrowSchema* s, const prism_sort_key* keys,
                           int32_t n_keys, int64_t limit, ArrowArray* out, ArrowSchema* os) {
  return run(c, [&] {
    prism_batch bw;
    bw.impl = import_batch(c->impl, batch, s, false);
    prism_batch* r = nullptr;
    int rc = prism_sort_batch(c, &bw, keys, n_keys, limit, &r);
    if (rc) fail(rc, c->impl.last_error);
    std::unique_ptr<prism_batch> hold(r);
    export_batch(c->impl, r->impl, out, os);
  });
}

int prism_hash_join_arrow(prism_ctx* c, const ArrowArray* probe, const ArrowSchema* ps, const ArrowArray* build,
                          const ArrowSchema* bs, const prism_join_config* cfg, ArrowArray* out, ArrowSchema* os) {
  return run(c, [&] {
    Batch p = import_batch(c->impl, probe, ps, false), b = import_batch(c->impl, build, bs, false);
    prism_batch pw, bw;
    pw.impl = p;
    bw.impl = b;
    prism_batch* r = nullptr;
    int rc = prism_hash_join(c, &pw, &bw, cfg, &r);
    if (rc) fail(rc, c->impl.last_error);
    std::unique_ptr<prism_batch> hold(r);
    export_batch(c->impl, r->impl, out, os);
  });
}

int prism_hash_aggregate_arrow(prism_ctx* c, const ArrowArray* batch, const ArrowSchema* s, const prism_agg_config* cfg,
                               ArrowArray* out, ArrowSchema* os) {
  return run(c, [&] {
    prism_batch bw;
    bw.impl = import_batch(c->impl, batch, s, false);
    prism_batch* r = nullptr;
    int rc = prism_hash_aggregate(c, &bw, cfg, &r);
    if (rc) fail(rc, c->impl.last_error);
    std::unique_ptr<prism_batch> hold(r);
    export_batch(c->impl, r->impl, out, os);
  });
}

int prism_filter_and_project_arrow(prism_ctx* c, const ArrowArray* batch, const ArrowSchema* s, const prism_predicate* p,
                                   const int32_t* cols, int32_t n, ArrowArray* out, ArrowSchema* os) {
  return run(c, [&] {
    prism_batch bw;
    bw.impl = import_batch(c->impl, batch, s, false);
    prism_batch* r = nullptr;
    int rc = prism_filter_and_project(c, &bw, p, cols, n, &r);
    if (rc) fail(rc, c->impl.last_error);
    std::unique_ptr<prism_batch> hold(r);
    export_batch(c->impl, r->impl, out, os);
  });
}

}  // extern "C"
