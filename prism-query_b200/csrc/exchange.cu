// exchange.cu — pack / unpack of device batches for a collective, and the
// reducer merge of per-worker partial aggregates on the GPU.
//
// The reference's distributed aggregation (prism-bench/src/handler.rs:270-344)
// runs the plan on every worker with the aggregates expanded (AVG -> SUM +
// COUNT), ships each worker's partial batch to one reducer over Flight, and
// the reducer runs hash_aggregate_batches over [its own partial, then the
// peers'] with SUM for SUM/COUNT/COUNT DISTINCT partials and MIN/MAX for
// MIN/MAX partials, then rebuilds the original aggregates (COUNT as Int64,
// AVG = SUM / COUNT, 0 when the count is 0, a null read as 0). Here the
// transport is one all-gather of packed device buffers (NCCL over NVLink),
// and the merge is this library's GPU aggregation plus one elementwise
// kernel, so partial tables never leave HBM.
//
// Packed layout (little-endian, every region 16-byte aligned):
//   PackHead | PackEntry x n_entries | entry names | buffers...
// Entries list the top-level columns in order; a dictionary column's value
// column follows it as an extra entry whose `parent` is the column's entry.
// Buffer offsets are relative to the start of the packed buffer; ~0 marks an
// absent buffer.
#include <algorithm>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>

#include "agg.hpp"
#include "exchange.hpp"

namespace prism {

namespace {

constexpr uint64_t PACK_MAGIC = 0x314B50534D495250ULL;  // "PRISMPK1"
constexpr uint64_t ABSENT = ~0ULL;

struct PackHead {
  uint64_t magic;
  uint64_t header_bytes;
  uint64_t total_bytes;
  int64_t rows;
  int64_t n_cols;
  int64_t n_entries;
};

struct PackEntry {
  int32_t type, index_type, precision, scale;
  int32_t nullable, parent, data_base, name_len;
  int64_t length, data_bytes;
  uint64_t dict_fingerprint;
  uint64_t off[4];  // validity, values, offsets, data
};
static_assert(sizeof(PackHead) == 48 && sizeof(PackEntry) == 88, "packed header layout");

inline uint64_t align16(uint64_t x) { return (x + 15) & ~15ULL; }

struct Piece {
  const void* src;
  uint64_t bytes;
};

// Sizes of a column's four buffers (validity, values, offsets, data).
void buffer_sizes(const Column& c, uint64_t sz[4], const void* ptr[4]) {
  const uint64_t n = (uint64_t)c.length;
  sz[0] = c.validity ? (n + 7) / 8 : 0;
  ptr[0] = c.validity;
  if (c.type == TY_BOOL) sz[1] = (n + 7) / 8;
  else if (c.type == TY_DICT) sz[1] = (uint64_t)width_of(c.index_type) * n;
  else sz[1] = (uint64_t)width_of(c.type) * n;
  ptr[1] = c.values;
  if (!c.values) sz[1] = 0;
  sz[2] = (c.type == TY_UTF8 && c.offsets) ? (n + 1) * 4 : 0;
  ptr[2] = c.offsets;
  sz[3] = (c.type == TY_UTF8 && c.data) ? (uint64_t)c.data_bytes : 0;
  ptr[3] = c.data;
}

// Header entries and payload pieces of `b`, offsets assigned.
struct Layout {
  std::vector<PackEntry> entries;
  std::vector<std::string> names;
  std::vector<std::pair<uint64_t, Piece>> pieces;  // (offset, piece)
  uint64_t header_bytes = 0, total = 0;
};

Layout layout_of(const Batch& b) {
  Layout L;
  std::vector<const Column*> cols;
  auto add = [&](const Column& c, int parent) {
    PackEntry e{};
    e.type = c.type;
    e.index_type = c.index_type;
    e.precision = c.precision;
    e.scale = c.scale;
    e.nullable = c.nullable ? 1 : 0;
    e.parent = parent;
    e.data_base = c.data_base;
    e.name_len = (int32_t)c.name.size();
    e.length = c.length;
    e.data_bytes = c.type == TY_UTF8 ? c.data_bytes : 0;
    e.dict_fingerprint = c.dict_fingerprint;
    L.entries.push_back(e);
    L.names.push_back(c.name);
    cols.push_back(&c);
  };
  for (const auto& c : b.cols) {
    const int at = (int)L.entries.size();
    add(*c, -1);
    if (c->type == TY_DICT) {
      if (!c->dict) fail(PRISM_ERR_INVALID_ARGUMENT, "dictionary column without values");
      add(*c->dict, at);
    }
  }
  uint64_t h = sizeof(PackHead) + L.entries.size() * sizeof(PackEntry);
  for (const auto& nm : L.names) h += (nm.size() + 7) & ~7ULL;
  L.header_bytes = align16(h);
  uint64_t pos = L.header_bytes;
  for (size_t i = 0; i < L.entries.size(); ++i) {
    uint64_t sz[4];
    const void* ptr[4];
    buffer_sizes(*cols[i], sz, ptr);
    for (int k = 0; k < 4; ++k) {
      if (!ptr[k]) {
        L.entries[i].off[k] = ABSENT;
        continue;
      }
      L.entries[i].off[k] = pos;
      if (sz[k]) L.pieces.push_back({pos, Piece{ptr[k], sz[k]}});
      pos += std::max<uint64_t>(16, align16(sz[k]));  // an empty buffer still gets an address
    }
  }
  L.total = pos;
  return L;
}

std::vector<uint8_t> header_bytes(const Batch& b, const Layout& L) {
  std::vector<uint8_t> h(L.header_bytes, 0);
  PackHead head{PACK_MAGIC, L.header_bytes, L.total, b.rows, (int64_t)b.cols.size(), (int64_t)L.entries.size()};
  std::memcpy(h.data(), &head, sizeof head);
  std::memcpy(h.data() + sizeof head, L.entries.data(), L.entries.size() * sizeof(PackEntry));
  uint64_t p = sizeof head + L.entries.size() * sizeof(PackEntry);
  for (const auto& nm : L.names) {
    std::memcpy(h.data() + p, nm.data(), nm.size());
    p += (nm.size() + 7) & ~7ULL;
  }
  return h;
}

bool valid_type(int32_t t) { return t >= TY_NULL && t <= TY_DICT; }

// Rust's `f64 as i64`: saturating, NaN -> 0 (handler.rs:558 via numeric_value_as_i64)
__device__ __forceinline__ long long sat_i64(double v) {
  if (v != v) return 0;
  if (v >= 9223372036854775807.0) return 9223372036854775807LL;
  if (v <= -9223372036854775808.0) return (-9223372036854775807LL - 1);
  return (long long)v;
}

// numeric_value_as_f64 / numeric_value_as_i64 (handler.rs:533-568): a null
// reads as 0; Float64, Int64 and Int32 columns are accepted.
__device__ __forceinline__ double num_f64(const DCol& c, int64_t i) {
  if (!dcol_valid(c, i)) return 0.0;
  if (c.type == TY_F64) return static_cast<const double*>(c.values)[i];
  if (c.type == TY_I64) return (double)static_cast<const long long*>(c.values)[i];
  return (double)static_cast<const int*>(c.values)[i];
}
__device__ __forceinline__ long long num_i64(const DCol& c, int64_t i) {
  if (!dcol_valid(c, i)) return 0;
  if (c.type == TY_F64) return sat_i64(static_cast<const double*>(c.values)[i]);
  if (c.type == TY_I64) return static_cast<const long long*>(c.values)[i];
  return static_cast<const int*>(c.values)[i];
}

enum RebuildKind : int32_t { RB_F64 = 0, RB_I64 = 1, RB_AVG = 2 };

// reconstruct_original_aggregate_batch (handler.rs:459-530), one column per launch
__global__ void rebuild_kernel(int32_t kind, DCol src, DCol cnt, void* out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    if (kind == RB_I64) {
      static_cast<long long*>(out)[i] = num_i64(src, i);
    } else if (kind == RB_AVG) {
      const double s = num_f64(src, i), c = num_f64(cnt, i);
      static_cast<double*>(out)[i] = c > 0.0 ? s / c : 0.0;
    } else {
      static_cast<double*>(out)[i] = num_f64(src, i);
    }
  }
}

// "agg_<i>" names with process lifetime (the expanded configs point at them)
const char* worker_name(size_t i) {
  static std::mutex mu;
  static std::deque<std::string> names;
  std::lock_guard<std::mutex> lk(mu);
  while (names.size() <= i) names.push_back("agg_" + std::to_string(names.size()));
  return names[i].c_str();
}

}  // namespace

WorkerAggs expand_worker_aggregates(const prism_agg_config& original) {
  if (original.n_aggs < 0 || (original.n_aggs > 0 && !original.aggs))
    fail(PRISM_ERR_INVALID_ARGUMENT, "null aggregate list");
  WorkerAggs w;
  for (int i = 0; i < original.n_aggs; ++i) {
    const prism_agg_expr& a = original.aggs[i];
    if (a.func < PRISM_AGG_SUM || a.func > PRISM_AGG_COUNT_DISTINCT)
      fail(PRISM_ERR_INVALID_ARGUMENT, "unknown aggregate function");
    if (a.func == PRISM_AGG_AVG) {
      const int32_t s = (int32_t)w.aggs.size();
      w.aggs.push_back({a.column, PRISM_AGG_SUM, worker_name(s)});
      w.aggs.push_back({a.column, PRISM_AGG_COUNT, worker_name(s + 1)});
      w.map.push_back(s);
      w.map.push_back(s + 1);
    } else {
      const int32_t s = (int32_t)w.aggs.size();
      w.aggs.push_back({a.column, a.func, worker_name(s)});
      w.map.push_back(s);
      w.map.push_back(-1);
    }
  }
  return w;
}

uint64_t packed_size(const Batch& b) { return layout_of(b).total; }

void pack_batch(Ctx& ctx, const Batch& b, void* dst, uint64_t capacity) {
  const Layout L = layout_of(b);
  if (!dst) fail(PRISM_ERR_INVALID_ARGUMENT, "null pack destination");
  if (capacity < L.total) fail(PRISM_ERR_INVALID_ARGUMENT, "pack destination smaller than the packed size");
  const std::vector<uint8_t> h = header_bytes(b, L);
  uint8_t* d = static_cast<uint8_t*>(dst);
  ctx.h2d_staged(d, h.data(), h.size());  // (copied out of `h` before this returns)
  for (const auto& p : L.pieces)
    PRISM_CUDA(cudaMemcpyAsync(d + p.first, p.second.src, p.second.bytes, cudaMemcpyDeviceToDevice, ctx.stream));
}

namespace {

void check_head(const PackHead& head, uint64_t size) {
  if (head.magic != PACK_MAGIC) fail(PRISM_ERR_INVALID_ARGUMENT, "not a packed batch");
  if (head.header_bytes < sizeof head || head.header_bytes > head.total_bytes || head.total_bytes > size ||
      head.n_entries < head.n_cols || head.n_cols < 0 || head.rows < 0 ||
      (uint64_t)head.n_entries > (head.header_bytes - sizeof head) / sizeof(PackEntry))
    fail(PRISM_ERR_INVALID_ARGUMENT, "packed batch header out of range");
}

// The columns described by a packed header `h` (host bytes), with every
// buffer at payload + (offset - header_bytes); `hold` (if any) owns the payload.
Batch parse_packed(const PackHead& head, const std::vector<uint8_t>& h, uint8_t* payload, const MemP& hold) {
  std::vector<PackEntry> ents((size_t)head.n_entries);
  std::memcpy(ents.data(), h.data() + sizeof head, ents.size() * sizeof(PackEntry));
  uint64_t p = sizeof head + ents.size() * sizeof(PackEntry);
  std::vector<ColP> all;
  Batch out;
  out.rows = head.rows;
  for (const PackEntry& e : ents) {
    if (!valid_type(e.type) || e.length < 0 || e.name_len < 0 || e.data_bytes < 0)
      fail(PRISM_ERR_INVALID_ARGUMENT, "packed column descriptor out of range");
    if (p + (uint64_t)e.name_len > head.header_bytes) fail(PRISM_ERR_INVALID_ARGUMENT, "packed column name out of range");
    auto c = std::make_shared<Column>();
    c->type = e.type;
    c->index_type = e.index_type;
    c->precision = e.precision;
    c->scale = e.scale;
    c->nullable = e.nullable != 0;
    c->data_base = e.data_base;
    c->length = e.length;
    c->data_bytes = e.data_bytes;
    c->dict_fingerprint = e.dict_fingerprint;
    c->name.assign(reinterpret_cast<const char*>(h.data() + p), (size_t)e.name_len);
    p += ((uint64_t)e.name_len + 7) & ~7ULL;
    uint64_t sz[4];
    const void* ptr[4];
    Column probe = *c;  // sizes follow from type and length
    probe.validity = reinterpret_cast<uint8_t*>(1);
    probe.values = reinterpret_cast<void*>(1);
    probe.offsets = reinterpret_cast<int32_t*>(1);
    probe.data = reinterpret_cast<uint8_t*>(1);
    buffer_sizes(probe, sz, ptr);
    void* at[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int k = 0; k < 4; ++k) {
      if (e.off[k] == ABSENT) continue;
      if (e.off[k] < head.header_bytes || e.off[k] % 16 || e.off[k] > head.total_bytes ||
          sz[k] > head.total_bytes - e.off[k])
        fail(PRISM_ERR_INVALID_ARGUMENT, "packed buffer out of range");
      at[k] = payload + (e.off[k] - head.header_bytes);
    }
    const bool fixed = e.type != TY_UTF8 && e.type != TY_NULL;
    if ((fixed && !at[1] && e.length > 0) || (e.type == TY_UTF8 && !at[2] && e.length > 0))
      fail(PRISM_ERR_INVALID_ARGUMENT, "packed column misses a buffer");
    c->validity = static_cast<uint8_t*>(at[0]);
    c->values = at[1];
    c->offsets = static_cast<int32_t*>(at[2]);
    c->data = static_cast<uint8_t*>(at[3]);
    if (hold) c->owners.push_back(hold);
    if (e.parent >= 0) {
      if (e.parent >= (int32_t)all.size() || all[e.parent]->type != TY_DICT || all[e.parent]->dict)
        fail(PRISM_ERR_INVALID_ARGUMENT, "packed dictionary entry out of order");
      all[e.parent]->dict = c;
    } else {
      out.cols.push_back(c);
    }
    all.push_back(c);
  }
  if ((int64_t)out.cols.size() != head.n_cols) fail(PRISM_ERR_INVALID_ARGUMENT, "packed column count mismatch");
  for (const auto& c : out.cols) {
    if (c->length != head.rows) fail(PRISM_ERR_INVALID_ARGUMENT, "packed column length mismatch");
    if (c->type == TY_DICT && !c->dict) fail(PRISM_ERR_INVALID_ARGUMENT, "packed dictionary without values");
  }
  return out;
}

}  // namespace

Batch unpack_batch(Ctx& ctx, const void* src, uint64_t size) {
  if (!src) fail(PRISM_ERR_INVALID_ARGUMENT, "null packed buffer");
  if (size < sizeof(PackHead)) fail(PRISM_ERR_INVALID_ARGUMENT, "packed buffer shorter than its header");
  PackHead head{};
  PRISM_CUDA(cudaMemcpyAsync(&head, src, sizeof head, cudaMemcpyDeviceToHost, ctx.stream));
  ctx.sync();
  check_head(head, size);
  std::vector<uint8_t> h(head.header_bytes);
  PRISM_CUDA(cudaMemcpyAsync(h.data(), src, h.size(), cudaMemcpyDeviceToHost, ctx.stream));
  // one owned copy of the payload; columns point into it
  const uint64_t payload = head.total_bytes - head.header_bytes;
  MemP hold = ctx.alloc(std::max<uint64_t>(payload, 16));
  if (payload)
    PRISM_CUDA(cudaMemcpyAsync(hold->ptr, static_cast<const uint8_t*>(src) + head.header_bytes, payload,
                               cudaMemcpyDeviceToDevice, ctx.stream));
  ctx.sync();
  return parse_packed(head, h, static_cast<uint8_t*>(hold->ptr), hold);
}

void pack_host(const Batch& b, void* dst, uint64_t capacity) {
  const Layout L = layout_of(b);
  if (!dst) fail(PRISM_ERR_INVALID_ARGUMENT, "null pack destination");
  if (capacity < L.total) fail(PRISM_ERR_INVALID_ARGUMENT, "pack destination smaller than the packed size");
  const std::vector<uint8_t> h = header_bytes(b, L);
  uint8_t* d = static_cast<uint8_t*>(dst);
  std::memcpy(d, h.data(), h.size());
  std::memset(d + h.size(), 0, L.total - h.size());  // padding between buffers is defined
  for (const auto& p : L.pieces) std::memcpy(d + p.first, p.second.src, p.second.bytes);
}

Batch unpack_host(const void* src, uint64_t size, std::shared_ptr<std::vector<uint8_t>>& payload) {
  if (!src) fail(PRISM_ERR_INVALID_ARGUMENT, "null packed buffer");
  if (size < sizeof(PackHead)) fail(PRISM_ERR_INVALID_ARGUMENT, "packed buffer shorter than its header");
  PackHead head{};
  std::memcpy(&head, src, sizeof head);
  check_head(head, size);
  std::vector<uint8_t> h(static_cast<const uint8_t*>(src), static_cast<const uint8_t*>(src) + head.header_bytes);
  payload = std::make_shared<std::vector<uint8_t>>(
      static_cast<const uint8_t*>(src) + head.header_bytes, static_cast<const uint8_t*>(src) + head.total_bytes);
  if (payload->empty()) payload->resize(16);
  return parse_packed(head, h, payload->data(), nullptr);
}

Batch merge_partial_aggregates(Ctx& ctx, const std::vector<const Batch*>& partials, const prism_agg_config& original,
                               const AggTuning& tune) {
  if (original.n_group_by < 0) fail(PRISM_ERR_INVALID_ARGUMENT, "negative group-by count");
  if (partials.empty()) fail(PRISM_ERR_INVALID_ARGUMENT, "no partial batches to merge");
  const WorkerAggs w = expand_worker_aggregates(original);
  const int nk = original.n_group_by;
  const int want = nk + (int)w.aggs.size();
  for (const Batch* p : partials)
    if (!p || (int)p->cols.size() != want)
      fail(PRISM_ERR_INVALID_ARGUMENT, "partial batch does not have the group columns plus the worker aggregates");
  // build_final_merge_config (handler.rs:430-457)
  std::vector<int32_t> group_by(nk);
  for (int k = 0; k < nk; ++k) group_by[k] = k;
  std::vector<prism_agg_expr> maggs;
  for (size_t i = 0; i < w.aggs.size(); ++i) {
    const int32_t f = w.aggs[i].func;
    const int32_t mf = (f == PRISM_AGG_MIN || f == PRISM_AGG_MAX) ? f : PRISM_AGG_SUM;
    maggs.push_back({nk + (int32_t)i, mf, w.aggs[i].output_name});
  }
  prism_agg_config mc{nk, group_by.data(), (int32_t)maggs.size(), maggs.data()};
  Batch merged = aggregate(ctx, partials, mc, nullptr, nullptr, 0, nullptr, 0, PRISM_ARITH_F64, false, tune);
  // reconstruct_original_aggregate_batch (handler.rs:459-530)
  Batch out;
  out.rows = merged.rows;
  for (int k = 0; k < nk; ++k) out.cols.push_back(merged.cols[k]);
  const int64_t n = merged.rows;
  for (int i = 0; i < original.n_aggs; ++i) {
    const prism_agg_expr& a = original.aggs[i];
    const int32_t kind = (a.func == PRISM_AGG_COUNT || a.func == PRISM_AGG_COUNT_DISTINCT) ? RB_I64
                         : a.func == PRISM_AGG_AVG                                        ? RB_AVG
                                                                                         : RB_F64;
    ColP col = make_column(ctx, kind == RB_I64 ? TY_I64 : TY_F64, a.output_name ? a.output_name : "", n, false);
    const DCol src = merged.cols[nk + w.map[2 * i]]->view();
    const DCol cnt = kind == RB_AVG ? merged.cols[nk + w.map[2 * i + 1]]->view() : src;
    if (n > 0) {
      rebuild_kernel<<<grid_for(ctx, n, 256), 256, 0, ctx.stream>>>(kind, src, cnt, col->values, n);
      ctx.check_launch("rebuild_kernel");
    }
    out.cols.push_back(col);
  }
  return out;
}

}  // namespace prism
