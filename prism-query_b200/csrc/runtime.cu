// runtime.cu — context, allocator and column helpers.
#include <cstring>
#include "runtime.hpp"

namespace prism {

DevMem::~DevMem() {
  if (!ptr || borrowed || !ctx) return;
  cudaFreeAsync(ptr, ctx->stream);
  ctx->in_use.fetch_sub(bytes);
}

MemP Ctx::alloc(size_t bytes) {
  auto m = std::make_shared<DevMem>();
  m->ctx = this;
  if (bytes == 0) return m;
  size_t rounded = (bytes + 255) & ~size_t(255);
  uint64_t cur = in_use.load();
  if (budget && cur + rounded > budget)
    fail(PRISM_ERR_NO_MEMORY, "device memory budget exceeded: " + std::to_string(cur) + " + " +
                                  std::to_string(rounded) + " > " + std::to_string(budget));
  void* p = nullptr;
  cudaError_t e = cudaMallocFromPoolAsync(&p, rounded, pool, stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    if (e == cudaErrorMemoryAllocation)
      fail(PRISM_ERR_NO_MEMORY, "device allocation of " + std::to_string(rounded) + " bytes failed");
    fail(PRISM_ERR_CUDA, std::string("cudaMallocFromPoolAsync: ") + cudaGetErrorString(e));
  }
  m->ptr = p;
  m->bytes = rounded;
  in_use.fetch_add(rounded);
  return m;
}

void Ctx::check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) fail(PRISM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
  note_launch();
}

uint32_t Ctx::take_device_errors() {
  PRISM_CUDA(cudaMemcpyAsync(h_err, d_err, sizeof(uint32_t), cudaMemcpyDeviceToHost, stream));
  PRISM_CUDA(cudaStreamSynchronize(stream));
  uint32_t v = *h_err;
  if (v) PRISM_CUDA(cudaMemsetAsync(d_err, 0, sizeof(uint32_t), stream));
  return v;
}

void Ctx::sync() { PRISM_CUDA(cudaStreamSynchronize(stream)); }

void Ctx::h2d_staged(void* dst, const void* src, size_t bytes) {
  if (!h_stage || !stage_ev || bytes > stage_cap / 2) {
    PRISM_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream));
    PRISM_CUDA(cudaStreamSynchronize(stream));  // the source must outlive the copy
    return;
  }
  const size_t n = (bytes + 255) & ~(size_t)255;
  if (stage_head + n > stage_cap) {
    if (stage_pending) PRISM_CUDA(cudaEventSynchronize(stage_ev));  // the ring's earlier copies are done
    stage_head = 0;
  }
  uint8_t* p = h_stage + stage_head;
  std::memcpy(p, src, bytes);
  PRISM_CUDA(cudaMemcpyAsync(dst, p, bytes, cudaMemcpyHostToDevice, stream));
  PRISM_CUDA(cudaEventRecord(stage_ev, stream));
  stage_pending = true;
  stage_head += n;
}

cudaEvent_t Ctx::take_event() {
  if (!event_pool.empty()) {
    cudaEvent_t e = event_pool.back();
    event_pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  PRISM_CUDA(cudaEventCreate(&e));
  return e;
}

void Ctx::clear_timings() {
  for (auto& kv : timings)
    for (auto& pr : kv.second) {
      event_pool.push_back(pr.first);
      event_pool.push_back(pr.second);
    }
  timings.clear();
}

DCol Column::view() const {
  DCol d{};
  d.type = type;
  d.index_type = index_type;
  d.length = length;
  d.validity = validity;
  d.values = values;
  d.offsets = offsets;
  d.data = data ? data - data_base : nullptr;  // so that data + offsets[i] addresses row i
  d.scale = scale;
  if (type == TY_DICT && dict) {
    d.dict_offsets = dict->offsets;
    d.dict_data = dict->data ? dict->data - dict->data_base : nullptr;
    d.dict_length = dict->length;
    d.dict_type = dict->type;
  }
  return d;
}

ColP make_column(Ctx& ctx, int32_t type, const std::string& name, int64_t n, bool with_validity) {
  auto c = std::make_shared<Column>();
  c->type = type;
  c->name = name;
  c->length = n;
  c->nullable = true;
  int w = width_of(type);
  MemP m;
  if (type == TY_BOOL) {
    c->values = ctx.alloc_t<uint8_t>((size_t)(n + 7) / 8 + 8, m);
    c->owners.push_back(m);
  } else if (w > 0) {
    MemP mv = ctx.alloc(std::max<int64_t>(1, n) * w);
    c->values = mv->ptr;
    c->owners.push_back(mv);
  }
  if (with_validity) {
    MemP mvb;
    c->validity = ctx.alloc_t<uint8_t>((size_t)(n + 7) / 8 + 8, mvb);
    c->owners.push_back(mvb);
  }
  return c;
}

ColP make_utf8_column(Ctx& ctx, const std::string& name, int64_t n, int64_t bytes, bool with_validity) {
  auto c = std::make_shared<Column>();
  c->type = TY_UTF8;
  c->name = name;
  c->length = n;
  MemP mo, md;
  c->offsets = ctx.alloc_t<int32_t>((size_t)n + 1, mo);
  c->data = ctx.alloc_t<uint8_t>((size_t)std::max<int64_t>(bytes, 1), md);
  c->data_bytes = bytes;
  c->owners = {mo, md};
  if (with_validity) {
    MemP mvb;
    c->validity = ctx.alloc_t<uint8_t>((size_t)(n + 7) / 8 + 8, mvb);
    c->owners.push_back(mvb);
  }
  return c;
}

}  // namespace prism
