// arrow_io.cu — Arrow C Data Interface import (host or device buffers) into
// device columns, and export of device columns back to host Arrow arrays.
#include <algorithm>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>

#include "arrow_io.hpp"

namespace prism {

namespace {

bool parse_format(const char* f, int32_t& t, int32_t& prec, int32_t& scale) {
  std::string s(f ? f : "");
  if (s == "n") t = TY_NULL;
  else if (s == "b") t = TY_BOOL;
  else if (s == "c") t = TY_I8;
  else if (s == "C") t = TY_U8;
  else if (s == "s") t = TY_I16;
  else if (s == "S") t = TY_U16;
  else if (s == "i") t = TY_I32;
  else if (s == "I") t = TY_U32;
  else if (s == "l") t = TY_I64;
  else if (s == "L") t = TY_U64;
  else if (s == "f") t = TY_F32;
  else if (s == "g") t = TY_F64;
  else if (s == "tdD") t = TY_DATE32;
  else if (s == "u") t = TY_UTF8;
  else if (s.rfind("d:", 0) == 0) {
    int p = 0, sc = 0, bw = 128;
    int k = sscanf(s.c_str() + 2, "%d,%d,%d", &p, &sc, &bw);
    if (k < 2 || bw != 128) return false;
    t = TY_DEC128;
    prec = p;
    scale = sc;
  } else return false;
  return true;
}

// out byte j = bits [off + 8j, off + 8j + 8) of in
__global__ void realign_bits_kernel(const uint8_t* __restrict__ in, int64_t off, int64_t nbytes,
                                    uint8_t* __restrict__ out) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < nbytes;
       j += (int64_t)gridDim.x * blockDim.x) {
    int64_t bit = off + 8 * j;
    int64_t b = bit >> 3;
    int sh = (int)(bit & 7);
    uint32_t lo = in[b];
    uint32_t hi = in[b + 1];
    out[j] = (uint8_t)(((hi << 8) | lo) >> sh);
  }
}

uint64_t fnv1a(const uint8_t* p, size_t n, uint64_t h = 1469598103934665603ULL) {
  for (size_t i = 0; i < n; ++i) {
    h ^= p[i];
    h *= 1099511628211ULL;
  }
  return h;
}

bool is_device_ptr(const void* p) {
  if (!p) return false;
  cudaPointerAttributes at;
  cudaError_t e = cudaPointerGetAttributes(&at, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

// ---------------------------------------------------------------- import --
// Host memcpy workers shared by every import: a pageable source is copied
// into page-locked staging by several threads at once (one thread moves
// ~10 GB/s; the link takes ~55 GB/s from pinned memory, ~11 GB/s when the
// driver stages pageable memory itself).
class CopyPool {
 public:
  static constexpr int kThreads = 8;
  CopyPool() {
    for (int i = 0; i < kThreads; ++i) th_.emplace_back([this] { run(); });
  }
  // copies n bytes, split over the workers and the calling thread
  void copy(void* dst, const void* src, size_t n) {
    const size_t piece = std::max<size_t>((size_t)1 << 20, (n + kThreads) / (kThreads + 1));
    size_t off = piece < n ? piece : n;  // the caller's own share: [0, off)
    {
      std::lock_guard<std::mutex> lk(mu_);
      for (size_t o = off; o < n; o += piece) {
        q_.push_back({static_cast<uint8_t*>(dst) + o, static_cast<const uint8_t*>(src) + o, std::min(piece, n - o)});
        ++pending_;
      }
    }
    cv_.notify_all();
    std::memcpy(dst, src, off);
    std::unique_lock<std::mutex> lk(mu_);
    done_.wait(lk, [this] { return pending_ == 0; });
  }

 private:
  struct Task {
    uint8_t* dst;
    const uint8_t* src;
    size_t n;
  };
  void run() {
    for (;;) {
      Task t;
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [this] { return !q_.empty(); });
        t = q_.front();
        q_.pop_front();
      }
      std::memcpy(t.dst, t.src, t.n);
      std::lock_guard<std::mutex> lk(mu_);
      if (--pending_ == 0) done_.notify_all();
    }
  }
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_, done_;
  std::deque<Task> q_;
  size_t pending_ = 0;
};

// never destroyed (workers block on the queue until exit)
CopyPool& copy_pool() {
  static CopyPool* p = new CopyPool();
  return *p;
}

// Pageable host -> device through SLOTS page-locked chunks: a chunk is
// refilled (by the copy pool) once its previous transfer has finished, so the
// host copy of one chunk overlaps the transfer of the others.
class Staging {
 public:
  static constexpr size_t kChunk = (size_t)32 << 20;
  static constexpr int kSlots = 4;
  explicit Staging(Ctx& c) : ctx_(c) {}
  ~Staging() {
    for (int k = 0; k < kSlots; ++k) {
      if (used_[k]) cudaEventSynchronize(ev_[k]);
      if (ev_[k]) cudaEventDestroy(ev_[k]);
      if (buf_[k]) pinned_put(buf_[k], size_[k]);
    }
  }
  // false when no page-locked memory could be had (the caller copies directly)
  bool copy(void* dst, const void* src, size_t bytes) {
    while (bytes) {
      const size_t piece = std::min(bytes, kChunk);
      const int k = next_;
      next_ = (next_ + 1) % kSlots;
      if (!buf_[k]) {
        buf_[k] = pinned_get(kChunk, &size_[k]);
        if (!buf_[k]) return fallback(dst, src, bytes);
        PRISM_CUDA(cudaEventCreateWithFlags(&ev_[k], cudaEventDisableTiming));
      }
      if (used_[k]) PRISM_CUDA(cudaEventSynchronize(ev_[k]));
      copy_pool().copy(buf_[k], src, piece);
      PRISM_CUDA(cudaMemcpyAsync(dst, buf_[k], piece, cudaMemcpyHostToDevice, ctx_.stream));
      PRISM_CUDA(cudaEventRecord(ev_[k], ctx_.stream));
      used_[k] = true;
      dst = static_cast<uint8_t*>(dst) + piece;
      src = static_cast<const uint8_t*>(src) + piece;
      bytes -= piece;
    }
    return true;
  }

 private:
  bool fallback(void* dst, const void* src, size_t bytes) {
    PRISM_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx_.stream));
    return true;
  }
  Ctx& ctx_;
  void* buf_[kSlots] = {};
  size_t size_[kSlots] = {};
  cudaEvent_t ev_[kSlots] = {};
  bool used_[kSlots] = {};
  int next_ = 0;
};

bool is_pageable(const void* p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();
    return true;
  }
  return at.type == cudaMemoryTypeUnregistered;
}

struct Importer {
  Ctx& ctx;
  bool device;  // buffers are device pointers
  std::unique_ptr<Staging> staging;  // pageable sources of at least kStageMin bytes
  static constexpr size_t kStageMin = (size_t)1 << 20;

  void copy_in(void* dst, const void* src, size_t bytes) {
    if (!bytes) return;
    if (!device && bytes >= kStageMin && is_pageable(src)) {
      if (!staging) staging = std::make_unique<Staging>(ctx);
      staging->copy(dst, src, bytes);
      return;
    }
    PRISM_CUDA(cudaMemcpyAsync(dst, src, bytes, device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                               ctx.stream));
  }

  // bitmap of n bits starting at bit `off` of src, realigned to bit 0
  uint8_t* bitmap(const void* src, int64_t off, int64_t n, Column& c) {
    int64_t nbytes = (n + 7) / 8;
    int64_t first = off >> 3;
    if (device && (off & 7) == 0) {
      auto m = std::make_shared<DevMem>();
      m->ctx = &ctx;
      m->ptr = (void*)(static_cast<const uint8_t*>(src) + first);
      m->borrowed = true;
      c.owners.push_back(m);
      return static_cast<uint8_t*>(m->ptr);
    }
    MemP raw;
    uint8_t* d = ctx.alloc_t<uint8_t>((size_t)nbytes + 8, raw);
    if ((off & 7) == 0) {
      copy_in(d, static_cast<const uint8_t*>(src) + first, (size_t)nbytes);
      c.owners.push_back(raw);
      return d;
    }
    // stage the covering bytes, then realign on the device
    int64_t span = ((off + n + 7) >> 3) - first + 1;
    MemP stage;
    uint8_t* s = ctx.alloc_t<uint8_t>((size_t)span + 8, stage);
    PRISM_CUDA(cudaMemsetAsync(s, 0, (size_t)span + 8, ctx.stream));
    copy_in(s, static_cast<const uint8_t*>(src) + first, (size_t)(((off + n + 7) >> 3) - first));
    if (nbytes > 0) {
      realign_bits_kernel<<<grid_for(ctx, nbytes, 256), 256, 0, ctx.stream>>>(s, off & 7, nbytes, d);
      ctx.check_launch("realign_bits_kernel");
    }
    c.owners.push_back(raw);
    c.owners.push_back(stage);
    return d;
  }

  void* values(const void* src, int64_t off, int64_t n, int w, Column& c) {
    if (device) {
      auto m = std::make_shared<DevMem>();
      m->ctx = &ctx;
      m->ptr = (void*)(static_cast<const uint8_t*>(src) + off * w);
      m->borrowed = true;
      c.owners.push_back(m);
      return m->ptr;
    }
    MemP mv = ctx.alloc(std::max<int64_t>(1, n) * w + 16);
    copy_in(mv->ptr, static_cast<const uint8_t*>(src) + off * w, (size_t)(n * w));
    c.owners.push_back(mv);
    return mv->ptr;
  }

  int32_t read_i32(const int32_t* p) {
    if (!device) return *p;
    int32_t v = 0;
    PRISM_CUDA(cudaMemcpyAsync(&v, p, 4, cudaMemcpyDeviceToHost, ctx.stream));
    PRISM_CUDA(cudaStreamSynchronize(ctx.stream));
    return v;
  }

  ColP column(const ArrowArray* a, const ArrowSchema* s, int64_t extra_off, int64_t len) {
    auto c = std::make_shared<Column>();
    c->name = s->name ? s->name : "";
    c->nullable = (s->flags & ARROW_FLAG_NULLABLE) != 0;
    c->length = len;
    int32_t t, prec = 38, scale = 0;
    if (!parse_format(s->format, t, prec, scale))
      fail(PRISM_ERR_ARROW, std::string("unsupported arrow format '") + (s->format ? s->format : "") + "'");
    c->precision = prec;
    c->scale = scale;
    int64_t off = a->offset + extra_off;
    if (s->dictionary) {
      if (t != TY_I8 && t != TY_I16 && t != TY_I32 && t != TY_I64 && t != TY_U8 && t != TY_U16 && t != TY_U32)
        fail(PRISM_ERR_ARROW, "unsupported dictionary index type");
      c->type = TY_DICT;
      c->index_type = t;
      c->dict = column(a->dictionary, s->dictionary, 0, a->dictionary->length);
      if (c->dict->type != TY_UTF8) fail(PRISM_ERR_ARROW, "only Utf8 dictionaries are supported");
      c->dict_fingerprint = fingerprint(a->dictionary, s->dictionary);
    } else {
      c->type = t;
    }
    if (t == TY_NULL) return c;
    if (a->null_count != 0 && a->buffers[0]) c->validity = bitmap(a->buffers[0], off, len, *c);
    if (c->type == TY_UTF8) {
      const int32_t* offs = static_cast<const int32_t*>(a->buffers[1]);
      int32_t lo = read_i32(offs + off), hi = read_i32(offs + off + len);
      c->data_base = lo;
      c->data_bytes = hi - lo;
      if (device) {
        c->offsets = const_cast<int32_t*>(offs + off);
        c->data = const_cast<uint8_t*>(static_cast<const uint8_t*>(a->buffers[2])) + lo;
      } else {
        MemP mo, md;
        c->offsets = ctx.alloc_t<int32_t>((size_t)len + 1, mo);
        copy_in(c->offsets, offs + off, (size_t)(len + 1) * 4);
        c->data = ctx.alloc_t<uint8_t>((size_t)std::max<int64_t>(1, hi - lo) + 8, md);
        copy_in(c->data, static_cast<const uint8_t*>(a->buffers[2]) + lo, (size_t)(hi - lo));
        c->owners.push_back(mo);
        c->owners.push_back(md);
      }
    } else if (c->type == TY_BOOL) {
      c->values = bitmap(a->buffers[1], off, len, *c);
    } else {
      int w = width_of(c->type == TY_DICT ? c->index_type : c->type);
      c->values = values(a->buffers[1], off, len, w, *c);
    }
    return c;
  }

  uint64_t fingerprint(const ArrowArray* d, const ArrowSchema* ds) {
    // content hash of a Utf8 dictionary (identity across batches)
    if (std::string(ds->format) != "u") return 0;
    const int32_t* offs = static_cast<const int32_t*>(d->buffers[1]);
    int64_t n = d->length, o = d->offset;
    if (device) {
      std::vector<int32_t> h((size_t)n + 1);
      PRISM_CUDA(cudaMemcpyAsync(h.data(), offs + o, (n + 1) * 4, cudaMemcpyDeviceToHost, ctx.stream));
      PRISM_CUDA(cudaStreamSynchronize(ctx.stream));
      std::vector<uint8_t> bytes((size_t)(h[n] - h[0]) + 1);
      PRISM_CUDA(cudaMemcpyAsync(bytes.data(), static_cast<const uint8_t*>(d->buffers[2]) + h[0], h[n] - h[0],
                                 cudaMemcpyDeviceToHost, ctx.stream));
      PRISM_CUDA(cudaStreamSynchronize(ctx.stream));
      uint64_t f = fnv1a(reinterpret_cast<const uint8_t*>(h.data()), 0);
      for (int64_t i = 0; i < n; ++i) {
        f = fnv1a(bytes.data() + (h[i] - h[0]), (size_t)(h[i + 1] - h[i]), f);
        f = fnv1a(reinterpret_cast<const uint8_t*>("\xff"), 1, f);
      }
      return f ^ (uint64_t)n;
    }
    const uint8_t* data = static_cast<const uint8_t*>(d->buffers[2]);
    uint64_t f = 1469598103934665603ULL;
    for (int64_t i = 0; i < n; ++i) {
      f = fnv1a(data + offs[o + i], (size_t)(offs[o + i + 1] - offs[o + i]), f);
      f = fnv1a(reinterpret_cast<const uint8_t*>("\xff"), 1, f);
    }
    return f ^ (uint64_t)n;
  }
};

// ------------------------------------------------------------------ export --
// Exported buffers are page-locked host memory from a process-wide pool: a
// device-to-host copy into pinned memory runs asynchronously at the link's
// full rate, where pageable memory is staged through a driver buffer. Pinning
// costs a system call per allocation, so buffers are recycled: an exported
// array returns its buffers to the pool when the consumer releases it. At
// most kPinnedCached bytes stay cached; small buffers use malloc.
class PinnedPool {
 public:
  static constexpr size_t kPinnedCached = (size_t)8 << 30;
  static constexpr size_t kPinnedMin = (size_t)64 << 10;
  // a pinned buffer of at least `bytes` (its size in *size), or nullptr
  void* get(size_t bytes, size_t* size) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      auto it = free_.lower_bound(bytes);
      if (it != free_.end() && it->first <= 2 * bytes) {
        void* p = it->second;
        *size = it->first;
        cached_ -= it->first;
        free_.erase(it);
        return p;
      }
    }
    size_t sz = (bytes + ((size_t)1 << 16) - 1) & ~(((size_t)1 << 16) - 1);
    void* p = nullptr;
    if (cudaHostAlloc(&p, sz, cudaHostAllocPortable) != cudaSuccess) {
      cudaGetLastError();  // not sticky: fall back to pageable memory
      return nullptr;
    }
    *size = sz;
    return p;
  }
  void put(void* p, size_t size) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      if (cached_ + size <= kPinnedCached) {
        free_.emplace(size, p);
        cached_ += size;
        return;
      }
    }
    cudaFreeHost(p);
  }

 private:
  std::mutex mu_;
  std::multimap<size_t, void*> free_;
  size_t cached_ = 0;
};

// never destroyed: exported arrays may be released at any time before exit
PinnedPool& pinned_pool() {
  static PinnedPool* pool = new PinnedPool();
  return *pool;
}

}  // namespace

void* pinned_get(size_t bytes, size_t* size) { return pinned_pool().get(bytes, size); }
void pinned_put(void* p, size_t size) { pinned_pool().put(p, size); }

namespace {

struct HostBuf {
  void* p = nullptr;
  size_t size = 0;
  bool pinned = false;
  ~HostBuf() {
    if (pinned) pinned_pool().put(p, size);
    else free(p);
  }
};
struct SchemaPriv {
  std::string format, name;
  std::vector<ArrowSchema*> children;
  ArrowSchema* dict = nullptr;
};
void release_schema(ArrowSchema* s) {
  if (!s || !s->release) return;
  auto* p = static_cast<SchemaPriv*>(s->private_data);
  for (auto* ch : p->children) {
    if (ch->release) ch->release(ch);
    delete ch;
  }
  if (p->dict) {
    if (p->dict->release) p->dict->release(p->dict);
    delete p->dict;
  }
  delete p;
  s->release = nullptr;
}
struct ArrayPriv {
  std::vector<std::shared_ptr<HostBuf>> bufs;
  std::vector<std::shared_ptr<void>> holds;  // other owners of the buffers (host_batch exports)
  std::vector<const void*> ptrs;
  std::vector<ArrowArray*> children;
  ArrowArray* dict = nullptr;
};
void release_array(ArrowArray* a) {
  if (!a || !a->release) return;
  auto* p = static_cast<ArrayPriv*>(a->private_data);
  for (auto* ch : p->children) {
    if (ch->release) ch->release(ch);
    delete ch;
  }
  if (p->dict) {
    if (p->dict->release) p->dict->release(p->dict);
    delete p->dict;
  }
  delete p;
  a->release = nullptr;
}

std::string format_of(const Column& c) {
  switch (c.type == TY_DICT ? c.index_type : c.type) {
    case TY_NULL: return "n";
    case TY_BOOL: return "b";
    case TY_I8: return "c";
    case TY_U8: return "C";
    case TY_I16: return "s";
    case TY_U16: return "S";
    case TY_I32: return "i";
    case TY_U32: return "I";
    case TY_I64: return "l";
    case TY_U64: return "L";
    case TY_F32: return "f";
    case TY_F64: return "g";
    case TY_DATE32: return "tdD";
    case TY_UTF8: return "u";
    case TY_DEC128: return "d:" + std::to_string(c.precision) + "," + std::to_string(c.scale);
  }
  return "n";
}

void export_schema_col(const Column& c, ArrowSchema* s) {
  auto* p = new SchemaPriv();
  p->format = format_of(c);
  p->name = c.name;
  *s = ArrowSchema{};
  s->format = p->format.c_str();
  s->name = p->name.c_str();
  s->flags = c.nullable ? ARROW_FLAG_NULLABLE : 0;
  if (c.type == TY_DICT) {
    p->dict = new ArrowSchema();
    export_schema_col(*c.dict, p->dict);
    s->dictionary = p->dict;
  }
  s->release = release_schema;
  s->private_data = p;
}

struct Exporter {
  Ctx& ctx;
  std::vector<std::pair<ArrowArray*, int64_t>> rebase;  // utf8 offsets to rebase after sync
  std::vector<std::pair<int32_t*, std::pair<int64_t, int32_t>>> rebase_offs;

  std::shared_ptr<HostBuf> host(size_t bytes) {
    auto h = std::make_shared<HostBuf>();
    if (bytes + 16 >= PinnedPool::kPinnedMin) {
      h->p = pinned_pool().get(bytes + 16, &h->size);
      h->pinned = h->p != nullptr;
    }
    if (!h->p) h->p = malloc(bytes + 16);
    if (!h->p) fail(PRISM_ERR_NO_MEMORY, "host allocation failed");
    return h;
  }
  void d2h(void* dst, const void* src, size_t bytes) {
    if (bytes) PRISM_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx.stream));
  }

  void array_col(const Column& c, ArrowArray* a) {
    auto* p = new ArrayPriv();
    *a = ArrowArray{};
    a->length = c.length;
    int64_t n = c.length;
    if (c.type == TY_NULL) {
      a->null_count = n;
      a->n_buffers = 0;
    } else {
      std::shared_ptr<HostBuf> vb;
      if (c.validity) {
        vb = host((size_t)(n + 7) / 8);
        d2h(vb->p, c.validity, (size_t)(n + 7) / 8);
        a->null_count = -1;
      } else {
        a->null_count = 0;
      }
      p->ptrs.push_back(vb ? vb->p : nullptr);
      if (vb) p->bufs.push_back(vb);
      if (c.type == TY_UTF8) {
        auto ob = host((size_t)(n + 1) * 4);
        auto db = host((size_t)c.data_bytes);
        if (c.offsets) {
          d2h(ob->p, c.offsets, (size_t)(n + 1) * 4);
        } else {  // an empty result column built without buffers
          if (n) fail(PRISM_ERR_INTERNAL, "Utf8 column without offsets");
          std::memset(ob->p, 0, 4);
        }
        d2h(db->p, c.data, (size_t)c.data_bytes);
        rebase_offs.push_back({static_cast<int32_t*>(ob->p), {n, c.data_base}});
        p->bufs.push_back(ob);
        p->bufs.push_back(db);
        p->ptrs.push_back(ob->p);
        p->ptrs.push_back(db->p);
      } else if (c.type == TY_BOOL) {
        auto bb = host((size_t)(n + 7) / 8);
        d2h(bb->p, c.values, (size_t)(n + 7) / 8);
        p->bufs.push_back(bb);
        p->ptrs.push_back(bb->p);
      } else {
        int w = width_of(c.type == TY_DICT ? c.index_type : c.type);
        auto bb = host((size_t)(n * w));
        d2h(bb->p, c.values, (size_t)(n * w));
        p->bufs.push_back(bb);
        p->ptrs.push_back(bb->p);
      }
      a->n_buffers = (int64_t)p->ptrs.size();
      a->buffers = p->ptrs.data();
    }
    if (c.type == TY_DICT) {
      p->dict = new ArrowArray();
      array_col(*c.dict, p->dict);
      a->dictionary = p->dict;
    }
    a->release = release_array;
    a->private_data = p;
  }

  void finish() {
    PRISM_CUDA(cudaStreamSynchronize(ctx.stream));
    for (auto& r : rebase_offs) {
      int32_t* o = r.first;
      int64_t n = r.second.first;
      int32_t base = r.second.second;
      if (base)
        for (int64_t i = 0; i <= n; ++i) o[i] -= base;
    }
  }
};

}  // namespace

Batch import_batch(Ctx& ctx, const ArrowArray* a, const ArrowSchema* s, bool device_buffers) {
  if (!a || !s) fail(PRISM_ERR_INVALID_ARGUMENT, "null ArrowArray/ArrowSchema");
  if (!s->format || std::string(s->format) != "+s")
    fail(PRISM_ERR_ARROW, "a RecordBatch must be exported as a struct array (format '+s')");
  if (a->n_children != s->n_children) fail(PRISM_ERR_ARROW, "array/schema child count mismatch");
  Importer im{ctx, device_buffers};
  Batch b;
  b.rows = a->length;
  for (int64_t i = 0; i < s->n_children; ++i)
    b.cols.push_back(im.column(a->children[i], s->children[i], a->offset, a->length));
  return b;
}

Batch import_device_batch(Ctx& ctx, const ArrowDeviceArray* a, const ArrowSchema* s) {
  if (!a) fail(PRISM_ERR_INVALID_ARGUMENT, "null ArrowDeviceArray");
  bool dev = a->device_type == ARROW_DEVICE_CUDA || a->device_type == ARROW_DEVICE_CUDA_MANAGED;
  if (dev && a->device_id != ctx.device)
    fail(PRISM_ERR_INVALID_ARGUMENT, "device array lives on another device");
  if (dev && a->sync_event) PRISM_CUDA(cudaStreamWaitEvent(ctx.stream, *static_cast<cudaEvent_t*>(a->sync_event), 0));
  return import_batch(ctx, &a->array, s, dev);
}


// ------------------------------------------------------- host-side batches --
namespace {

// bits [off, off + n) of `in`, realigned to bit 0
std::vector<uint8_t> realign_bits_host(const uint8_t* in, int64_t off, int64_t n) {
  const int64_t nbytes = (n + 7) / 8;
  std::vector<uint8_t> out((size_t)nbytes + 1, 0);
  const int sh = (int)(off & 7);
  const uint8_t* b = in + (off >> 3);
  const int64_t src_bytes = ((off & 7) + n + 7) / 8;  // bytes of `in` that hold the bits
  for (int64_t j = 0; j < nbytes; ++j) {
    const uint32_t lo = b[j];
    const uint32_t hi = j + 1 < src_bytes ? b[j + 1] : 0u;
    out[(size_t)j] = (uint8_t)(((hi << 8) | lo) >> sh);
  }
  return out;
}

ColP host_column(const ArrowArray* a, const ArrowSchema* s, int64_t extra_off, int64_t len,
                 std::vector<std::shared_ptr<std::vector<uint8_t>>>& keep) {
  auto c = std::make_shared<Column>();
  c->name = s->name ? s->name : "";
  c->nullable = (s->flags & ARROW_FLAG_NULLABLE) != 0;
  c->length = len;
  int32_t t, prec = 38, scale = 0;
  if (!parse_format(s->format, t, prec, scale))
    fail(PRISM_ERR_ARROW, std::string("unsupported arrow format '") + (s->format ? s->format : "") + "'");
  c->precision = prec;
  c->scale = scale;
  const int64_t off = a->offset + extra_off;
  if (s->dictionary) {
    c->type = TY_DICT;
    c->index_type = t;
    c->dict = host_column(a->dictionary, s->dictionary, 0, a->dictionary->length, keep);
    if (c->dict->type != TY_UTF8) fail(PRISM_ERR_ARROW, "only Utf8 dictionaries are supported");
  } else {
    c->type = t;
  }
  if (t == TY_NULL) return c;
  auto bits = [&](const void* src) -> uint8_t* {
    const uint8_t* b = static_cast<const uint8_t*>(src);
    if ((off & 7) == 0) return const_cast<uint8_t*>(b + (off >> 3));
    keep.push_back(std::make_shared<std::vector<uint8_t>>(realign_bits_host(b, off, len)));
    return keep.back()->data();
  };
  if (a->null_count != 0 && a->buffers[0]) c->validity = bits(a->buffers[0]);
  if (c->type == TY_UTF8) {
    const int32_t* offs = static_cast<const int32_t*>(a->buffers[1]);
    c->offsets = const_cast<int32_t*>(offs + off);
    c->data_base = offs[off];
    c->data_bytes = offs[off + len] - offs[off];
    c->data = const_cast<uint8_t*>(static_cast<const uint8_t*>(a->buffers[2])) + c->data_base;
  } else if (c->type == TY_BOOL) {
    c->values = bits(a->buffers[1]);
  } else {
    const int w = width_of(c->type == TY_DICT ? c->index_type : c->type);
    c->values = const_cast<uint8_t*>(static_cast<const uint8_t*>(a->buffers[1]) + off * w);
  }
  return c;
}

void host_array_col(const Column& c, ArrowArray* a, const std::shared_ptr<void>& hold) {
  auto* p = new ArrayPriv();
  p->holds.push_back(hold);
  *a = ArrowArray{};
  a->length = c.length;
  const int64_t n = c.length;
  if (c.type == TY_NULL) {
    a->null_count = n;
    a->n_buffers = 0;
  } else {
    a->null_count = c.validity ? -1 : 0;
    p->ptrs.push_back(c.validity);
    if (c.type == TY_UTF8) {
      // offsets rebased to the column's first byte
      auto o = std::make_shared<std::vector<int32_t>>((size_t)n + 1, 0);
      if (c.offsets)
        for (int64_t i = 0; i <= n; ++i) (*o)[(size_t)i] = c.offsets[i] - c.data_base;
      p->holds.push_back(o);
      p->ptrs.push_back(o->data());
      p->ptrs.push_back(c.data ? c.data : reinterpret_cast<uint8_t*>(o->data()));
    } else {
      p->ptrs.push_back(c.values);
    }
    a->n_buffers = (int64_t)p->ptrs.size();
    a->buffers = p->ptrs.data();
  }
  if (c.type == TY_DICT) {
    p->dict = new ArrowArray();
    host_array_col(*c.dict, p->dict, hold);
    a->dictionary = p->dict;
  }
  a->release = release_array;
  a->private_data = p;
}

}  // namespace

Batch host_batch(const ArrowArray* a, const ArrowSchema* s, std::vector<std::shared_ptr<std::vector<uint8_t>>>& keep) {
  if (!a || !s) fail(PRISM_ERR_INVALID_ARGUMENT, "null ArrowArray/ArrowSchema");
  if (!s->format || std::string(s->format) != "+s")
    fail(PRISM_ERR_ARROW, "a RecordBatch must be exported as a struct array (format '+s')");
  if (a->n_children != s->n_children) fail(PRISM_ERR_ARROW, "array/schema child count mismatch");
  Batch b;
  b.rows = a->length;
  for (int64_t i = 0; i < s->n_children; ++i) b.cols.push_back(host_column(a->children[i], s->children[i], a->offset, a->length, keep));
  return b;
}

void export_host_batch(const Batch& b, const std::shared_ptr<void>& hold, ArrowArray* a, ArrowSchema* s) {
  if (!a || !s) fail(PRISM_ERR_INVALID_ARGUMENT, "null output ArrowArray/ArrowSchema");
  auto* ap = new ArrayPriv();
  ap->ptrs = {nullptr};
  auto* sp = new SchemaPriv();
  sp->format = "+s";
  for (auto& c : b.cols) {
    auto* ca = new ArrowArray();
    host_array_col(*c, ca, hold);
    ap->children.push_back(ca);
    auto* cs = new ArrowSchema();
    export_schema_col(*c, cs);
    sp->children.push_back(cs);
  }
  *s = ArrowSchema{};
  s->format = sp->format.c_str();
  s->name = sp->name.c_str();
  s->n_children = (int64_t)sp->children.size();
  s->children = sp->children.data();
  s->release = release_schema;
  s->private_data = sp;
  *a = ArrowArray{};
  a->length = b.rows;
  a->n_buffers = 1;
  a->buffers = ap->ptrs.data();
  a->n_children = (int64_t)ap->children.size();
  a->children = ap->children.data();
  a->release = release_array;
  a->private_data = ap;
}

bool arrow_format_type(const char* format, int32_t& type, int32_t& precision, int32_t& scale) {
  return parse_format(format, type, precision, scale);
}

std::vector<HostView> host_view(const ArrowArray* a, const ArrowSchema* s) {
  if (!a || !s) fail(PRISM_ERR_INVALID_ARGUMENT, "null ArrowArray/ArrowSchema");
  if (!s->format || std::string(s->format) != "+s")
    fail(PRISM_ERR_ARROW, "a RecordBatch must be exported as a struct array (format '+s')");
  if (a->n_children != s->n_children) fail(PRISM_ERR_ARROW, "array/schema child count mismatch");
  std::vector<HostView> v;
  for (int64_t i = 0; i < s->n_children; ++i) {
    const ArrowArray* ca = a->children[i];
    const ArrowSchema* cs = s->children[i];
    HostView h;
    h.meta = std::make_shared<Column>();
    Column& c = *h.meta;
    c.name = cs->name ? cs->name : "";
    c.nullable = (cs->flags & ARROW_FLAG_NULLABLE) != 0;
    c.length = a->length;
    int32_t t, prec = 38, scale = 0;
    if (!parse_format(cs->format, t, prec, scale))
      fail(PRISM_ERR_ARROW, std::string("unsupported arrow format '") + (cs->format ? cs->format : "") + "'");
    c.type = cs->dictionary ? TY_DICT : t;
    c.precision = prec;
    c.scale = scale;
    h.null_count = ca->null_count;
    const int w = width_of(t);
    if (!cs->dictionary && t != TY_UTF8 && t != TY_BOOL && t != TY_NULL && w > 0 && ca->n_buffers >= 2 && ca->buffers[1])
      h.values = static_cast<const uint8_t*>(ca->buffers[1]) + (ca->offset + a->offset) * w;
    v.push_back(h);
  }
  return v;
}

HostOutCol host_out_column(ColP meta, size_t bytes) {
  auto h = std::make_shared<HostBuf>();
  if (bytes + 16 >= PinnedPool::kPinnedMin) {
    h->p = pinned_pool().get(bytes + 16, &h->size);
    h->pinned = h->p != nullptr;
  }
  if (!h->p) h->p = malloc(bytes + 16);
  if (!h->p) fail(PRISM_ERR_NO_MEMORY, "host allocation failed");
  HostOutCol c;
  c.meta = std::move(meta);
  c.values = h->p;
  c.hold = h;
  return c;
}

void export_host_columns(const std::vector<HostOutCol>& cols, int64_t rows, ArrowArray* a, ArrowSchema* s) {
  if (!a || !s) fail(PRISM_ERR_INVALID_ARGUMENT, "null output ArrowArray/ArrowSchema");
  auto* ap = new ArrayPriv();
  ap->ptrs = {nullptr};
  auto* sp = new SchemaPriv();
  sp->format = "+s";
  for (auto& c : cols) {
    auto* p = new ArrayPriv();
    auto* ca = new ArrowArray();
    *ca = ArrowArray{};
    ca->length = rows;
    ca->null_count = 0;
    p->bufs.push_back(std::static_pointer_cast<HostBuf>(c.hold));
    p->ptrs = {nullptr, c.values};
    ca->n_buffers = 2;
    ca->buffers = p->ptrs.data();
    ca->release = release_array;
    ca->private_data = p;
    ap->children.push_back(ca);
    auto* cs = new ArrowSchema();
    export_schema_col(*c.meta, cs);
    sp->children.push_back(cs);
  }
  *s = ArrowSchema{};
  s->format = sp->format.c_str();
  s->name = sp->name.c_str();
  s->n_children = (int64_t)sp->children.size();
  s->children = sp->children.data();
  s->release = release_schema;
  s->private_data = sp;
  *a = ArrowArray{};
  a->length = rows;
  a->n_buffers = 1;
  a->buffers = ap->ptrs.data();
  a->n_children = (int64_t)ap->children.size();
  a->children = ap->children.data();
  a->release = release_array;
  a->private_data = ap;
}

void export_batch(Ctx& ctx, const Batch& b, ArrowArray* a, ArrowSchema* s) {
  if (!a || !s) fail(PRISM_ERR_INVALID_ARGUMENT, "null output ArrowArray/ArrowSchema");
  for (auto& c : b.cols)
    if (c->length != b.rows) fail(PRISM_ERR_INTERNAL, "column length mismatch on export");
  Exporter ex{ctx};
  auto* ap = new ArrayPriv();
  ap->ptrs = {nullptr};
  for (auto& c : b.cols) {
    auto* ca = new ArrowArray();
    ex.array_col(*c, ca);
    ap->children.push_back(ca);
  }
  try {
    ex.finish();
  } catch (...) {
    for (auto* ch : ap->children) { release_array(ch); delete ch; }
    delete ap;
    throw;
  }
  auto* sp = new SchemaPriv();
  sp->format = "+s";
  for (auto& c : b.cols) {
    auto* cs = new ArrowSchema();
    export_schema_col(*c, cs);
    sp->children.push_back(cs);
  }
  *s = ArrowSchema{};
  s->format = sp->format.c_str();
  s->name = sp->name.c_str();
  s->n_children = (int64_t)sp->children.size();
  s->children = sp->children.data();
  s->release = release_schema;
  s->private_data = sp;

  *a = ArrowArray{};
  a->length = b.rows;
  a->n_buffers = 1;
  a->buffers = ap->ptrs.data();
  a->n_children = (int64_t)ap->children.size();
  a->children = ap->children.data();
  a->release = release_array;
  a->private_data = ap;
}

}  // namespace prism
