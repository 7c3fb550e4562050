// runtime.hpp — host runtime of the engine: context, budgeted device
// allocator, device columns/batches, and status plumbing behind the C ABI.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <map>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/prism_gpu.h"
#include "common.cuh"

namespace prism {

// ------------------------------------------------------------- failures ----
struct Failure {
  int code;
  std::string msg;
};
[[noreturn]] inline void fail(int code, std::string msg) { throw Failure{code, std::move(msg)}; }

#define PRISM_CUDA(expr)                                                              \
  do {                                                                                \
    cudaError_t _e = (expr);                                                          \
    if (_e != cudaSuccess) {                                                          \
      if (_e == cudaErrorMemoryAllocation)                                            \
        ::prism::fail(PRISM_ERR_NO_MEMORY, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
      ::prism::fail(PRISM_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
    }                                                                                 \
  } while (0)

struct Ctx;

// A device allocation owned through shared_ptr; freed stream-ordered.
struct DevMem {
  Ctx* ctx = nullptr;
  void* ptr = nullptr;
  size_t bytes = 0;
  bool borrowed = false;  // caller-owned memory (zero-copy import)
  ~DevMem();
};
using MemP = std::shared_ptr<DevMem>;

struct Column {
  int32_t type = TY_NULL;
  int32_t index_type = TY_I32;  // TY_DICT
  std::string name;
  bool nullable = true;
  int64_t length = 0;
  int32_t precision = 38, scale = 0;
  // device pointers (see DCol)
  uint8_t* validity = nullptr;
  void* values = nullptr;
  int32_t* offsets = nullptr;
  uint8_t* data = nullptr;
  int32_t data_base = 0;    // offsets[0] (UTF8): bytes before it are not resident
  int64_t data_bytes = 0;   // resident UTF8 bytes (offsets[n] - offsets[0])
  std::shared_ptr<Column> dict;  // TY_DICT values
  uint64_t dict_fingerprint = 0;
  std::vector<MemP> owners;

  DCol view() const;
};
using ColP = std::shared_ptr<Column>;

struct Batch {
  std::vector<ColP> cols;
  int64_t rows = 0;
};

struct Ctx {
  int device = 0;
  cudaStream_t own_stream = nullptr;
  cudaStream_t stream = nullptr;
  cudaMemPool_t pool = nullptr;
  uint64_t budget = 0;
  std::atomic<uint64_t> in_use{0};
  std::atomic<uint64_t> launches{0};
  std::recursive_mutex mu;
  std::string last_error;
  int sm_count = 148;
  int64_t l2_bytes = 126LL << 20;  // the device's L2 size
  uint32_t* d_err = nullptr;  // device error flags (one word; bytes 8-15: a call's match counter)
  uint32_t* h_err = nullptr;  // pinned mirror (128 bytes; bytes 64-127: small readbacks of a call)
  // page-locked ring for small host -> device copies whose host source may
  // go away at once (program uploads): the bytes are copied into the ring and
  // the device copy is queued without waiting for the stream; a wrap of the
  // ring waits for the last copy queued (all of them are on this stream: a
  // stream change synchronises the old one)
  uint8_t* h_stage = nullptr;
  size_t stage_cap = 0, stage_head = 0;
  cudaEvent_t stage_ev = nullptr;
  bool stage_pending = false;
  void h2d_staged(void* dst, const void* src, size_t bytes);
  // the one-pass probe's steady shape, instantiated once per kernel variant
  // and replayed with new arguments: memset of the match counter -> kernel
  // -> one copy of the error word and the counter to the host
  struct ProbeGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraphNode_t kernel = nullptr;
  };
  std::map<const void*, ProbeGraph> probe_graphs;
  // per-kernel CUDA-event timing (off unless enabled)
  bool profiling = false;
  std::map<std::string, std::vector<std::pair<cudaEvent_t, cudaEvent_t>>> timings;
  std::vector<cudaEvent_t> event_pool;
  cudaEvent_t take_event();
  void clear_timings();

  MemP alloc(size_t bytes);
  template <class T>
  T* alloc_t(size_t n, MemP& hold) {
    hold = alloc(n * sizeof(T));
    return static_cast<T*>(hold->ptr);
  }
  void note_launch(uint64_t n = 1) { launches.fetch_add(n, std::memory_order_relaxed); }
  void check_launch(const char* what);
  // Reads and clears the device error word (synchronises the stream).
  uint32_t take_device_errors();
  void sync();
};

// Brackets one kernel launch with CUDA events when profiling is on.
struct KernelTimer {
  Ctx& ctx;
  const char* name;
  cudaEvent_t start = nullptr;
  KernelTimer(Ctx& c, const char* n) : ctx(c), name(n) {
    if (ctx.profiling) {
      start = ctx.take_event();
      cudaEventRecord(start, ctx.stream);
    }
  }
  ~KernelTimer() {
    if (start) {
      cudaEvent_t stop = ctx.take_event();
      cudaEventRecord(stop, ctx.stream);
      ctx.timings[name].push_back({start, stop});
    }
  }
};

// Ceil-pow2 helper
inline uint64_t next_pow2(uint64_t x) {
  uint64_t p = 1;
  while (p < x) p <<= 1;
  return p;
}

inline int grid_for(const Ctx& c, int64_t n, int block, int per_sm = 8) {
  int64_t g = (n + block - 1) / block;
  int64_t cap = (int64_t)c.sm_count * per_sm;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

// Column helpers
ColP make_column(Ctx& ctx, int32_t type, const std::string& name, int64_t n, bool with_validity);
ColP make_utf8_column(Ctx& ctx, const std::string& name, int64_t n, int64_t bytes, bool with_validity);

}  // namespace prism

// The opaque handles of the C ABI.
struct prism_ctx {
  prism::Ctx impl;
};
struct prism_batch {
  prism::Batch impl;
  prism_ctx* ctx = nullptr;
};
