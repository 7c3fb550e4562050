// queue.cu — the device work queue and its persistent probe kernel (see
// queue.hpp).
#include <algorithm>
#include <condition_variable>
#include <cstring>

#include "join_device.cuh"
#include "queue.hpp"

namespace prism {

// one probe request (device ring; written by host-to-device copies)
struct QItem {
  const int64_t* keys;
  uint32_t* out_prow;
  void* out_pay;
  int64_t rows;
  uint64_t tile_begin;  // first tile of the request in the global tile sequence
  uint64_t n_tiles;
  int32_t table;
  int32_t pad;
  uint64_t ready;       // seq + 1: this descriptor belongs to request seq
};
static_assert(sizeof(QItem) == 64, "descriptor layout");

struct QCtl {
  unsigned long long published;  // tiles published (host copies, after the descriptors)
  unsigned long long next_tile;  // tiles claimed (device atomics)
  unsigned int stop;             // the kernel exits at its next idle check
  unsigned int abort;            // a wait ran out: every CTA exits
};

struct QSlot {  // per ring slot, device
  unsigned long long matches;   // output rows reserved so far (final once every tile is done)
  unsigned int tiles_done;
  unsigned int pad;
};

struct QDone {  // per ring slot, page-locked host memory written by the device
  unsigned long long seq1;      // seq + 1 once the request is complete
  unsigned long long matches;
};

struct QStatus {  // page-locked host memory written by the device
  unsigned int err;
  unsigned int pad;
  unsigned long long err_seq;
};

struct QTable {
  const uint32_t* dense;  // dense mode: build row per key - dmin
  int64_t dmin;
  uint64_t drange;
  const ulonglong2* slots;  // hash mode
  uint64_t mask;
  uint64_t cap;
  const void* payload;
  int32_t shift;
  int32_t width;  // payload bytes: 4 or 8
};

namespace {

constexpr int QB = 256;           // threads per CTA
constexpr int QV = 4;             // 16-byte key loads per thread (2 rows each)
constexpr int64_t QT = QB * QV * 2;  // probe rows per tile (2048)
constexpr unsigned long long NONE = ~0ULL;

__device__ __forceinline__ uint32_t q_scan32(uint32_t x) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
    if (lane >= d) x += y;
  }
  return x;
}

// The persistent kernel: CTAs claim tiles in order until the queue stays
// empty for `idle_limit` checks (or stop / abort is set).
__global__ void __launch_bounds__(QB, 4) queue_probe_kernel(QCtl* ctl, const QItem* ring, QSlot* qslots,
                                                            QDone* done, QStatus* status, const QTable* tables,
                                                            unsigned long long first_seq, uint32_t idle_limit,
                                                            uint32_t wait_limit) {
  __shared__ unsigned long long s_tile;
  __shared__ unsigned long long s_seq;
  __shared__ QItem s_item;
  __shared__ uint32_t seg[QV * (QB / 32)];
  __shared__ unsigned long long s_off;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  unsigned long long seq = first_seq;  // thread 0's cursor: the request holding its last tile
  for (;;) {
    if (threadIdx.x == 0) {
      unsigned long long g = NONE;
      uint32_t idle = 0;
      for (;;) {
        if (*(volatile unsigned int*)&ctl->abort) break;
        const unsigned long long pub = *(volatile unsigned long long*)&ctl->published;
        const unsigned long long c = *(volatile unsigned long long*)&ctl->next_tile;
        if (c < pub) {
          if (atomicCAS(&ctl->next_tile, c, c + 1) == c) {
            g = c;
            break;
          }
          continue;
        }
        if (*(volatile unsigned int*)&ctl->stop || ++idle > idle_limit) break;
        __nanosleep(idle < 32 ? 200 : 2000);
      }
      if (g != NONE) {
        // requests cover consecutive tile ranges in sequence order
        uint32_t spins = 0;
        for (;;) {
          const QItem* it = &ring[seq % DeviceQueue::kRing];
          const unsigned long long ready = *(volatile const unsigned long long*)&it->ready;
          if (ready > seq + 1) {  // finished and its slot reused: not the one
            ++seq;
            continue;
          }
          if (ready < seq + 1) {  // its descriptor is not there: bounded wait
            if (++spins > wait_limit) {
              atomicOr(&status->err, (unsigned int)DERR_TIMEOUT);
              status->err_seq = seq;
              __threadfence_system();
              atomicExch(&ctl->abort, 1u);
              g = NONE;
              break;
            }
            __nanosleep(1000);
            continue;
          }
          __threadfence();
          const volatile QItem* v = it;
          const unsigned long long tb = v->tile_begin, nt = v->n_tiles;
          if (g >= tb + nt) {
            ++seq;
            continue;
          }
          s_item.keys = v->keys;
          s_item.out_prow = v->out_prow;
          s_item.out_pay = v->out_pay;
          s_item.rows = v->rows;
          s_item.tile_begin = tb;
          s_item.n_tiles = nt;
          s_item.table = v->table;
          break;
        }
      }
      s_tile = g;
      s_seq = seq;
    }
    __syncthreads();
    const unsigned long long g = s_tile;
    if (g == NONE) break;
    const unsigned long long rseq = s_seq;
    const int slot = (int)(rseq % DeviceQueue::kRing);
    const QTable tb = tables[s_item.table];
    const int64_t n = s_item.rows;
    const int64_t base = (int64_t)(g - s_item.tile_begin) * QT;
    const int64_t* keys = s_item.keys;
    const bool vec = (reinterpret_cast<uintptr_t>(keys) & 15) == 0;
    uint64_t key[QV][2];
#pragma unroll
    for (int v = 0; v < QV; ++v) {
      const int64_t q = base + 2 * (v * QB + threadIdx.x);
      if (vec && q + 1 < n) {
        const longlong2 kv = __ldcs(reinterpret_cast<const longlong2*>(keys + q));
        key[v][0] = (uint64_t)kv.x;
        key[v][1] = (uint64_t)kv.y;
      } else {
        key[v][0] = q < n ? (uint64_t)__ldcs(keys + q) : 0;
        key[v][1] = q + 1 < n ? (uint64_t)__ldcs(keys + q + 1) : 0;
      }
    }
    uint32_t brow[QV][2];
    if (tb.dense) {
#pragma unroll
      for (int v = 0; v < QV; ++v)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int64_t q = base + 2 * (v * QB + threadIdx.x) + j;
          const uint64_t d = key[v][j] - (uint64_t)tb.dmin;
          brow[v][j] = (q < n && d < tb.drange) ? __ldg(tb.dense + d) : JOIN_NO_MATCH;
        }
    } else {
      uint64_t s[QV][2];
      ulonglong2 e[QV][2];
#pragma unroll
      for (int v = 0; v < QV; ++v)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int64_t q = base + 2 * (v * QB + threadIdx.x) + j;
          s[v][j] = key[v][j] == JOIN_EMPTY ? tb.cap : join_slot_of(key[v][j], tb.shift);
          e[v][j] = q < n ? __ldg(tb.slots + s[v][j]) : make_ulonglong2(JOIN_EMPTY, 0);
        }
#pragma unroll
      for (int v = 0; v < QV; ++v)
#pragma unroll
        for (int j = 0; j < 2; ++j) {
          const int64_t q = base + 2 * (v * QB + threadIdx.x) + j;
          uint64_t steps = 0;
          while (e[v][j].x != key[v][j] && e[v][j].x != JOIN_EMPTY && steps <= tb.mask) {
            s[v][j] = (s[v][j] + 1) & tb.mask;
            e[v][j] = __ldg(tb.slots + s[v][j]);
            ++steps;
          }
          const bool hit = q < n && e[v][j].x == key[v][j] && (e[v][j].y >> 32) != 0;
          brow[v][j] = hit ? (uint32_t)e[v][j].y : JOIN_NO_MATCH;
        }
    }
    unsigned long long pay[QV][2];
#pragma unroll
    for (int v = 0; v < QV; ++v)
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        pay[v][j] = 0;
        if (brow[v][j] != JOIN_NO_MATCH)
          pay[v][j] = tb.width == 8 ? __ldg(static_cast<const unsigned long long*>(tb.payload) + brow[v][j])
                                    : (unsigned long long)__ldg(static_cast<const unsigned int*>(tb.payload) + brow[v][j]);
      }
    // rank the tile's matches in row order, reserve the range, write
    uint32_t lpos[QV];
    const uint32_t lt = (1u << lane) - 1u;
#pragma unroll
    for (int v = 0; v < QV; ++v) {
      const uint32_t m0 = __ballot_sync(0xffffffffu, brow[v][0] != JOIN_NO_MATCH);
      const uint32_t m1 = __ballot_sync(0xffffffffu, brow[v][1] != JOIN_NO_MATCH);
      lpos[v] = __popc(m0 & lt) + __popc(m1 & lt);
      if (lane == 0) seg[v * (QB / 32) + warp] = __popc(m0) + __popc(m1);
    }
    __syncthreads();
    if (warp == 0) {
      const uint32_t x = seg[lane];
      const uint32_t incl = q_scan32(x);
      seg[lane] = incl - x;
      const uint32_t total = __shfl_sync(0xffffffffu, incl, 31);
      if (lane == 0) s_off = total ? atomicAdd(&qslots[slot].matches, (unsigned long long)total) : 0ULL;
    }
    __syncthreads();
    const unsigned long long off = s_off;
#pragma unroll
    for (int v = 0; v < QV; ++v) {
      uint64_t pos = off + seg[v * (QB / 32) + warp] + lpos[v];
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        if (brow[v][j] == JOIN_NO_MATCH) continue;
        const int64_t q = base + 2 * (v * QB + threadIdx.x) + j;
        if (pos < (uint64_t)n) {  // unique keys: at most one match per probe row
          __stcs(s_item.out_prow + pos, (uint32_t)q);
          if (tb.width == 8) __stcs(static_cast<unsigned long long*>(s_item.out_pay) + pos, pay[v][j]);
          else __stcs(static_cast<unsigned int*>(s_item.out_pay) + pos, (unsigned int)pay[v][j]);
        }
        ++pos;
      }
    }
    __threadfence();  // this thread's outputs before the tile counts as done
    __syncthreads();
    if (threadIdx.x == 0) {
      const unsigned int d = atomicAdd(&qslots[slot].tiles_done, 1u) + 1u;
      if (d == (unsigned int)s_item.n_tiles) {  // the request's last tile
        __threadfence();
        const unsigned long long m = atomicAdd(&qslots[slot].matches, 0ULL);
        qslots[slot].matches = 0;  // the slot's next request starts from zero
        qslots[slot].tiles_done = 0;
        __threadfence();
        volatile QDone* dn = &done[slot];
        dn->matches = m;
        __threadfence_system();
        dn->seq1 = rseq + 1;
        __threadfence_system();
      }
    }
    __syncthreads();  // s_item / s_tile are rewritten by the next claim
  }
}

}  // namespace

DeviceQueue::DeviceQueue(Ctx& ctx, int ctas_per_sm, int64_t wait_limit_us, int64_t idle_us) : ctx_(ctx) {
  PRISM_CUDA(cudaSetDevice(ctx.device));
  grid_ = ctx.sm_count * std::max(1, std::min(ctas_per_sm, 2));
  wait_limit_ = (uint32_t)std::max<int64_t>(1, std::min<int64_t>(wait_limit_us, 60LL * 1000 * 1000));
  // idle checks: 32 of ~0.2 us, then ~2 us each
  idle_limit_ = 32u + (uint32_t)std::max<int64_t>(0, std::min<int64_t>(idle_us, 1000000) / 2);
  PRISM_CUDA(cudaStreamCreateWithFlags(&qstream_, cudaStreamNonBlocking));
  // the persistent kernel's stream at the highest priority: its CTAs are
  // placed before the workers' pending blocks as SMs free up
  int lo = 0, hi = 0;
  PRISM_CUDA(cudaDeviceGetStreamPriorityRange(&lo, &hi));
  PRISM_CUDA(cudaStreamCreateWithPriority(&kstream_, cudaStreamNonBlocking, hi));
  PRISM_CUDA(cudaMalloc(&d_ring_, sizeof(QItem) * kRing));
  PRISM_CUDA(cudaMalloc(&d_ctl_, sizeof(QCtl)));
  PRISM_CUDA(cudaMalloc(&d_slots_, sizeof(QSlot) * kRing));
  PRISM_CUDA(cudaMalloc(&d_tables_, sizeof(QTable) * 256));
  PRISM_CUDA(cudaMemset(d_ring_, 0, sizeof(QItem) * kRing));
  PRISM_CUDA(cudaMemset(d_ctl_, 0, sizeof(QCtl)));
  PRISM_CUDA(cudaMemset(d_slots_, 0, sizeof(QSlot) * kRing));
  PRISM_CUDA(cudaHostAlloc(&h_items_, sizeof(QItem) * kRing, cudaHostAllocDefault));
  PRISM_CUDA(cudaHostAlloc(&h_pub_, sizeof(uint64_t) * kRing, cudaHostAllocDefault));
  PRISM_CUDA(cudaHostAlloc(&h_done_, sizeof(QDone) * kRing, cudaHostAllocMapped));
  PRISM_CUDA(cudaHostAlloc(&h_status_, sizeof(QStatus), cudaHostAllocMapped));
  std::memset(h_done_, 0, sizeof(QDone) * kRing);
  std::memset(h_status_, 0, sizeof(QStatus));
  PRISM_CUDA(cudaHostGetDevicePointer((void**)&d_done_, h_done_, 0));
  PRISM_CUDA(cudaHostGetDevicePointer((void**)&d_status_, h_status_, 0));
}

DeviceQueue::~DeviceQueue() {
  // ask the kernel to stop, wait for it (its waits are bounded), release
  const unsigned int one = 1;
  cudaMemcpyAsync(&d_ctl_->stop, &one, sizeof one, cudaMemcpyHostToDevice, qstream_);
  cudaStreamSynchronize(qstream_);
  cudaStreamSynchronize(kstream_);
  cudaFree(d_ring_);
  cudaFree(d_ctl_);
  cudaFree(d_slots_);
  cudaFree(d_tables_);
  cudaFreeHost(h_items_);
  cudaFreeHost(h_pub_);
  cudaFreeHost(h_done_);
  cudaFreeHost(h_status_);
  cudaStreamDestroy(qstream_);
  cudaStreamDestroy(kstream_);
}

int DeviceQueue::add_table(const JoinTable& t, const Column& payload) {
  std::lock_guard<std::mutex> lk(mu_);
  if (!t.int64_fast || t.has_dups) fail(PRISM_ERR_INVALID_ARGUMENT, "the device queue takes single Int64 keys without repeats");
  const int w = width_of(payload.type);
  if (payload.validity || (w != 4 && w != 8) || payload.type == TY_DICT)
    fail(PRISM_ERR_INVALID_ARGUMENT, "the device queue emits a fixed-width payload without nulls");
  if (tables_.size() >= 256) fail(PRISM_ERR_INVALID_ARGUMENT, "at most 256 tables on the device queue");
  QTable q{};
  q.dense = t.dense ? static_cast<const uint32_t*>(t.dense_rows->ptr) : nullptr;
  q.dmin = t.dmin;
  q.drange = t.drange;
  q.slots = t.slots ? static_cast<const ulonglong2*>(t.slots->ptr) : nullptr;
  q.mask = t.capacity ? t.capacity - 1 : 0;
  q.cap = t.capacity;
  q.shift = 64 - t.log2cap;
  q.payload = payload.values;
  q.width = w;
  tables_.push_back(q);
  const int id = (int)tables_.size() - 1;
  PRISM_CUDA(cudaMemcpyAsync(d_tables_ + id, &tables_.back(), sizeof q, cudaMemcpyHostToDevice, qstream_));
  PRISM_CUDA(cudaStreamSynchronize(qstream_));
  return id;
}

void DeviceQueue::ensure_running() {
  if (launched_) {
    const cudaError_t e = cudaStreamQuery(kstream_);
    if (e == cudaErrorNotReady) return;
    if (e != cudaSuccess) fail(PRISM_ERR_CUDA, std::string("device queue kernel: ") + cudaGetErrorString(e));
  }
  const unsigned long long first = pending_.empty() ? (unsigned long long)next_seq_ : (unsigned long long)pending_.begin()->first;
  // idle CTAs exit (after idle_limit_ checks) so they do not hold SMs the
  // workers' kernels could use
  queue_probe_kernel<<<grid_, QB, 0, kstream_>>>(d_ctl_, d_ring_, d_slots_, d_done_, d_status_, d_tables_, first,
                                                   idle_limit_, wait_limit_);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) fail(PRISM_ERR_CUDA, std::string("device queue kernel launch: ") + cudaGetErrorString(e));
  ctx_.note_launch();
  launched_ = true;
}

int64_t DeviceQueue::submit(int table, const int64_t* keys, int64_t rows, uint32_t* out_prow, void* out_pay) {
  std::lock_guard<std::mutex> lk(mu_);
  if (table < 0 || table >= (int)tables_.size()) fail(PRISM_ERR_INVALID_ARGUMENT, "unknown device queue table");
  if (rows <= 0 || rows >= (int64_t)UINT32_MAX) fail(PRISM_ERR_INVALID_ARGUMENT, "device queue request rows out of range");
  if ((int64_t)pending_.size() >= kRing) fail(PRISM_ERR_NO_MEMORY, "device queue full");
  const int64_t seq = next_seq_++;
  const int slot = (int)(seq % kRing);
  const uint64_t tiles = (uint64_t)((rows + QT - 1) / QT);
  QItem& it = h_items_[slot];
  it.keys = keys;
  it.out_prow = out_prow;
  it.out_pay = out_pay;
  it.rows = rows;
  it.tile_begin = published_;
  it.n_tiles = tiles;
  it.table = table;
  it.pad = 0;
  it.ready = (uint64_t)seq + 1;
  published_ += tiles;
  h_pub_[slot] = published_;
  // the descriptor, then the count that makes its tiles claimable (one stream: in this order)
  PRISM_CUDA(cudaMemcpyAsync(d_ring_ + slot, &it, sizeof it, cudaMemcpyHostToDevice, qstream_));
  PRISM_CUDA(cudaMemcpyAsync(&d_ctl_->published, &h_pub_[slot], sizeof(uint64_t), cudaMemcpyHostToDevice, qstream_));
  pending_[seq] = false;
  ensure_running();
  return seq;
}

int64_t DeviceQueue::submit_unready(int64_t tiles) {
  std::lock_guard<std::mutex> lk(mu_);
  if ((int64_t)pending_.size() >= kRing) fail(PRISM_ERR_NO_MEMORY, "device queue full");
  const int64_t seq = next_seq_++;
  const int slot = (int)(seq % kRing);
  published_ += (uint64_t)std::max<int64_t>(1, tiles);
  h_pub_[slot] = published_;
  // no descriptor: the tiles are published, the ring slot keeps an older one
  PRISM_CUDA(cudaMemcpyAsync(&d_ctl_->published, &h_pub_[slot], sizeof(uint64_t), cudaMemcpyHostToDevice, qstream_));
  pending_[seq] = true;
  ensure_running();
  return seq;
}

void DeviceQueue::recover() {
  // the kernel has exited: skip the tiles it gave up on, clear the counters
  PRISM_CUDA(cudaStreamSynchronize(qstream_));
  QCtl c{};
  c.published = published_;
  c.next_tile = published_;
  PRISM_CUDA(cudaMemcpyAsync(d_ctl_, &c, sizeof c, cudaMemcpyHostToDevice, qstream_));
  PRISM_CUDA(cudaMemsetAsync(d_slots_, 0, sizeof(QSlot) * kRing, qstream_));
  PRISM_CUDA(cudaStreamSynchronize(qstream_));
  h_status_->err = 0;
  launched_ = false;
}

int DeviceQueue::poll(const std::function<void(int64_t, int, int64_t)>& done) {
  std::vector<std::tuple<int64_t, int, int64_t>> out;
  {
    std::lock_guard<std::mutex> lk(mu_);
    for (auto it = pending_.begin(); it != pending_.end();) {
      const int slot = (int)(it->first % kRing);
      const volatile QDone* d = &h_done_[slot];
      if (!it->second && d->seq1 == (unsigned long long)it->first + 1) {
        out.emplace_back(it->first, PRISM_OK, (int64_t)d->matches);
        it = pending_.erase(it);
      } else {
        ++it;
      }
    }
    if (*(volatile unsigned int*)&h_status_->err) {
      // a wait ran out: every CTA exits; what is still pending fails
      PRISM_CUDA(cudaStreamSynchronize(kstream_));
      for (auto& p : pending_) out.emplace_back(p.first, PRISM_ERR_TIMEOUT, 0);
      pending_.clear();
      recover();
    } else if (!pending_.empty()) {
      ensure_running();  // the kernel may have gone idle just before a publish
    }
  }
  for (auto& [seq, st, m] : out) done(seq, st, m);
  return (int)out.size();
}

int64_t DeviceQueue::in_flight() {
  std::lock_guard<std::mutex> lk(mu_);
  return (int64_t)pending_.size();
}

}  // namespace prism
