// queue.hpp — the device work queue of the serving loop: probe requests of
// resident tables are drained by one persistent kernel.
//
// The host writes each request's descriptor into a ring in device memory and
// then advances the count of published tiles (2,048 probe rows each), both
// by asynchronous copies on one stream, so a descriptor is in place before
// its tiles can be claimed. The resident kernel's CTAs claim tiles in order
// (one atomic each), look up the request holding the tile, probe its keys
// against the request's table (dense rows or hash slots), reserve the tile's
// output range with one atomic on the request's match counter and write
// (probe row, payload) there; the CTA finishing a request's last tile writes
// its match count into page-locked host memory, which a host thread polls.
// Requests of different tables and sizes share the launch, tile by tile, and
// no request pays a launch or a stream synchronisation of its own.
//
// Every wait in the kernel is bounded: a CTA with nothing to claim exits
// after an idle period (the host relaunches the kernel when work arrives),
// and a CTA waiting for a descriptor that never arrives gives up after the
// configured limit, records DERR_TIMEOUT and makes every CTA exit; the host
// then fails the requests in flight with PRISM_ERR_TIMEOUT and resets the
// queue, which stays usable.
#pragma once

#include <cstdint>
#include <functional>
#include <map>
#include <mutex>
#include <vector>

#include "join.hpp"
#include "runtime.hpp"

namespace prism {

struct QItem;
struct QCtl;
struct QSlot;
struct QDone;
struct QStatus;
struct QTable;

class DeviceQueue {
 public:
  static constexpr int kRing = 4096;  // requests in flight at most

  // ctx: the context whose pool holds the outputs (kept alive by the caller)
  // idle_us: a CTA with nothing to claim exits after about this long
  DeviceQueue(Ctx& ctx, int ctas_per_sm, int64_t wait_limit_us, int64_t idle_us = 100);
  ~DeviceQueue();

  // Registers a resident table (single Int64 key, no repeated keys) and its
  // payload column (fixed width 4 or 8, no nulls); returns its queue index.
  int add_table(const JoinTable& t, const Column& payload);

  // Queues a probe of `rows` device-resident keys; outputs must hold `rows`
  // entries (unique keys: at most one match per probe row). Returns the
  // request's sequence number. Blocks while kRing requests are in flight.
  int64_t submit(int table, const int64_t* keys, int64_t rows, uint32_t* out_prow, void* out_pay);
  // Failure injection for tests: publishes `tiles` tiles of a request whose
  // descriptor is never written, so the kernel's bounded wait runs out.
  int64_t submit_unready(int64_t tiles);

  // Calls done(seq, status, matches) for every request finished since the
  // last call (status PRISM_OK or PRISM_ERR_TIMEOUT); relaunches the kernel
  // when requests wait and it has exited. Returns the number reported.
  int poll(const std::function<void(int64_t, int, int64_t)>& done);
  int64_t in_flight();

 private:
  void ensure_running();  // mu_ held
  void recover();         // mu_ held: after an abort

  Ctx& ctx_;
  int grid_ = 0;
  uint32_t wait_limit_ = 0;
  uint32_t idle_limit_ = 0;
  std::mutex mu_;
  cudaStream_t qstream_ = nullptr;  // descriptor / publish copies
  cudaStream_t kstream_ = nullptr;  // the persistent kernel
  QItem* d_ring_ = nullptr;
  QCtl* d_ctl_ = nullptr;
  QSlot* d_slots_ = nullptr;
  QTable* d_tables_ = nullptr;
  QItem* h_items_ = nullptr;      // page-locked staging of the descriptors
  uint64_t* h_pub_ = nullptr;     // page-locked staging of the published counts
  QDone* h_done_ = nullptr;       // mapped: written by the device
  QStatus* h_status_ = nullptr;   // mapped: written by the device
  QDone* d_done_ = nullptr;       // device aliases of the mapped memory
  QStatus* d_status_ = nullptr;
  std::vector<QTable> tables_;
  int64_t next_seq_ = 0;
  uint64_t published_ = 0;
  std::map<int64_t, bool> pending_;  // seq -> injected (never completes by itself)
  bool launched_ = false;
};

}  // namespace prism
