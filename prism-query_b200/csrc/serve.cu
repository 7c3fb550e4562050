// serve.cu — the serving loop behind the C ABI (prism_server_*, prism_serve_*).
//
// Requests of uneven sizes (probes of resident hash tables, GROUP BYs over
// device-resident batches) arrive one at a time from any host thread. The
// server keeps the caller's tables resident, runs requests on several worker
// threads that each own a context and CUDA stream (so their kernels overlap
// on the device), admits a job only while its device footprint fits the
// budget, hands the smallest ready job to the next free worker (the oldest
// one once it has waited 10 ms, so no job starves), and coalesces
// small requests that arrive close together into one launch:
//   * small probes of one table are concatenated and probed once; the output
//     is in probe-row order, so each request's matches are one contiguous
//     range, cut out by a binary search and rebased to the request's rows;
//   * small GROUP BYs with one config and schema are concatenated with a
//     segment id as the first group key; groups come out in first-seen order,
//     hence grouped by segment, and each request takes its range.
// Every result equals the result of running the request alone.
//
// The reference has no serving loop; its analogue is the Flight action
// handler answering one operator call at a time (prism-flight/src/shuffle_writer.rs:294-349
// calling prism-bench/src/handler.rs:78,
// with PartitionStore as the resident-table registry,
// shuffle_writer.rs:42-86).
#include <algorithm>
#include <cstdlib>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <queue>
#include <string>
#include <thread>
#include <vector>

#include "join.hpp"
#include "prims.hpp"
#include "prism_gpu.h"
#include "queue.hpp"
#include "runtime.hpp"

using namespace prism;

namespace {

// index of the first element >= v in the ascending array a[0, n)
__device__ __forceinline__ int64_t lower_bound_u32(const uint32_t* a, int64_t n, uint64_t v) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    int64_t mid = (lo + hi) >> 1;
    if ((uint64_t)a[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// segment of row r: the last i with starts[i] <= r (starts ascending, k entries)
__device__ __forceinline__ int segment_of(const uint64_t* starts, int k, uint64_t r) {
  int lo = 0, hi = k - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (starts[mid] <= r) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__global__ void cuts_kernel(const uint32_t* prow, int64_t m, const uint64_t* starts, int nb, unsigned long long* cuts) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < nb) cuts[i] = (unsigned long long)lower_bound_u32(prow, m, starts[i]);
}

__global__ void rebase_kernel(const uint32_t* prow, int64_t m, const uint64_t* starts, int k, uint32_t* rel) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < m; j += (int64_t)gridDim.x * blockDim.x)
    rel[j] = prow[j] - (uint32_t)starts[segment_of(starts, k, prow[j])];
}

__global__ void segments_kernel(int32_t* seg, int64_t n, const uint64_t* starts, int k) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
    seg[j] = segment_of(starts, k, (uint64_t)j);
}

__global__ void iota_kernel(uint32_t* p, int64_t n) {
  for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
    p[j] = (uint32_t)j;
}

// an aggregate config owned by the server (the caller's may go away)
struct AggConfig {
  std::vector<int32_t> group_by;
  std::vector<std::string> names;
  std::vector<prism_agg_expr> aggs;
  prism_agg_config cfg{};
  void fix() {
    for (size_t i = 0; i < aggs.size(); ++i) aggs[i].output_name = names[i].c_str();
    cfg.n_group_by = (int32_t)group_by.size();
    cfg.group_by = group_by.data();
    cfg.n_aggs = (int32_t)aggs.size();
    cfg.aggs = aggs.data();
  }
};

struct Request {
  int64_t ticket = 0;
  int kind = 0;  // 0 probe, 1 aggregate
  int32_t table = -1;
  const int64_t* keys = nullptr;
  int64_t rows = 0;
  const prism_batch* batch = nullptr;
  std::shared_ptr<AggConfig> cfg;
  std::string shape;  // requests of one shape may share a launch ("" = never)
};

struct Job {
  std::vector<Request> reqs;
  int64_t rows = 0;
};

struct JobOrder {  // smallest job first, then arrival
  int64_t rows;
  int64_t seq;
  bool operator<(const JobOrder& o) const { return rows != o.rows ? rows > o.rows : seq > o.seq; }
};

struct Result {
  bool done = false;
  int status = PRISM_OK;
  std::string message;
  prism_batch* out = nullptr;
};

struct TableRef {
  const prism_hash_table* table;
  int32_t payload_col;  // build column emitted with the probe row
  bool coalesce;        // payload null-free and fixed width: results can be views
  int queue_id = -1;    // index on the device queue, or -1
};

// a probe in flight on the device queue
struct Queued {
  Request req;
  MemP prow, pay;
  uint64_t footprint = 0;
};

}  // namespace

struct prism_server {
  int device = 0;
  uint64_t budget = 0;
  int64_t coalesce_rows = 0;
  int max_coalesce = 1;
  std::vector<prism_ctx*> ctxs;
  std::vector<std::thread> threads;
  std::thread dispatcher;
  std::mutex mu;
  std::condition_variable cv_inbox, cv_jobs, cv_done, cv_admit;
  std::deque<Request> inbox;
  std::priority_queue<std::pair<JobOrder, int64_t>> order;  // (order, job id)
  std::deque<std::pair<int64_t, std::chrono::steady_clock::time_point>> fifo;  // (job id, queued at)
  std::map<int64_t, Job> jobs;  // queued jobs (ids in order/fifo that are gone here were taken)
  int64_t next_job = 0, next_seq = 0, next_ticket = 1;
  std::map<int64_t, Result> results;
  std::deque<int64_t> completed;  // tickets in completion order (prism_serve_wait_any)
  std::vector<TableRef> tables;
  uint64_t in_use = 0;
  bool closing = false, dispatcher_done = false;
  std::string last_error;
  // the device work queue (prism_server_set_device_queue): eligible probes
  // are drained by one persistent kernel; a host thread reports completions
  prism_ctx* qctx = nullptr;
  std::unique_ptr<DeviceQueue> queue;
  int64_t queue_max_rows = 0;
  std::map<int64_t, Queued> queued;  // queue seq -> request
  std::thread qthread;
  bool qstop = false;
};

namespace {

uint64_t footprint(const Job& j) {
  if (j.reqs[0].kind == 0) return (uint64_t)j.rows * (8 + 4 + 4 + 12) + ((uint64_t)1 << 20);
  uint64_t in = 0;
  for (auto& r : j.reqs)
    for (auto& c : r.batch->impl.cols) in += (uint64_t)r.rows * std::max(1, width_of(c->type) > 0 ? width_of(c->type) : 8);
  return 2 * in + (uint64_t)j.rows * 4 + ((uint64_t)64 << 20);
}

void push_job(prism_server* s, Job&& j) {  // s->mu held
  int64_t id = s->next_job++;
  s->order.push({JobOrder{j.rows, s->next_seq++}, id});
  s->fifo.push_back({id, std::chrono::steady_clock::now()});
  s->jobs.emplace(id, std::move(j));
  s->cv_jobs.notify_one();
}

// The next job: the smallest queued one, unless the oldest has waited longer
// than kMaxWait (smallest-first alone could starve a large job under a
// steady stream of small ones). s->mu held, some job queued.
constexpr auto kMaxWait = std::chrono::milliseconds(10);
int64_t take_job(prism_server* s) {
  while (!s->fifo.empty() && !s->jobs.count(s->fifo.front().first)) s->fifo.pop_front();
  while (!s->order.empty() && !s->jobs.count(s->order.top().second)) s->order.pop();
  int64_t id;
  if (!s->fifo.empty() && std::chrono::steady_clock::now() - s->fifo.front().second > kMaxWait) {
    id = s->fifo.front().first;
    s->fifo.pop_front();
  } else {
    id = s->order.top().second;
    s->order.pop();
  }
  return id;
}

void finish(prism_server* s, const Request& r, int status, const std::string& msg, prism_batch* out) {
  std::lock_guard<std::mutex> lk(s->mu);
  Result& res = s->results[r.ticket];
  res.done = true;
  res.status = status;
  res.message = msg;
  res.out = out;
  s->completed.push_back(r.ticket);
  s->cv_done.notify_all();
}

void dispatch(prism_server* s) {
  std::map<std::string, Job> pending;
  std::unique_lock<std::mutex> lk(s->mu);
  for (;;) {
    if (s->inbox.empty()) {
      if (!pending.empty()) {
        // nothing more within half a millisecond: hand over what is pending
        s->cv_inbox.wait_for(lk, std::chrono::microseconds(500), [&] { return !s->inbox.empty() || s->closing; });
        if (s->inbox.empty()) {
          for (auto& p : pending) push_job(s, std::move(p.second));
          pending.clear();
          continue;
        }
      } else {
        s->cv_inbox.wait(lk, [&] { return !s->inbox.empty() || s->closing; });
      }
      if (s->inbox.empty() && s->closing) break;
    }
    Request r = std::move(s->inbox.front());
    s->inbox.pop_front();
    if (r.shape.empty() || r.rows >= s->coalesce_rows) {
      Job j;
      j.rows = r.rows;
      j.reqs.push_back(std::move(r));
      push_job(s, std::move(j));
      continue;
    }
    Job& j = pending[r.shape];
    j.rows += r.rows;
    j.reqs.push_back(std::move(r));
    if (j.rows >= s->coalesce_rows || (int)j.reqs.size() >= s->max_coalesce) {
      std::string key = j.reqs[0].shape;
      push_job(s, std::move(j));
      pending.erase(key);
    }
  }
  for (auto& p : pending) push_job(s, std::move(p.second));
  s->dispatcher_done = true;
  s->cv_jobs.notify_all();
}

prism_batch* new_batch(prism_ctx* w, Batch b) {
  auto* out = new prism_batch();
  out->impl = std::move(b);
  out->ctx = w;
  return out;
}

MemP upload_starts(Ctx& x, const std::vector<uint64_t>& starts) {
  MemP m = x.alloc(starts.size() * 8);
  x.h2d_staged(m->ptr, starts.data(), starts.size() * 8);
  return m;
}

void run_probe(prism_server* s, prism_ctx* w, Job& job) {
  Ctx& x = w->impl;
  const TableRef& tb = s->tables[job.reqs[0].table];
  const int k = (int)job.reqs.size();
  std::vector<uint64_t> starts(k + 1, 0);
  for (int i = 0; i < k; ++i) starts[i + 1] = starts[i] + (uint64_t)job.reqs[i].rows;
  const int64_t n = (int64_t)starts[k];
  auto kc = std::make_shared<Column>();
  kc->type = TY_I64;
  kc->name = "key";
  kc->nullable = false;
  kc->length = n;
  if (k == 1) {
    kc->values = const_cast<int64_t*>(job.reqs[0].keys);
  } else {  // one probe over the concatenated keys
    MemP stage = x.alloc((size_t)std::max<int64_t>(n, 1) * 8);
    for (int i = 0; i < k; ++i)
      if (job.reqs[i].rows)
        PRISM_CUDA(cudaMemcpyAsync(static_cast<int64_t*>(stage->ptr) + starts[i], job.reqs[i].keys,
                                   (size_t)job.reqs[i].rows * 8, cudaMemcpyDeviceToDevice, x.stream));
    kc->values = stage->ptr;
    kc->owners.push_back(stage);
  }
  prism_batch probe;
  probe.impl.rows = n;
  probe.impl.cols.push_back(kc);
  probe.ctx = w;
  const int32_t pk = 0;
  const int32_t oc[2] = {PRISM_COL_PROBE_ROW_INDEX, 1 + tb.payload_col};
  prism_batch* res = nullptr;
  int rc = prism_join_project(w, tb.table, &probe, &pk, 1, oc, 2, &res);
  if (rc) fail(rc, prism_last_error(w));
  std::unique_ptr<prism_batch> hold(res);
  if (k == 1) {
    x.sync();
    finish(s, job.reqs[0], PRISM_OK, "", hold.release());
    return;
  }
  const int64_t m = res->impl.rows;
  const Column& prow = *res->impl.cols[0];
  const Column& pay = *res->impl.cols[1];
  MemP dstarts = upload_starts(x, starts);
  MemP dcuts, drel;
  unsigned long long* cuts = x.alloc_t<unsigned long long>(k + 1, dcuts);
  uint32_t* rel = x.alloc_t<uint32_t>((size_t)std::max<int64_t>(m, 1), drel);
  const uint64_t* st = static_cast<const uint64_t*>(dstarts->ptr);
  const uint32_t* pr = static_cast<const uint32_t*>(prow.values);
  cuts_kernel<<<1, 128, 0, x.stream>>>(pr, m, st, k + 1, cuts);
  x.check_launch("cuts_kernel");
  if (m) {
    rebase_kernel<<<grid_for(x, m, 256), 256, 0, x.stream>>>(pr, m, st, k, rel);
    x.check_launch("rebase_kernel");
  }
  std::vector<unsigned long long> hc(k + 1);
  PRISM_CUDA(cudaMemcpyAsync(hc.data(), cuts, (k + 1) * 8, cudaMemcpyDeviceToHost, x.stream));
  x.sync();
  const int pw = width_of(pay.type);
  for (int i = 0; i < k; ++i) {
    const int64_t a = (int64_t)hc[i], rows = (int64_t)hc[i + 1] - a;
    Batch b;
    b.rows = rows;
    auto c0 = std::make_shared<Column>(prow);
    c0->values = rel + a;
    c0->length = rows;
    c0->owners = {drel};
    auto c1 = std::make_shared<Column>(pay);  // a view: the payload is null-free and fixed width
    c1->values = static_cast<uint8_t*>(pay.values) + a * pw;
    c1->length = rows;
    b.cols = {c0, c1};
    finish(s, job.reqs[i], PRISM_OK, "", new_batch(w, std::move(b)));
  }
}

void run_aggregate(prism_server* s, prism_ctx* w, Job& job) {
  Ctx& x = w->impl;
  const int k = (int)job.reqs.size();
  if (k == 1) {
    prism_batch* out = nullptr;
    int rc = prism_hash_aggregate(w, job.reqs[0].batch, &job.reqs[0].cfg->cfg, &out);
    if (rc) fail(rc, prism_last_error(w));
    x.sync();
    finish(s, job.reqs[0], PRISM_OK, "", out);
    return;
  }
  // one GROUP BY over the concatenated batches, a segment id as the first key
  std::vector<uint64_t> starts(k + 1, 0);
  for (int i = 0; i < k; ++i) starts[i + 1] = starts[i] + (uint64_t)job.reqs[i].rows;
  const int64_t n = (int64_t)starts[k];
  Batch cat;
  cat.rows = n;
  MemP dstarts = upload_starts(x, starts);
  ColP seg = make_column(x, TY_I32, "__segment", n, false);
  seg->nullable = false;
  if (n) {
    segments_kernel<<<grid_for(x, n, 256), 256, 0, x.stream>>>(static_cast<int32_t*>(seg->values), n,
                                                                static_cast<const uint64_t*>(dstarts->ptr), k);
    x.check_launch("segments_kernel");
  }
  cat.cols.push_back(seg);
  const Batch& b0 = job.reqs[0].batch->impl;
  for (size_t c = 0; c < b0.cols.size(); ++c) {
    std::vector<const Column*> parts;
    for (auto& r : job.reqs) parts.push_back(r.batch->impl.cols[c].get());
    cat.cols.push_back(concat_columns(x, parts));
  }
  AggConfig sc = *job.reqs[0].cfg;
  sc.group_by.insert(sc.group_by.begin(), -1);
  for (auto& g : sc.group_by) g += 1;
  for (auto& a : sc.aggs) a.column += 1;
  sc.fix();
  prism_batch cb;
  cb.impl = std::move(cat);
  cb.ctx = w;
  prism_batch* out = nullptr;
  int rc = prism_hash_aggregate(w, &cb, &sc.cfg, &out);
  if (rc) fail(rc, prism_last_error(w));
  std::unique_ptr<prism_batch> hold(out);
  const int64_t G = out->impl.rows;
  std::vector<int32_t> hseg((size_t)std::max<int64_t>(G, 1));
  if (G)
    PRISM_CUDA(cudaMemcpyAsync(hseg.data(), out->impl.cols[0]->values, (size_t)G * 4, cudaMemcpyDeviceToHost, x.stream));
  MemP mi;
  uint32_t* iota = x.alloc_t<uint32_t>((size_t)std::max<int64_t>(G, 1), mi);
  if (G) {
    iota_kernel<<<grid_for(x, G, 256), 256, 0, x.stream>>>(iota, G);
    x.check_launch("iota_kernel");
  }
  x.sync();
  // groups are in first-seen order over the concatenation: by segment
  int64_t lo = 0;
  for (int i = 0; i < k; ++i) {
    int64_t hi = lo;
    while (hi < G && hseg[hi] == i) ++hi;
    Batch b;
    b.rows = hi - lo;
    for (size_t c = 1; c < out->impl.cols.size(); ++c) {
      const Column& src = *out->impl.cols[c];
      b.cols.push_back(take(x, src, iota + lo, nullptr, hi - lo, src.name, src.nullable));
    }
    x.sync();
    finish(s, job.reqs[i], PRISM_OK, "", new_batch(w, std::move(b)));
    lo = hi;
  }
  if (lo != G) fail(PRISM_ERR_INTERNAL, "coalesced groups are not in segment order");
}

void work(prism_server* s, prism_ctx* w) {
  cudaSetDevice(s->device);
  for (;;) {
    Job job;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_jobs.wait(lk, [&] { return !s->jobs.empty() || s->dispatcher_done; });
      if (s->jobs.empty()) return;
      int64_t id = take_job(s);
      job = std::move(s->jobs.at(id));
      s->jobs.erase(id);
    }
    const uint64_t fp = footprint(job);
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_admit.wait(lk, [&] { return s->in_use == 0 || s->in_use + fp <= s->budget; });
      s->in_use += fp;
    }
    int status = PRISM_OK;
    std::string msg;
    try {
      if (job.reqs[0].kind == 0) run_probe(s, w, job);
      else run_aggregate(s, w, job);
    } catch (const Failure& f) {
      status = f.code;
      msg = f.msg;
    } catch (const std::exception& e) {
      status = PRISM_ERR_INTERNAL;
      msg = e.what();
    }
    if (status != PRISM_OK) {  // every request of the job not yet answered fails alike
      cudaGetLastError();
      for (auto& r : job.reqs) {
        bool answered;
        {
          std::lock_guard<std::mutex> lk(s->mu);
          answered = s->results[r.ticket].done;
        }
        if (!answered) finish(s, r, status, msg, nullptr);
      }
    }
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->in_use -= fp;
      s->cv_admit.notify_all();
    }
  }
}

// Reports the device queue's finished requests: each result is a batch of
// views into the request's own output buffers.
void queue_loop(prism_server* s) {
  cudaSetDevice(s->device);
  int quiet = 0;
  for (;;) {
    int got = 0;
    try {
      got = s->queue->poll([&](int64_t seq, int status, int64_t matches) {
        Queued q;
        {
          std::lock_guard<std::mutex> lk(s->mu);
          auto it = s->queued.find(seq);
          if (it == s->queued.end()) return;
          q = std::move(it->second);
          s->queued.erase(it);
        }
        prism_batch* out = nullptr;
        std::string msg;
        if (status == PRISM_OK) {
          const TableRef& tb = s->tables[q.req.table];
          const Column& pay = *tb.table->t->build.cols[tb.payload_col];
          Batch b;
          b.rows = matches;
          auto c0 = std::make_shared<Column>();
          c0->type = TY_U32;
          c0->name = "probe_idx";
          c0->nullable = false;
          c0->length = matches;
          c0->values = q.prow->ptr;
          c0->owners = {q.prow};
          auto c1 = std::make_shared<Column>();
          c1->type = pay.type;
          c1->name = pay.name;
          c1->nullable = pay.nullable;
          c1->precision = pay.precision;
          c1->scale = pay.scale;
          c1->length = matches;
          c1->values = q.pay->ptr;
          c1->owners = {q.pay};
          b.cols = {c0, c1};
          out = new prism_batch();
          out->impl = std::move(b);
          out->ctx = s->qctx;
        } else {
          msg = "device queue: a wait in the persistent kernel ran out";
        }
        finish(s, q.req, status, msg, out);
        std::lock_guard<std::mutex> lk(s->mu);
        s->in_use -= q.footprint;
        s->cv_admit.notify_all();
      });
    } catch (const Failure& f) {
      std::lock_guard<std::mutex> lk(s->mu);
      s->last_error = f.msg;
    }
    {
      std::lock_guard<std::mutex> lk(s->mu);
      if (s->qstop && s->queued.empty()) return;
    }
    if (got) {
      quiet = 0;
      continue;
    }
    // spin briefly after activity, then sleep in short steps
    if (++quiet < 2000) std::this_thread::yield();
    else std::this_thread::sleep_for(std::chrono::microseconds(50));
  }
}

// Queues an eligible probe on the device queue (admission by the outputs'
// footprint, outputs from the queue context's pool). Returns false when the
// probe should take the worker path.
bool queue_probe(prism_server* s, Request& r, int64_t* ticket) {
  int qid;
  int w;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (!s->queue || s->closing || r.rows <= 0 || r.rows > s->queue_max_rows) return false;
    qid = s->tables[r.table].queue_id;
    if (qid < 0) return false;
    const TableRef& tb = s->tables[r.table];
    w = width_of(tb.table->t->build.cols[tb.payload_col]->type);
  }
  const uint64_t fp = (uint64_t)r.rows * (4 + (uint64_t)w) + 512;
  {
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv_admit.wait(lk, [&] { return s->in_use == 0 || s->in_use + fp <= s->budget; });
    s->in_use += fp;
    r.ticket = s->next_ticket++;
    s->results[r.ticket] = Result{};
  }
  Queued q;
  try {
    Ctx& x = s->qctx->impl;
    {
      std::lock_guard<std::recursive_mutex> lk(x.mu);
      q.prow = x.alloc((size_t)r.rows * 4);
      q.pay = x.alloc((size_t)r.rows * w);
      x.sync();  // the outputs exist before the kernel may write them
    }
    q.req = r;
    q.footprint = fp;
    std::lock_guard<std::mutex> lk(s->mu);  // registered before its completion can be reported
    const int64_t seq = s->queue->submit(qid, r.keys, r.rows, static_cast<uint32_t*>(q.prow->ptr), q.pay->ptr);
    s->queued.emplace(seq, std::move(q));
  } catch (const Failure& f) {
    finish(s, r, f.code, f.msg, nullptr);
    std::lock_guard<std::mutex> lk(s->mu);
    s->in_use -= fp;
    s->cv_admit.notify_all();
  }
  *ticket = r.ticket;
  return true;
}

std::string agg_shape(const prism_batch* b, const prism_agg_config* cfg) {
  if (cfg->n_group_by == 0) return "";  // a global aggregate must run alone (grouped semantics differ)
  std::string k = "agg";
  for (int i = 0; i < cfg->n_group_by; ++i) k += "|g" + std::to_string(cfg->group_by[i]);
  for (int i = 0; i < cfg->n_aggs; ++i)
    k += "|a" + std::to_string(cfg->aggs[i].column) + ":" + std::to_string(cfg->aggs[i].func) + ":" +
         (cfg->aggs[i].output_name ? cfg->aggs[i].output_name : "");
  for (auto& c : b->impl.cols) {
    if (c->type == TY_DICT) return "";  // dictionaries differ per batch
    k += "|t" + std::to_string(c->type) + ":" + std::to_string(c->scale) + ":" + (c->nullable ? "n" : "") + c->name;
  }
  return k;
}

int submit(prism_server* s, Request&& r, int64_t* ticket) {
  std::lock_guard<std::mutex> lk(s->mu);
  if (s->closing) return PRISM_ERR_INVALID_ARGUMENT;
  r.ticket = s->next_ticket++;
  s->results[r.ticket] = Result{};
  *ticket = r.ticket;
  s->inbox.push_back(std::move(r));
  s->cv_inbox.notify_one();
  return PRISM_OK;
}

}  // namespace

extern "C" {

int prism_server_create(int32_t device, uint64_t budget_bytes, int32_t workers, int64_t coalesce_rows,
                        int32_t max_coalesce, prism_server** out) {
  if (!out || workers < 1 || workers > 64 || max_coalesce < 1) return PRISM_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  auto* s = new prism_server();
  s->device = device;
  s->budget = budget_bytes ? budget_bytes : ((uint64_t)120 << 30);
  s->coalesce_rows = std::max<int64_t>(0, coalesce_rows);
  s->max_coalesce = max_coalesce;
  for (int i = 0; i < workers; ++i) {
    prism_ctx* c = nullptr;
    int rc = prism_ctx_create(device, 0, &c);
    if (rc) {
      for (auto* x : s->ctxs) prism_ctx_destroy(x);
      delete s;
      return rc;
    }
    s->ctxs.push_back(c);
  }
  // each worker's memory pool grown once up front (one block allocated and
  // returned; the pool keeps it), so that the first jobs do not map new
  // device memory while other workers' kernels run.
  // PRISM_SERVER_POOL_MB sets the size per worker (default 2048, 0: none).
  uint64_t pre = (uint64_t)2048 << 20;
  if (const char* e = std::getenv("PRISM_SERVER_POOL_MB")) pre = (uint64_t)std::max(0LL, std::atoll(e)) << 20;
  pre = std::min<uint64_t>(pre, s->budget / (uint64_t)workers);
  if (pre) {
    try {
      for (auto* c : s->ctxs) {
        MemP m = c->impl.alloc(pre);
        m.reset();
        c->impl.sync();
      }
    } catch (const Failure&) {
      // not enough free memory for the whole block: the pools grow on demand
    }
  }
  s->dispatcher = std::thread(dispatch, s);
  for (auto* c : s->ctxs) s->threads.emplace_back(work, s, c);
  *out = s;
  return PRISM_OK;
}

int prism_server_add_table(prism_server* s, const prism_hash_table* table, int32_t payload_col, int32_t* table_id) {
  if (!s || !table || !table_id) return PRISM_ERR_INVALID_ARGUMENT;
  const Batch& b = table->t->build;
  if (payload_col < 0 || payload_col >= (int32_t)b.cols.size()) {
    std::lock_guard<std::mutex> lk(s->mu);
    s->last_error = "payload column out of range";
    return PRISM_ERR_INVALID_ARGUMENT;
  }
  const Column& p = *b.cols[payload_col];
  const int w = width_of(p.type);
  const bool coalesce = !p.validity && (w == 4 || w == 8) && p.type != TY_DICT;
  std::lock_guard<std::mutex> lk(s->mu);
  TableRef ref{table, payload_col, coalesce, -1};
  if (s->queue && coalesce && table->t->int64_fast && !table->t->has_dups) {
    try {
      ref.queue_id = s->queue->add_table(*table->t, p);
    } catch (const Failure& f) {
      s->last_error = f.msg;
      return f.code;
    }
  }
  s->tables.push_back(ref);
  *table_id = (int32_t)s->tables.size() - 1;
  return PRISM_OK;
}

int prism_serve_probe(prism_server* s, int32_t table_id, const int64_t* keys, int64_t n, int64_t* ticket) {
  if (!s || !ticket || n < 0 || (n > 0 && !keys)) return PRISM_ERR_INVALID_ARGUMENT;
  Request r;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (table_id < 0 || table_id >= (int32_t)s->tables.size()) {
      s->last_error = "unknown table id";
      return PRISM_ERR_INVALID_ARGUMENT;
    }
    if (s->tables[table_id].coalesce && s->tables[table_id].table->t->int64_fast)
      r.shape = "probe|" + std::to_string(table_id);
  }
  if (n >= (int64_t)UINT32_MAX) return PRISM_ERR_INVALID_ARGUMENT;
  r.kind = 0;
  r.table = table_id;
  r.keys = keys;
  r.rows = n;
  if (queue_probe(s, r, ticket)) return PRISM_OK;
  return submit(s, std::move(r), ticket);
}

int prism_server_set_device_queue(prism_server* s, int32_t enable, int64_t max_rows, int32_t ctas_per_sm,
                                  int32_t wait_limit_ms) {
  if (!s || max_rows < 0 || ctas_per_sm < 0 || wait_limit_ms < 0) return PRISM_ERR_INVALID_ARGUMENT;
  if (!enable) {
    std::lock_guard<std::mutex> lk(s->mu);
    s->queue_max_rows = 0;  // new probes take the worker path; the queue drains
    return PRISM_OK;
  }
  try {
    std::lock_guard<std::mutex> lk(s->mu);
    if (!s->queue) {
      int rc = prism_ctx_create(s->device, 0, &s->qctx);
      if (rc) fail(rc, "device queue context");
      // PRISM_QUEUE_IDLE_US: how long an idle CTA of the persistent kernel
      // waits for work before it exits (default 100)
      const char* iu = std::getenv("PRISM_QUEUE_IDLE_US");
      const int64_t idle_us = iu ? std::max<int64_t>(0, std::atoll(iu)) : 100;
      s->queue = std::make_unique<DeviceQueue>(s->qctx->impl, ctas_per_sm ? ctas_per_sm : 1,
                                               (int64_t)(wait_limit_ms ? wait_limit_ms : 1000) * 1000, idle_us);
      for (auto& tb : s->tables)
        if (tb.coalesce && tb.table->t->int64_fast && !tb.table->t->has_dups)
          tb.queue_id = s->queue->add_table(*tb.table->t, *tb.table->t->build.cols[tb.payload_col]);
      s->qthread = std::thread(queue_loop, s);
    }
    s->queue_max_rows = max_rows ? max_rows : (int64_t)UINT32_MAX - 1;
    return PRISM_OK;
  } catch (const Failure& f) {
    s->last_error = f.msg;
    return f.code;
  }
}

int prism_server_inject_unready(prism_server* s, int64_t* ticket) {
  if (!s || !ticket) return PRISM_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(s->mu);
  if (!s->queue) {
    s->last_error = "the device queue is not enabled";
    return PRISM_ERR_INVALID_ARGUMENT;
  }
  try {
    Request r;
    r.ticket = s->next_ticket++;
    r.kind = 0;
    s->results[r.ticket] = Result{};
    Queued q;
    q.req = r;
    const int64_t seq = s->queue->submit_unready(1);
    s->queued.emplace(seq, std::move(q));
    *ticket = r.ticket;
    return PRISM_OK;
  } catch (const Failure& f) {
    s->last_error = f.msg;
    return f.code;
  }
}

int prism_serve_aggregate(prism_server* s, const prism_batch* batch, const prism_agg_config* cfg, int64_t* ticket) {
  if (!s || !batch || !cfg || !ticket || (cfg->n_group_by > 0 && !cfg->group_by) || (cfg->n_aggs > 0 && !cfg->aggs))
    return PRISM_ERR_INVALID_ARGUMENT;
  Request r;
  r.kind = 1;
  r.batch = batch;
  r.rows = batch->impl.rows;
  auto c = std::make_shared<AggConfig>();
  c->group_by.assign(cfg->group_by, cfg->group_by + cfg->n_group_by);
  for (int i = 0; i < cfg->n_aggs; ++i) {
    c->aggs.push_back(cfg->aggs[i]);
    c->names.push_back(cfg->aggs[i].output_name ? cfg->aggs[i].output_name : "");
  }
  c->fix();
  r.cfg = c;
  r.shape = agg_shape(batch, cfg);
  return submit(s, std::move(r), ticket);
}

int prism_serve_poll(prism_server* s, int64_t ticket, int32_t wait_ms, prism_batch** out) {
  if (!s || !out) return PRISM_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->results.find(ticket);
  if (it == s->results.end()) {
    s->last_error = "unknown ticket";
    return PRISM_ERR_INVALID_ARGUMENT;
  }
  auto ready = [&] {
    auto f = s->results.find(ticket);
    return f == s->results.end() || f->second.done;
  };
  if (!it->second.done && wait_ms < 0) s->cv_done.wait(lk, ready);
  else if (!it->second.done && wait_ms > 0) s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), ready);
  it = s->results.find(ticket);
  if (it == s->results.end()) {  // another thread took the result meanwhile
    s->last_error = "unknown ticket";
    return PRISM_ERR_INVALID_ARGUMENT;
  }
  Result& r = it->second;
  if (!r.done) return PRISM_ERR_TIMEOUT;
  int status = r.status;
  if (status) s->last_error = r.message;
  *out = r.out;
  s->results.erase(ticket);
  return status;
}

int prism_serve_wait_any(prism_server* s, int32_t wait_ms, int64_t* ticket) {
  if (!s || !ticket) return PRISM_ERR_INVALID_ARGUMENT;
  std::unique_lock<std::mutex> lk(s->mu);
  auto ready = [&] { return !s->completed.empty(); };
  if (wait_ms < 0) s->cv_done.wait(lk, ready);
  else if (wait_ms > 0) s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), ready);
  if (s->completed.empty()) return PRISM_ERR_TIMEOUT;
  *ticket = s->completed.front();
  s->completed.pop_front();
  return PRISM_OK;
}

const char* prism_server_last_error(prism_server* s) { return s ? s->last_error.c_str() : "null server"; }

void prism_server_destroy(prism_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->closing = true;
    s->cv_inbox.notify_all();
  }
  s->dispatcher.join();
  for (auto& t : s->threads) t.join();
  if (s->queue) {
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->qstop = true;
    }
    s->qthread.join();  // after every queued request is reported
    s->queue.reset();   // stops the persistent kernel
  }
  for (auto& r : s->results)
    if (r.second.out) prism_batch_free(r.second.out);
  s->results.clear();
  // results already handed out may outlive the server and free their device
  // memory through the worker context that allocated it: the contexts are
  // retired (unused pool memory released), not destroyed
  for (auto* c : s->ctxs) {
    cudaStreamSynchronize(c->impl.stream);
    cudaMemPoolTrimTo(c->impl.pool, 0);
  }
  if (s->qctx) {
    cudaStreamSynchronize(s->qctx->impl.stream);
    cudaMemPoolTrimTo(s->qctx->impl.pool, 0);
  }
  delete s;
}

}  // extern "C"
