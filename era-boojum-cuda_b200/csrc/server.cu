// server.cu -- continuous-batching LDE server.
//
// No counterpart in the reference (a library of stream-ordered calls).  A
// server owns, on one device: the twiddle tables (the context), a device
// arena of `memory_budget_bytes` allocated once at start-up, and `slots`
// pipelines (three streams each, host_lde.cuh).  Requests carry host buffers
// (pinned for overlap) and are queued by bc_lde_server_submit; a worker
// thread admits them in arrival order whenever a slot is free and the arena
// has room for the request's workspace, so requests that arrive while others
// are on the GPU join as soon as a slot and memory free up and their copies
// and kernels overlap on the device.  A request larger than its share of the
// arena is streamed through in column chunks that fit.  Completion is stamped
// by a host callback on the request's stream; latency = completion - submit.
//
// Device requests (bc_lde_server_submit_device: columns and outputs already in
// device memory, as a prover that produced them on the GPU has them) need no
// copies and no arena.  The worker takes every device request pending at that
// moment: those of at most max_batch_elems output elements are coalesced into
// ONE persistent batch launch (lde_batch.cu), larger ones run as their own
// fused LDE, all on the server's device stream.  At most two launches are in
// flight on it, so requests that arrive while they run wait for the next
// launch and join it.  The batch schedule goes through a pinned staging buffer
// and a device scratch buffer the server allocates once (two of each).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <mutex>
#include <new>
#include <thread>
#include <vector>

#include "../../include/bc_ntt.h"
#include "host_lde.cuh"

namespace bc {
namespace {

using Clock = std::chrono::steady_clock;

enum ReqState : int { PENDING = 0, RUNNING = 1, DONE = 2, CANCELLED = 3, FAILED = 4 };

struct Request {
  uint64_t id;
  const uint64_t *in;
  uint64_t *out;
  uint32_t log_n, cols, log_blowup;
  Clock::time_point submit, start, finish;
  int state = PENDING;
  cudaError_t error = cudaSuccess;
  // while running
  int slot = -1;
  size_t arena_off = 0, arena_bytes = 0;
  bool device = false; // buffers in device memory (bc_lde_server_submit_device)
};

// First-fit allocator over the device arena (offsets, 256-byte granules).
struct Arena {
  size_t size = 0;
  std::map<size_t, size_t> free_; // offset -> length
  void init(size_t s) {
    size = s;
    free_.clear();
    free_[0] = s;
  }
  bool alloc(size_t bytes, size_t &off) {
    bytes = (bytes + 255) & ~(size_t)255;
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        off = it->first;
        const size_t rest = it->second - bytes;
        free_.erase(it);
        if (rest) free_[off + bytes] = rest;
        return true;
      }
    }
    return false;
  }
  void release(size_t off, size_t bytes) {
    bytes = (bytes + 255) & ~(size_t)255;
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  size_t largest_free() const {
    size_t m = 0;
    for (auto &kv : free_) m = std::max(m, kv.second);
    return m;
  }
};

} // namespace
} // namespace bc

using namespace bc;

struct bc_lde_server {
  int device = 0;
  bc_lde_server_config cfg{};
  uint64_t *arena_base = nullptr;
  Arena arena;
  std::vector<HostPipe> pipes;
  std::vector<int> slot_busy;
  std::vector<Request *> slot_req; // the request holding each slot (until retired)
  std::mutex mu;
  std::condition_variable cv;      // worker wake-up
  std::condition_variable done_cv; // request completions
  std::deque<Request *> pending;
  std::map<uint64_t, Request *> all;
  // device requests: their queue, stream, and the batch schedule buffers (two of each)
  std::deque<Request *> pending_dev;
  cudaStream_t s_dev = nullptr;
  // completions of device launches are signalled from a second stream that waits on an event recorded after
  // each launch, so the device stream never stalls on a host callback; used events are destroyed by the worker
  cudaStream_t s_cb = nullptr;
  std::vector<cudaEvent_t> dead_events;
  void *d_sched[2] = {}, *h_stage[2] = {};
  cudaEvent_t stage_done[2] = {};
  int stage_next = 0;
  int dev_in_flight = 0;
  uint64_t dev_running = 0;
  uint64_t max_batch_elems = 1ull << 22; // 0: every device request as its own fused LDE
  uint64_t dev_batches = 0, dev_batched_requests = 0, dev_single_requests = 0;
  uint64_t next_id = 1;
  bool stop = false;
  std::thread worker;
  // stats
  uint64_t completed = 0, out_elems = 0;
  double busy_ms = 0;
  Clock::time_point first_submit{}, last_finish{};
  // latencies of the last LAT_WINDOW completed requests (ring), the worst of all
  std::vector<double> latencies_ms;
  size_t lat_next = 0;
  double max_latency_ms = 0;
};

namespace {

struct DoneCtx {
  bc_lde_server *srv;
  Request *req;
};

// Runs on a CUDA driver thread when the request's stream reaches its end;
// makes no CUDA calls.
void CUDART_CB on_request_done(void *p) {
  DoneCtx *d = static_cast<DoneCtx *>(p);
  {
    std::lock_guard<std::mutex> lock(d->srv->mu);
    d->req->finish = Clock::now();
    d->req->state = DONE;
  }
  d->srv->cv.notify_all();
  d->srv->done_cv.notify_all();
  delete d;
}

constexpr size_t LAT_WINDOW = 1u << 16;
constexpr size_t SERVER_SCHED_BYTES = 16u << 20; // one batch schedule (device scratch and pinned staging)

// Books a finished request's latency and output (caller holds the lock).
void book_done(bc_lde_server *s, Request *r);

// Frees a finished request's slot and arena region and books its latency
// (caller holds the lock; no-op unless the request holds a slot and finished).
void retire(bc_lde_server *s, Request *r) {
  if (r->slot < 0 || (r->state != DONE && r->state != FAILED)) return;
  s->slot_busy[r->slot] = 0;
  s->slot_req[r->slot] = nullptr;
  s->arena.release(r->arena_off, r->arena_bytes);
  r->slot = -1;
  if (r->state == DONE) book_done(s, r);
}


void book_done(bc_lde_server *s, Request *r) {
  const double lat = std::chrono::duration<double, std::milli>(r->finish - r->submit).count();
  if (s->latencies_ms.size() < LAT_WINDOW)
    s->latencies_ms.push_back(lat);
  else
    s->latencies_ms[s->lat_next] = lat;
  s->lat_next = (s->lat_next + 1) % LAT_WINDOW;
  s->max_latency_ms = std::max(s->max_latency_ms, lat);
  s->completed++;
  s->out_elems += ((uint64_t)r->cols << r->log_n) << r->log_blowup;
  if (r->finish > s->last_finish) s->last_finish = r->finish;
}

size_t request_workspace(const bc_lde_server *s, const Request &r, uint32_t &chunk) {
  const uint64_t per_col = 8ull * ((1ull << r.log_n) + ((1ull << r.log_n) << r.log_blowup));
  const size_t share = s->cfg.memory_budget_bytes / std::max<uint32_t>(1, s->cfg.slots);
  uint64_t cols = std::min<uint64_t>(r.cols, share / (per_col * HOST_NBUF));
  if (s->cfg.max_chunk_cols) cols = std::min<uint64_t>(cols, s->cfg.max_chunk_cols);
  chunk = (uint32_t)cols;
  return (size_t)cols * per_col * HOST_NBUF;
}

// Tries to start the oldest pending request; returns true if one started.
bool admit_one(bc_lde_server *s, std::unique_lock<std::mutex> &lock) {
  if (s->pending.empty()) return false;
  Request *r = s->pending.front();
  int slot = -1;
  for (size_t i = 0; i < s->slot_busy.size(); i++)
    if (!s->slot_busy[i]) {
      slot = (int)i;
      break;
    }
  if (slot < 0) return false;
  uint32_t chunk = 0;
  const size_t bytes = request_workspace(s, *r, chunk);
  size_t off = 0;
  if (chunk == 0 || !s->arena.alloc(bytes, off)) return false; // wait for memory to free up
  s->pending.pop_front();
  s->slot_busy[slot] = 1;
  s->slot_req[slot] = r;
  r->slot = slot;
  r->arena_off = off;
  r->arena_bytes = bytes;
  r->state = RUNNING;
  r->start = Clock::now();
  lock.unlock(); // enqueue without holding the lock (the done callback takes it)
  HostPipe &hp = s->pipes[slot];
  const uint64_t n = 1ull << r->log_n;
  cudaError_t e = host_lde_enqueue(hp, r->in, r->out, r->log_n, r->cols, n, n, (uint64_t)r->cols * n, r->log_blowup,
                                   s->arena_base + off / 8, chunk, false, nullptr);
  if (e == cudaSuccess) {
    DoneCtx *d = new (std::nothrow) DoneCtx{s, r};
    e = d ? cudaLaunchHostFunc(hp.s_out, on_request_done, d) : cudaErrorMemoryAllocation;
    if (e != cudaSuccess) delete d; // never handed to the stream
  }
  if (e != cudaSuccess) {
    // chunks enqueued before the failure may still run on this slot's streams:
    // wait for them before the slot and its arena region are handed out again
    cudaStreamSynchronize(hp.s_in);
    cudaStreamSynchronize(hp.s_comp);
    cudaStreamSynchronize(hp.s_out);
  }
  lock.lock();
  if (e != cudaSuccess) {
    r->error = e;
    r->state = FAILED;
    r->finish = Clock::now();
    s->done_cv.notify_all();
  }
  return true;
}

// Completion of one launch on the device stream (a batch or a single fused
// LDE): every request of it is done.  Runs on a CUDA driver thread; no CUDA calls.
struct GroupCtx {
  bc_lde_server *srv;
  std::vector<Request *> reqs;
  cudaEvent_t done = nullptr;
};

void CUDART_CB on_group_done(void *p) {
  GroupCtx *g = static_cast<GroupCtx *>(p);
  {
    std::lock_guard<std::mutex> lock(g->srv->mu);
    const Clock::time_point now = Clock::now();
    for (Request *r : g->reqs) {
      r->finish = now;
      r->state = DONE;
      book_done(g->srv, r);
    }
    g->srv->dev_running -= g->reqs.size();
    g->srv->dev_in_flight--;
    g->srv->dead_events.push_back(g->done);
  }
  g->srv->cv.notify_all();
  g->srv->done_cv.notify_all();
  delete g;
}

uint64_t out_elems(const Request &r) { return ((uint64_t)r.cols << r.log_n) << r.log_blowup; }

// Enqueues one launch of device requests (caller holds no lock); on failure
// the requests are marked failed.
void launch_device_group(bc_lde_server *s, std::vector<Request *> group, bool batch,
                         std::unique_lock<std::mutex> &lock) {
  const int stage = s->stage_next;
  if (batch) s->stage_next ^= 1;
  lock.unlock();
  cudaError_t e = cudaSuccess;
  if (batch) {
    // the staging buffer's previous copy (two launches ago) must have completed
    e = cudaEventSynchronize(s->stage_done[stage]);
    std::vector<bc_lde_job> jobs(group.size());
    for (size_t i = 0; i < group.size(); i++) {
      const Request &r = *group[i];
      const uint64_t n = 1ull << r.log_n;
      jobs[i] = bc_lde_job{r.in, r.out, n, n, (uint64_t)r.cols * n, r.log_n, r.cols, r.log_blowup, 0};
    }
    if (e == cudaSuccess)
      e = batch_enqueue_into(jobs.data(), (uint32_t)jobs.size(), s->d_sched[stage], s->h_stage[stage],
                             SERVER_SCHED_BYTES, s->s_dev);
    if (e == cudaSuccess) e = cudaEventRecord(s->stage_done[stage], s->s_dev);
  } else {
    const Request &r = *group[0];
    const uint64_t n = 1ull << r.log_n;
    e = lde_fused(tuned_plan(r.log_n, r.log_blowup), r.in, r.out, r.log_n, r.cols, n, n, (uint64_t)r.cols * n,
                  r.log_blowup, s->s_dev);
  }
  GroupCtx *g = nullptr;
  cudaEvent_t done = nullptr;
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&done, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventRecord(done, s->s_dev);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(s->s_cb, done, 0);
  if (e == cudaSuccess) {
    g = new (std::nothrow) GroupCtx{s, group, done};
    e = g ? cudaLaunchHostFunc(s->s_cb, on_group_done, g) : cudaErrorMemoryAllocation;
    if (e != cudaSuccess) {
      delete g;
      g = nullptr;
    }
  }
  if (e != cudaSuccess && done) {
    cudaStreamSynchronize(s->s_cb);
    cudaEventDestroy(done);
  }
  if (e != cudaSuccess) cudaStreamSynchronize(s->s_dev); // nothing of this group stays in flight
  lock.lock();
  if (e != cudaSuccess) {
    const Clock::time_point now = Clock::now();
    for (Request *r : group) {
      r->error = e;
      r->state = FAILED;
      r->finish = now;
    }
    s->dev_running -= group.size();
    s->dev_in_flight--;
    s->done_cv.notify_all();
  }
}

// Starts launches for the pending device requests while fewer than two are in
// flight (caller holds the lock).
void dispatch_device(bc_lde_server *s, std::unique_lock<std::mutex> &lock) {
  while (!s->pending_dev.empty() && s->dev_in_flight < 2 && !s->stop) {
    std::vector<Request *> small, big;
    uint64_t small_items = 0;
    while (!s->pending_dev.empty()) {
      Request *r = s->pending_dev.front();
      const bool batchable = s->max_batch_elems && out_elems(*r) <= s->max_batch_elems;
      // a schedule holds about 8 bytes per 4096-element work item and kernel: stop well before the scratch is full
      const uint64_t items = 4 * ((((uint64_t)r->cols << r->log_n) + 4095) / 4096) << r->log_blowup;
      if (batchable && !small.empty() && (small_items + items) * 8 > SERVER_SCHED_BYTES / 2) break;
      s->pending_dev.pop_front();
      r->state = RUNNING;
      r->start = Clock::now();
      s->dev_running++;
      if (batchable) {
        small.push_back(r);
        small_items += items;
      } else {
        big.push_back(r);
      }
    }
    if (small.size() == 1) {
      big.push_back(small[0]);
      small.clear();
    }
    if (!small.empty()) {
      s->dev_in_flight++;
      s->dev_batches++;
      s->dev_batched_requests += small.size();
      launch_device_group(s, small, true, lock);
    }
    for (Request *r : big) {
      s->dev_in_flight++;
      s->dev_single_requests++;
      launch_device_group(s, std::vector<Request *>{r}, false, lock);
    }
  }
}

void worker_main(bc_lde_server *s) {
  cudaSetDevice(s->device);
  std::unique_lock<std::mutex> lock(s->mu);
  while (!s->stop) {
    // retire finished requests: free their slot and memory
    for (Request *r : s->slot_req)
      if (r) retire(s, r);
    while (admit_one(s, lock)) {
    }
    dispatch_device(s, lock);
    for (cudaEvent_t ev : s->dead_events) cudaEventDestroy(ev); // their launches have completed
    s->dead_events.clear();
    s->cv.wait_for(lock, std::chrono::milliseconds(5));
  }
}

} // namespace

extern "C" cudaError_t bc_lde_server_create(const bc_lde_server_config *cfg, bc_lde_server **out) {
  if (!cfg || !out || cfg->slots == 0 || cfg->slots > 64 || cfg->memory_budget_bytes < (1u << 20))
    return cudaErrorInvalidValue;
  *out = nullptr;
  cudaError_t e = bc_ntt_context_create(12, 12);
  if (e != cudaSuccess) return e;
  bc_lde_server *s = new (std::nothrow) bc_lde_server();
  if (!s) return cudaErrorMemoryAllocation;
  s->cfg = *cfg;
  cudaGetDevice(&s->device);
  e = cudaMalloc(&s->arena_base, cfg->memory_budget_bytes);
  if (e != cudaSuccess) {
    delete s;
    return e;
  }
  s->arena.init(cfg->memory_budget_bytes);
  s->pipes.resize(cfg->slots);
  s->slot_busy.assign(cfg->slots, 0);
  s->slot_req.assign(cfg->slots, nullptr);
  for (auto &p : s->pipes) {
    if ((e = host_pipe_init(p)) != cudaSuccess) {
      for (auto &q : s->pipes) host_pipe_destroy(q);
      cudaFree(s->arena_base);
      delete s;
      return e;
    }
  }
  e = cudaStreamCreateWithFlags(&s->s_dev, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->s_cb, cudaStreamNonBlocking);
  for (int i = 0; i < 2 && e == cudaSuccess; i++) {
    e = cudaMalloc(&s->d_sched[i], SERVER_SCHED_BYTES);
    if (e == cudaSuccess) e = cudaMallocHost(&s->h_stage[i], SERVER_SCHED_BYTES);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->stage_done[i], cudaEventDisableTiming);
  }
  if (e != cudaSuccess) {
    for (int i = 0; i < 2; i++) {
      if (s->stage_done[i]) cudaEventDestroy(s->stage_done[i]);
      cudaFreeHost(s->h_stage[i]);
      cudaFree(s->d_sched[i]);
    }
    if (s->s_dev) cudaStreamDestroy(s->s_dev);
    if (s->s_cb) cudaStreamDestroy(s->s_cb);
    for (auto &q : s->pipes) host_pipe_destroy(q);
    cudaFree(s->arena_base);
    delete s;
    return e;
  }
  s->worker = std::thread(worker_main, s);
  *out = s;
  return cudaSuccess;
}

extern "C" cudaError_t bc_lde_server_submit_device(bc_lde_server *s, const uint64_t *dev_evals_bitrev,
                                                   uint64_t *dev_out, uint32_t log_n, uint32_t num_cols,
                                                   uint32_t log_blowup, uint64_t *request_id) {
  if (!s || !dev_evals_bitrev || !dev_out || !request_id || num_cols == 0) return cudaErrorInvalidValue;
  const uint64_t n = 1ull << log_n;
  if (!lde_args_ok(log_n, num_cols, n, n, (uint64_t)num_cols * n, log_blowup)) return cudaErrorInvalidValue;
  Request *r = new (std::nothrow) Request();
  if (!r) return cudaErrorMemoryAllocation;
  r->in = dev_evals_bitrev;
  r->out = dev_out;
  r->log_n = log_n;
  r->cols = num_cols;
  r->log_blowup = log_blowup;
  r->device = true;
  r->submit = Clock::now();
  {
    std::lock_guard<std::mutex> lock(s->mu);
    r->id = s->next_id++;
    if (s->first_submit == Clock::time_point{}) s->first_submit = r->submit;
    s->all[r->id] = r;
    s->pending_dev.push_back(r);
    *request_id = r->id;
  }
  s->cv.notify_all();
  return cudaSuccess;
}

extern "C" cudaError_t bc_lde_server_set_device_batching(bc_lde_server *s, uint64_t max_batch_elems) {
  if (!s) return cudaErrorInvalidValue;
  std::lock_guard<std::mutex> lock(s->mu);
  s->max_batch_elems = max_batch_elems;
  return cudaSuccess;
}

extern "C" cudaError_t bc_lde_server_get_device_stats(bc_lde_server *s, uint64_t *batches, uint64_t *batched_requests,
                                                      uint64_t *single_requests) {
  if (!s) return cudaErrorInvalidValue;
  std::lock_guard<std::mutex> lock(s->mu);
  if (batches) *batches = s->dev_batches;
  if (batched_requests) *batched_requests = s->dev_batched_requests;
  if (single_requests) *single_requests = s->dev_single_requests;
  return cudaSuccess;
}

extern "C" cudaError_t bc_lde_server_submit(bc_lde_server *s, const uint64_t *host_evals_bitrev, uint64_t *host_out,
                                            uint32_t log_n, uint32_t num_cols, uint32_t log_blowup,
                                            uint64_t *request_id) {
  if (!s || !host_evals_bitrev || !host_out || !request_id || num_cols == 0) return cudaErrorInvalidValue;
  const uint64_t n = 1ull << log_n;
  if (!lde_args_ok(log_n, num_cols, n, n, (uint64_t)num_cols * n, log_blowup)) return cudaErrorInvalidValue;
  // a request must fit the arena at least one column at a time
  const uint64_t per_col = 8ull * (n + (n << log_blowup));
  if (per_col * HOST_NBUF > s->cfg.memory_budget_bytes / s->cfg.slots) return cudaErrorInvalidValue;
  Request *r = new (std::nothrow) Request();
  if (!r) return cudaErrorMemoryAllocation;
  r->in = host_evals_bitrev;
  r->out = host_out;
  r->log_n = log_n;
  r->cols = num_cols;
  r->log_blowup = log_blowup;
  r->submit = Clock::now();
  {
    std::lock_guard<std::mutex> lock(s->mu);
    r->id = s->next_id++;
    if (s->first_submit == Clock::time_point{}) s->first_submit = r->submit;
    s->all[r->id] = r;
    s->pending.push_back(r);
    *request_id = r->id;
  }
  s->cv.notify_all();
  return cudaSuccess;
}

// state: 0 pending, 1 running, 2 done, 3 cancelled, 4 failed (see *error).
extern "C" cudaError_t bc_lde_server_poll(bc_lde_server *s, uint64_t id, int *state, double *latency_ms) {
  if (!s || !state) return cudaErrorInvalidValue;
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end()) return cudaErrorInvalidValue;
  Request *r = it->second;
  *state = r->state;
  if (latency_ms)
    *latency_ms = (r->state == DONE) ? std::chrono::duration<double, std::milli>(r->finish - r->submit).count() : -1.0;
  return r->state == FAILED ? r->error : cudaSuccess;
}

extern "C" cudaError_t bc_lde_server_wait(bc_lde_server *s, uint64_t id, uint32_t timeout_ms, double *latency_ms) {
  if (!s) return cudaErrorInvalidValue;
  std::unique_lock<std::mutex> lock(s->mu);
  if (s->all.find(id) == s->all.end()) return cudaErrorInvalidValue;
  // the record is looked up again after every wake-up: another thread may
  // release it meanwhile
  Request *r = nullptr;
  const bool ok = s->done_cv.wait_for(lock, std::chrono::milliseconds(timeout_ms), [&] {
    auto it = s->all.find(id);
    r = it == s->all.end() ? nullptr : it->second;
    return !r || r->state == DONE || r->state == FAILED || r->state == CANCELLED;
  });
  if (!ok) return cudaErrorTimeout;
  if (!r) return cudaErrorInvalidValue;
  if (latency_ms)
    *latency_ms = (r->state == DONE) ? std::chrono::duration<double, std::milli>(r->finish - r->submit).count() : -1.0;
  if (r->state == FAILED) return r->error;
  if (r->state == CANCELLED) return cudaErrorNotReady;
  return cudaSuccess;
}

// Cancels a request that has not been admitted yet (cudaErrorNotReady if it already runs or ran).
extern "C" cudaError_t bc_lde_server_cancel(bc_lde_server *s, uint64_t id) {
  if (!s) return cudaErrorInvalidValue;
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end()) return cudaErrorInvalidValue;
  Request *r = it->second;
  if (r->state != PENDING) return cudaErrorNotReady;
  s->pending.erase(std::remove(s->pending.begin(), s->pending.end(), r), s->pending.end());
  s->pending_dev.erase(std::remove(s->pending_dev.begin(), s->pending_dev.end(), r), s->pending_dev.end());
  r->state = CANCELLED;
  s->done_cv.notify_all();
  return cudaSuccess;
}

// Forgets a finished, cancelled or failed request (its id is then unknown);
// cudaErrorNotReady while it is pending or running.
extern "C" cudaError_t bc_lde_server_release(bc_lde_server *s, uint64_t id) {
  if (!s) return cudaErrorInvalidValue;
  std::lock_guard<std::mutex> lock(s->mu);
  auto it = s->all.find(id);
  if (it == s->all.end()) return cudaErrorInvalidValue;
  Request *r = it->second;
  if (r->state == PENDING || r->state == RUNNING) return cudaErrorNotReady;
  retire(s, r); // finished but not yet retired by the worker
  s->all.erase(it);
  delete r;
  s->done_cv.notify_all(); // waiters on this id return
  return cudaSuccess;
}

extern "C" cudaError_t bc_lde_server_get_stats(bc_lde_server *s, bc_lde_server_stats *st) {
  if (!s || !st) return cudaErrorInvalidValue;
  std::lock_guard<std::mutex> lock(s->mu);
  *st = bc_lde_server_stats{};
  st->completed = s->completed;
  uint64_t run = 0;
  for (Request *r : s->slot_req) run += r && r->state == RUNNING;
  st->pending = s->pending.size() + s->pending_dev.size();
  st->running = run + s->dev_running;
  std::vector<double> l = s->latencies_ms;
  std::sort(l.begin(), l.end());
  auto pct = [&](double q) { return l.empty() ? 0.0 : l[std::min(l.size() - 1, (size_t)(q * (l.size() - 1) + 0.5))]; };
  st->p50_ms = pct(0.50);
  st->p99_ms = pct(0.99);
  st->max_ms = s->max_latency_ms;
  const double span = std::chrono::duration<double>(s->last_finish - s->first_submit).count();
  st->span_s = span > 0 ? span : 0;
  st->out_melem_per_s = span > 0 ? (double)s->out_elems / span / 1e6 : 0;
  st->arena_largest_free = s->arena.largest_free();
  return cudaSuccess;
}

extern "C" cudaError_t bc_lde_server_destroy(bc_lde_server *s) {
  if (!s) return cudaErrorInvalidValue;
  {
    std::lock_guard<std::mutex> lock(s->mu);
    s->stop = true;
    for (Request *r : s->pending) r->state = CANCELLED;
    s->pending.clear();
    for (Request *r : s->pending_dev) r->state = CANCELLED;
    s->pending_dev.clear();
  }
  s->cv.notify_all();
  s->worker.join();
  cudaError_t e = cudaSuccess;
  for (auto &p : s->pipes) {
    cudaError_t e2 = cudaStreamSynchronize(p.s_out);
    if (e2 != cudaSuccess) e = e2;
  }
  cudaError_t e3 = cudaStreamSynchronize(s->s_dev);
  if (e3 != cudaSuccess) e = e3;
  e3 = cudaStreamSynchronize(s->s_cb);
  if (e3 != cudaSuccess) e = e3;
  cudaDeviceSynchronize(); // host callbacks of finished requests have run
  for (cudaEvent_t ev : s->dead_events) cudaEventDestroy(ev);
  for (auto &p : s->pipes) host_pipe_destroy(p);
  for (int i = 0; i < 2; i++) {
    cudaEventDestroy(s->stage_done[i]);
    cudaFreeHost(s->h_stage[i]);
    cudaFree(s->d_sched[i]);
  }
  cudaStreamDestroy(s->s_dev);
  cudaStreamDestroy(s->s_cb);
  cudaFree(s->arena_base);
  for (auto &kv : s->all) delete kv.second;
  delete s;
  return e;
}
