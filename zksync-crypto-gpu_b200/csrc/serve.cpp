// Serving runtime: commitment requests arrive over time; a worker thread admits them onto the
// device by HBM footprint and in-flight slots, runs them concurrently on a pool of streams
// (continuous batching: a request that arrives while others run starts as soon as memory and a
// slot free up, and its kernels overlap theirs), and reports per-request latency.
//
// Device memory is stream-ordered (cudaMallocFromPoolAsync / cudaFreeAsync from a memory pool
// private to the server, which keeps freed blocks cached between requests), so admission costs
// no device synchronisation and the device's default pool keeps its settings.
// The streams carry CUDA stream priorities by request size: a small request's blocks are
// scheduled ahead of the remaining blocks of a large one as SMs free up, so its latency does not
// include the large request's kernels (unless flat_priority is set).
//
// Locking: the server mutex guards the queues, the request table and the counters only.  The
// worker decides admissions and completions under it, then releases it for the CUDA calls that
// can block the host (a host-to-device copy from pageable memory runs synchronously, the cap
// copy waits for its stream), so submit, wait and stats never wait behind a copy.  A request
// that is started and not yet done belongs to the worker: nothing else erases it from the table
// (std::map keeps the addresses of its other entries stable).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "glc_internal.h"

namespace glc {

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

struct Request {
  uint64_t ticket = 0;
  glc_serve_request req{};
  uint64_t footprint = 0;
  double t_submit = 0, t_start = 0, t_done = 0;
  int status = 0;
  bool started = false, done = false, cancelled = false;
  int stream = -1;
  cudaEvent_t done_event = nullptr;
  uint64_t *d_evals = nullptr, *d_lde = nullptr, *d_trees = nullptr, *d_cap = nullptr;
};

struct Server {
  glc_server_config cfg{};
  int device = 0;
  std::vector<cudaStream_t> streams;
  std::vector<uint32_t> stream_load;
  std::vector<uint32_t> stream_class;  // 0 = highest priority
  uint32_t classes = 1;
  cudaStream_t copy_stream = nullptr;  // result copies to the host
  cudaMemPool_t pool = nullptr;        // private stream-ordered pool (release threshold: never)
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<uint64_t> pending;
  std::map<uint64_t, Request> reqs;
  uint64_t next_ticket = 1;
  uint64_t used_bytes = 0;
  uint32_t inflight = 0;
  bool stop = false;
  std::thread worker;
  // stats
  uint64_t completed = 0, rejected = 0, peak_bytes = 0;
  uint32_t peak_inflight = 0;
};

uint64_t request_footprint(const glc_serve_request &r) {
  const uint64_t n = 1ull << r.log_n, f = 1ull << r.log_lde;
  return 8ull * ((uint64_t)r.cols * n * (1 + f) + f * 8 * n + (4ull << r.log_cap));
}

static int request_check(const glc_serve_request &r) {
  if (!r.host_evals || !r.host_cap) return fail("serve: null host buffer");
  glc_commit_job j{};
  j.evals = reinterpret_cast<const uint64_t *>(1);
  j.evals_stride = 1ull << std::min(r.log_n, 31u);
  j.log_n = r.log_n;
  j.cols = r.cols;
  j.log_lde = r.log_lde;
  j.log_cap = r.log_cap;
  j.lde = j.trees = j.cap = reinterpret_cast<uint64_t *>(1);
  return commit_check(j);
}

// Priority class of a request: its footprint against the budget, in factors of 4 (below 1/64,
// 1/16, 1/4, above), so a small job's kernels are not queued behind a large job's blocks.
static uint32_t request_class(const Server &s, uint64_t footprint) {
  uint32_t c = 0;
  for (uint64_t edge = s.cfg.hbm_budget_bytes / 64; c + 1 < s.classes && footprint >= edge; edge *= 4) c++;
  return c;
}

// Picks the stream of an admitted request (worker thread, lock held by the caller).
static void assign_stream(Server &s, Request &q) {
  // least-loaded stream of the request's priority class (any stream when none has that class)
  const uint32_t cls = request_class(s, q.footprint);
  int best = -1;
  for (size_t i = 0; i < s.streams.size(); i++)
    if (s.stream_class[i] == cls && (best < 0 || s.stream_load[i] < s.stream_load[best])) best = (int)i;
  if (best < 0) {
    best = 0;
    for (size_t i = 1; i < s.streams.size(); i++)
      if (s.stream_load[i] < s.stream_load[best]) best = (int)i;
  }
  q.stream = best;
  s.stream_load[best]++;
}

// Allocates, copies and enqueues one admitted request (worker thread, lock NOT held: the copy
// from pageable host memory blocks this thread until the data is staged).
static int start_request(Server &s, Request &q) {
  const glc_serve_request &r = q.req;
  const uint64_t n = 1ull << r.log_n, f = 1ull << r.log_lde;
  cudaStream_t st = s.streams[q.stream];
  cudaError_t e = cudaSuccess;
  // The pool keeps freed blocks mapped (release threshold: never), so requests of other sizes can
  // find the device full of cached blocks they cannot use.  On an allocation failure the pool
  // gives those blocks back (trim) and the allocation is retried; if that is not enough, the
  // frees still queued on the server's streams are waited for and the pool trimmed again.
  auto alloc = [&](uint64_t **p, uint64_t elems) {
    if (e != cudaSuccess) return;
    const size_t bytes = elems * sizeof(uint64_t);
    e = cudaMallocFromPoolAsync((void **)p, bytes, s.pool, st);
    for (int attempt = 0; e == cudaErrorMemoryAllocation && attempt < 2; attempt++) {
      cudaGetLastError();  // allocation failures are not sticky; clear the record
      if (attempt == 1)
        for (cudaStream_t x : s.streams) cudaStreamSynchronize(x);
      cudaMemPoolTrimTo(s.pool, 0);
      e = cudaMallocFromPoolAsync((void **)p, bytes, s.pool, st);
    }
  };
  alloc(&q.d_evals, (uint64_t)r.cols * n);
  alloc(&q.d_lde, f * r.cols * n);
  alloc(&q.d_trees, f * 8 * n);
  alloc(&q.d_cap, 4ull << r.log_cap);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(q.d_evals, r.host_evals, (uint64_t)r.cols * n * 8, cudaMemcpyHostToDevice, st);
  int err = (int)e;
  if (!err) {
    glc_commit_job j{};
    j.evals = q.d_evals;
    j.evals_stride = n;
    j.log_n = r.log_n;
    j.cols = r.cols;
    j.log_lde = r.log_lde;
    j.log_cap = r.log_cap;
    j.lde = q.d_lde;
    j.trees = q.d_trees;
    j.cap = q.d_cap;
    err = commit_enqueue(j, st);
  }
  // the cap goes to the host at completion (worker thread, private copy stream): a copy enqueued
  // here into pageable memory would block this thread until the whole job had finished
  if (!err) err = (int)cudaEventCreateWithFlags(&q.done_event, cudaEventDisableTiming);
  if (!err) err = (int)cudaEventRecord(q.done_event, st);
  return err;
}

static void free_request(Server &s, Request &q, bool keep_resident) {
  cudaStream_t st = s.streams[q.stream >= 0 ? q.stream : 0];
  if (q.d_evals) cudaFreeAsync(q.d_evals, st);
  if (q.d_cap) cudaFreeAsync(q.d_cap, st);
  q.d_evals = q.d_cap = nullptr;
  if (!keep_resident) {
    if (q.d_lde) cudaFreeAsync(q.d_lde, st);
    if (q.d_trees) cudaFreeAsync(q.d_trees, st);
    q.d_lde = q.d_trees = nullptr;
  }
  if (q.done_event) cudaEventDestroy(q.done_event);
  q.done_event = nullptr;
}

// Copies the cap of a finished request to the host and frees its buffers (worker thread, lock
// NOT held).  Returns the request's final status.
static int finish_request(Server &s, Request &q, int status) {
  if (!status) {
    cudaError_t ce = cudaMemcpyAsync(q.req.host_cap, q.d_cap, (4ull << q.req.log_cap) * 8, cudaMemcpyDeviceToHost,
                                     s.copy_stream);
    if (ce == cudaSuccess) ce = cudaStreamSynchronize(s.copy_stream);
    status = (int)ce;
  }
  free_request(s, q, q.req.keep_resident && !status);
  return status;
}

static void worker_main(Server *s) {
  cudaSetDevice(s->device);
  std::vector<Request *> admitted, finished;
  std::vector<int> finished_status;
  std::unique_lock<std::mutex> lk(s->mu);
  while (true) {
    // admit: FIFO; a request that does not fit lets smaller ones behind it start (backfill)
    admitted.clear();
    for (auto it = s->pending.begin(); it != s->pending.end() && s->inflight < s->cfg.max_inflight;) {
      Request &q = s->reqs[*it];
      if (q.cancelled) {
        it = s->pending.erase(it);
        continue;
      }
      if (s->used_bytes + q.footprint > s->cfg.hbm_budget_bytes) {
        ++it;
        continue;
      }
      q.started = true;
      q.t_start = now_s();
      s->used_bytes += q.footprint;
      s->inflight++;
      s->peak_bytes = std::max(s->peak_bytes, s->used_bytes);
      s->peak_inflight = std::max(s->peak_inflight, s->inflight);
      assign_stream(*s, q);
      admitted.push_back(&q);
      it = s->pending.erase(it);
    }
    if (!admitted.empty()) {
      lk.unlock();
      for (Request *q : admitted) q->status = start_request(*s, *q);
      lk.lock();
    }
    // completions: decided under the lock, copies and frees outside it
    finished.clear();
    finished_status.clear();
    bool any_inflight = false;
    for (auto &kv : s->reqs) {
      Request &q = kv.second;
      if (!q.started || q.done) continue;
      cudaError_t qe = q.status ? cudaSuccess : cudaEventQuery(q.done_event);
      if (q.status || qe != cudaErrorNotReady) {
        finished.push_back(&q);
        finished_status.push_back(q.status ? q.status : (qe != cudaSuccess ? (int)qe : 0));
      } else {
        any_inflight = true;
      }
    }
    if (!finished.empty()) {
      lk.unlock();
      for (size_t i = 0; i < finished.size(); i++) finished_status[i] = finish_request(*s, *finished[i], finished_status[i]);
      lk.lock();
      for (size_t i = 0; i < finished.size(); i++) {
        Request &q = *finished[i];
        q.status = finished_status[i];
        q.done = true;
        q.t_done = now_s();
        s->stream_load[q.stream]--;
        if (!(q.req.keep_resident && !q.status)) s->used_bytes -= q.footprint;
        s->inflight--;
        s->completed++;
      }
      s->cv_done.notify_all();
      continue;  // admissions may fit now
    }
    if (s->stop && s->pending.empty() && !any_inflight) break;
    if (any_inflight)
      s->cv_work.wait_for(lk, std::chrono::microseconds(50));
    else
      s->cv_work.wait_for(lk, std::chrono::milliseconds(20));
  }
}

}  // namespace glc

using namespace glc;

struct glc_server {
  Server s;
};

extern "C" glc_status glc_server_create(const glc_server_config *config, glc_server **out) {
  if (!config || !out) return fail("serve: null argument");
  if (config->max_inflight == 0 || config->hbm_budget_bytes == 0) return fail("serve: zero budget or slots");
  if (!current_tables()) return fail("serve: glc_context_create has not been called on this device");
  auto *srv = new glc_server();
  Server &s = srv->s;
  s.cfg = *config;
  if (s.cfg.streams == 0) s.cfg.streams = 8;
  cudaGetDevice(&s.device);
  // a private pool that keeps freed blocks: requests of similar sizes reuse them without new
  // mappings, and the device's default pool (shared with other code in the process) is untouched
  cudaMemPoolProps props{};
  props.allocType = cudaMemAllocationTypePinned;
  props.handleTypes = cudaMemHandleTypeNone;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = s.device;
  cudaError_t pe = cudaMemPoolCreate(&s.pool, &props);
  if (pe == cudaSuccess) {
    uint64_t threshold = UINT64_MAX;
    pe = cudaMemPoolSetAttribute(s.pool, cudaMemPoolAttrReleaseThreshold, &threshold);
  }
  if (pe != cudaSuccess) {
    if (s.pool) cudaMemPoolDestroy(s.pool);
    delete srv;
    return (int)pe;
  }
  if (cudaStreamCreateWithFlags(&s.copy_stream, cudaStreamNonBlocking) != cudaSuccess) {
    cudaMemPoolDestroy(s.pool);
    delete srv;
    return fail("serve: cannot create the copy stream");
  }
  // stream priorities: up to 4 classes from the device's range (greatest is numerically lowest)
  int least = 0, greatest = 0;
  if (!s.cfg.flat_priority && cudaDeviceGetStreamPriorityRange(&least, &greatest) == cudaSuccess)
    s.classes = std::max<uint32_t>(1, std::min<uint32_t>({4u, (uint32_t)(least - greatest + 1), s.cfg.streams}));
  for (uint32_t i = 0; i < s.cfg.streams; i++) {
    cudaStream_t st;
    const uint32_t cls = i % s.classes;
    const int prio = s.classes > 1 ? greatest + (int)(cls * (uint32_t)(least - greatest) / (s.classes - 1)) : 0;
    const cudaError_t e = s.classes > 1 ? cudaStreamCreateWithPriority(&st, cudaStreamNonBlocking, prio)
                                        : cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
      for (auto x : s.streams) cudaStreamDestroy(x);
      cudaStreamDestroy(s.copy_stream);
      cudaMemPoolDestroy(s.pool);
      delete srv;
      return (int)e;
    }
    s.streams.push_back(st);
    s.stream_load.push_back(0);
    s.stream_class.push_back(cls);
  }
  s.worker = std::thread(worker_main, &s);
  *out = srv;
  return 0;
}

extern "C" glc_status glc_server_submit(glc_server *srv, const glc_serve_request *req, uint64_t *ticket) {
  if (!srv || !req || !ticket) return fail("serve: null argument");
  int e = request_check(*req);
  if (e) return e;
  Server &s = srv->s;
  const double t_submit = now_s();  // before the lock: latency counts any wait for it
  const uint64_t fp = request_footprint(*req);
  std::lock_guard<std::mutex> lk(s.mu);
  if (fp > s.cfg.hbm_budget_bytes) {
    s.rejected++;
    return fail("serve: request footprint exceeds the HBM budget");
  }
  if (s.stop) return fail("serve: server is shutting down");
  Request q;
  q.ticket = s.next_ticket++;
  q.req = *req;
  q.footprint = fp;
  q.t_submit = t_submit;
  s.reqs[q.ticket] = q;
  s.pending.push_back(q.ticket);
  *ticket = q.ticket;
  s.cv_work.notify_all();
  return 0;
}

extern "C" glc_status glc_server_cancel(glc_server *srv, uint64_t ticket) {
  if (!srv) return fail("serve: null server");
  Server &s = srv->s;
  std::lock_guard<std::mutex> lk(s.mu);
  auto it = s.reqs.find(ticket);
  if (it == s.reqs.end()) return fail("serve: unknown ticket");
  if (it->second.started) return fail("serve: request already started");
  it->second.cancelled = true;
  it->second.done = true;
  it->second.status = (int)cudaErrorInvalidValue;
  s.cv_done.notify_all();
  return 0;
}

extern "C" glc_status glc_server_wait(glc_server *srv, uint64_t ticket, double timeout_s, glc_serve_result *out) {
  if (!srv || !out) return fail("serve: null argument");
  Server &s = srv->s;
  std::unique_lock<std::mutex> lk(s.mu);
  auto it = s.reqs.find(ticket);
  if (it == s.reqs.end()) return fail("serve: unknown ticket");
  const auto deadline = std::chrono::steady_clock::now() + std::chrono::duration<double>(timeout_s);
  while (!s.reqs[ticket].done) {
    if (timeout_s >= 0 && s.cv_done.wait_until(lk, deadline) == std::cv_status::timeout && !s.reqs[ticket].done)
      return (int)cudaErrorNotReady;
    if (timeout_s < 0) s.cv_done.wait(lk);
  }
  Request &q = s.reqs[ticket];
  out->ticket = ticket;
  out->status = q.status;
  out->queue_s = q.started ? q.t_start - q.t_submit : 0;
  out->latency_s = q.t_done - q.t_submit;
  out->device_lde = q.d_lde;
  out->device_trees = q.d_trees;
  if (!q.req.keep_resident || q.status) s.reqs.erase(ticket);
  return 0;
}

extern "C" glc_status glc_server_release(glc_server *srv, uint64_t ticket) {
  if (!srv) return fail("serve: null server");
  Server &s = srv->s;
  std::lock_guard<std::mutex> lk(s.mu);
  auto it = s.reqs.find(ticket);
  if (it == s.reqs.end() || !it->second.done) return fail("serve: no finished resident request with this ticket");
  Request &q = it->second;
  cudaStream_t st = s.streams[q.stream >= 0 ? q.stream : 0];
  if (q.d_lde) cudaFreeAsync(q.d_lde, st);
  if (q.d_trees) cudaFreeAsync(q.d_trees, st);
  if (q.req.keep_resident && !q.status) s.used_bytes -= q.footprint;
  s.reqs.erase(it);
  s.cv_work.notify_all();
  return 0;
}

extern "C" glc_status glc_server_get_stats(glc_server *srv, glc_server_stats *out) {
  if (!srv || !out) return fail("serve: null argument");
  Server &s = srv->s;
  std::lock_guard<std::mutex> lk(s.mu);
  out->completed = s.completed;
  out->rejected = s.rejected;
  out->pending = s.pending.size();
  out->inflight = s.inflight;
  out->used_bytes = s.used_bytes;
  out->peak_bytes = s.peak_bytes;
  out->peak_inflight = s.peak_inflight;
  return 0;
}

extern "C" glc_status glc_server_destroy(glc_server *srv) {
  if (!srv) return 0;
  Server &s = srv->s;
  {
    std::lock_guard<std::mutex> lk(s.mu);
    s.stop = true;
    s.cv_work.notify_all();
  }
  if (s.worker.joinable()) s.worker.join();
  cudaSetDevice(s.device);
  for (auto &kv : s.reqs) {
    Request &q = kv.second;
    if (q.started) {
      if (q.d_lde) cudaFreeAsync(q.d_lde, s.streams[q.stream]);
      if (q.d_trees) cudaFreeAsync(q.d_trees, s.streams[q.stream]);
    }
  }
  for (auto st : s.streams) {
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
  }
  if (s.copy_stream) cudaStreamDestroy(s.copy_stream);
  if (s.pool) cudaMemPoolDestroy(s.pool);  // every block was freed above (stream-ordered, synchronised)
  delete srv;
  return 0;
}
