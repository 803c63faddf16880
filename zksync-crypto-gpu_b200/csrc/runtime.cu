// Batched commitment runtime: stream pool, cost-balanced scheduling of uneven jobs, CUDA graphs.
//
// glc_commit_batch enqueues many commitment jobs behind one caller stream: it forks onto a pool
// of non-blocking streams (event fork/join, so the whole batch is one unit on the caller's
// stream and can be captured into a CUDA graph), assigns jobs largest-first to the least-loaded
// stream by estimated cost, and joins.  Small jobs then fill SMs that a single job leaves idle,
// and the memory-bound NTT passes of one job run beside the integer-bound hashing of another.
// glc_commit_graph_* capture a batch once and replay it with one launch.
#include <algorithm>
#include <mutex>
#include <numeric>
#include <vector>

#include "glc_internal.h"

namespace glc {

struct StreamPool {
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> done;
  cudaEvent_t fork = nullptr;
  std::mutex mu;
};

static StreamPool g_pools[MAX_DEVICES];

static int pool_get(uint32_t want, StreamPool **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  if (dev < 0 || dev >= MAX_DEVICES) return fail("batch: device ordinal out of range");
  StreamPool &p = g_pools[dev];
  if (!p.fork) {
    e = cudaEventCreateWithFlags(&p.fork, cudaEventDisableTiming);
    if (e != cudaSuccess) return (int)e;
  }
  while (p.streams.size() < want) {
    cudaStream_t s;
    cudaEvent_t ev;
    e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) return (int)e;
    e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e != cudaSuccess) return (int)e;
    p.streams.push_back(s);
    p.done.push_back(ev);
  }
  *out = &p;
  return 0;
}

// Work estimate of a job: Poseidon2 permutations dominate (472 modmul each) plus the NTT butterflies.
double job_cost(const glc_commit_job &j) {
  const double n = double(1ull << j.log_n), f = double(1u << j.log_lde);
  const double perms = f * n * ((j.cols + 7) / 8) + f * n;
  const double butterflies = (1.0 + f) * j.cols * n * 0.5 * j.log_n;
  return perms * 472.0 + butterflies * 1.5;
}

int commit_batch_enqueue(const glc_commit_job *jobs, uint32_t n_jobs, uint32_t n_streams, cudaStream_t stream) {
  for (uint32_t i = 0; i < n_jobs; i++) {
    const int e = commit_check(jobs[i]);
    if (e) return e;
  }
  if (!current_tables()) return fail("batch: glc_context_create has not been called on this device");
  if (n_jobs == 0) return 0;
  if (n_streams == 0) n_streams = 8;
  n_streams = std::min<uint32_t>(n_streams, std::min<uint32_t>(n_jobs, 32));
  StreamPool *pool = nullptr;
  int e = pool_get(n_streams, &pool);
  if (e) return e;
  std::lock_guard<std::mutex> lock(pool->mu);
  // largest first onto the least-loaded stream
  std::vector<uint32_t> order(n_jobs);
  std::iota(order.begin(), order.end(), 0);
  std::vector<double> cost(n_jobs);
  for (uint32_t i = 0; i < n_jobs; i++) cost[i] = job_cost(jobs[i]);
  std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return cost[a] > cost[b]; });
  std::vector<double> load(n_streams, 0.0);
  std::vector<std::vector<uint32_t>> assign(n_streams);
  for (uint32_t i : order) {
    const uint32_t s = (uint32_t)(std::min_element(load.begin(), load.end()) - load.begin());
    load[s] += cost[i];
    assign[s].push_back(i);
  }
  cudaError_t ce = cudaEventRecord(pool->fork, stream);
  if (ce != cudaSuccess) return (int)ce;
  for (uint32_t s = 0; s < n_streams; s++) {
    ce = cudaStreamWaitEvent(pool->streams[s], pool->fork, 0);
    if (ce != cudaSuccess) return (int)ce;
  }
  // enqueue round-robin over streams so that every stream starts its first (largest) job early
  size_t max_len = 0;
  for (auto &a : assign) max_len = std::max(max_len, a.size());
  for (size_t k = 0; k < max_len; k++)
    for (uint32_t s = 0; s < n_streams; s++)
      if (k < assign[s].size()) {
        e = commit_enqueue(jobs[assign[s][k]], pool->streams[s]);
        if (e) return e;
      }
  for (uint32_t s = 0; s < n_streams; s++) {
    ce = cudaEventRecord(pool->done[s], pool->streams[s]);
    if (ce != cudaSuccess) return (int)ce;
    ce = cudaStreamWaitEvent(stream, pool->done[s], 0);
    if (ce != cudaSuccess) return (int)ce;
  }
  return 0;
}

}  // namespace glc

using namespace glc;

struct glc_graph {
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  uint32_t n_jobs = 0;
};

extern "C" glc_status glc_commit_batch(const glc_commit_job *jobs, uint32_t n_jobs, uint32_t n_streams, void *stream) {
  if (!jobs && n_jobs) return fail("batch: null job array");
  return commit_batch_enqueue(jobs, n_jobs, n_streams, (cudaStream_t)stream);
}

extern "C" glc_status glc_commit_graph_create(const glc_commit_job *jobs, uint32_t n_jobs, uint32_t n_streams,
                                              glc_graph **out) {
  if (!out) return fail("graph: null output");
  *out = nullptr;
  if (!jobs && n_jobs) return fail("graph: null job array");
  cudaStream_t s;
  cudaError_t ce = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  if (ce != cudaSuccess) return (int)ce;
  glc_graph *g = new glc_graph();
  g->n_jobs = n_jobs;
  ce = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
  int e = (int)ce;
  if (!e) {
    e = commit_batch_enqueue(jobs, n_jobs, n_streams, s);
    cudaGraph_t graph = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(s, &graph);
    if (!e) e = (int)ee;
    g->graph = graph;
  }
  if (!e) e = (int)cudaGraphInstantiate(&g->exec, g->graph, 0);
  cudaStreamDestroy(s);
  if (e) {
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    delete g;
    return e;
  }
  *out = g;
  return 0;
}

extern "C" glc_status glc_commit_graph_launch(glc_graph *g, void *stream) {
  if (!g || !g->exec) return fail("graph: not instantiated");
  return (int)cudaGraphLaunch(g->exec, (cudaStream_t)stream);
}

extern "C" glc_status glc_commit_graph_destroy(glc_graph *g) {
  if (!g) return 0;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  delete g;
  return 0;
}
