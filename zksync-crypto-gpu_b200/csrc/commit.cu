// Commitment jobs: evaluations -> monomials -> coset LDE -> Poseidon2 Merkle subtrees -> cap.
//
// This is the sequence shivini runs around boojum-cuda for one commitment
// (crates/shivini/src/data_structures/storage.rs:155-330, cache.rs:353-418, oracle.rs:62-88):
//   monomials = bitreverse(iNTT_n2b(evaluations))                  (storage.rs:155-192)
//   coset c of f: lde[c] = NTT_n2b(monomials, log_ext, bitrev(c))  (primitives/ntt.rs:25)
//   subtree per coset with cap/f entries, caps concatenated coset by coset.
//
// glc_commit issues it for one job on one stream (the plain per-call form).  glc_commit_batch
// runs many jobs at once: the jobs are spread over a pool of streams so that the memory-bound
// NTT passes of one job overlap the integer-bound hashing of another, and the whole batch can
// be captured into a CUDA graph and replayed (glc_commit_graph_*).
#include <algorithm>
#include <mutex>
#include <vector>

#include "glc_field.cuh"
#include "glc_internal.h"

namespace glc {

// cap[j*cap + c*ccap + m] = tree_c[cap_off + j*ccap + m]
__global__ void gather_caps_kernel(const uint64_t *trees, uint64_t tree_len, uint64_t cap_off, uint32_t ccap,
                                   uint32_t cosets, uint64_t *cap) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t total = 4 * ccap * cosets;
  if (t >= total) return;
  const uint32_t m = t % ccap, c = (t / ccap) % cosets, j = t / (ccap * cosets);
  cap[(uint64_t)j * ccap * cosets + (uint64_t)c * ccap + m] = trees[c * tree_len + cap_off + (uint64_t)j * ccap + m];
}

int commit_check(const glc_commit_job &j) {
  if (j.log_n < 1 || j.log_n > MAX_LOG_N) return fail("commit: log_n must be in 1..24");
  if (j.log_lde > 4 || j.log_n + j.log_lde > OMEGA_LOG_ORDER) return fail("commit: log_lde must be in 0..4");
  if (j.log_cap < j.log_lde) return fail("commit: the cap must have at least one entry per coset");
  if (j.log_cap - j.log_lde > j.log_n) return fail("commit: cap per coset larger than the coset");
  if (j.cols == 0) return fail("commit: no columns");
  if (j.evals_stride < (1ull << j.log_n)) return fail("commit: evals_stride < 2^log_n");
  if (!j.evals || !j.lde || !j.trees || !j.cap) return fail("commit: null buffer");
  return 0;
}

static uint32_t brev_bits(uint32_t x, uint32_t bits) {
  uint32_t r = 0;
  for (uint32_t i = 0; i < bits; i++) r |= ((x >> i) & 1u) << (bits - 1 - i);
  return r;
}

// Streams that let the cosets of one commitment run side by side: the memory- and ALU-heavy NTT
// of coset c+1 fills the issue slots the leaf hashing of coset c leaves idle.
struct CosetStreams {
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> joins;
  std::vector<cudaEvent_t> ntt_done;  // coset c's NTT has read the monomials (c < f - 1)
  cudaEvent_t fork = nullptr;
  std::mutex mu;
};
static CosetStreams g_coset_streams[MAX_DEVICES];

static int coset_streams_get(uint32_t n, CosetStreams **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  if (dev < 0 || dev >= MAX_DEVICES) return fail("commit: device ordinal out of range");
  CosetStreams &c = g_coset_streams[dev];
  if (!c.fork && (e = cudaEventCreateWithFlags(&c.fork, cudaEventDisableTiming)) != cudaSuccess) return (int)e;
  while (c.streams.size() < n) {
    cudaStream_t st;
    cudaEvent_t ev, nd;
    if ((e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking)) != cudaSuccess) return (int)e;
    if ((e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming)) != cudaSuccess) return (int)e;
    if ((e = cudaEventCreateWithFlags(&nd, cudaEventDisableTiming)) != cudaSuccess) return (int)e;
    c.streams.push_back(st);
    c.joins.push_back(ev);
    c.ntt_done.push_back(nd);
  }
  *out = &c;
  return 0;
}

int commit_enqueue(const glc_commit_job &j, cudaStream_t stream, cudaEvent_t *events, bool coset_parallel) {
  uint32_t ev = 0;
  cudaStream_t cur = stream;
  auto mark = [&]() -> int { return events ? (int)cudaEventRecord(events[ev++], cur) : 0; };
  const uint64_t n = 1ull << j.log_n;
  const uint32_t f = 1u << j.log_lde;
  const uint64_t coset_elems = n * j.cols;
  // monomials: the caller's buffer, or the last coset's LDE buffer (transformed last, in place)
  uint64_t *mono = j.monomials ? j.monomials : j.lde + (uint64_t)(f - 1) * coset_elems;
  int e = mark();
  if (e) return e;
  e = ntt_launch(j.evals, mono, j.log_n, j.cols, j.evals_stride, n, false, true, 0, 0, stream, 0);
  if (e) return e;
  e = bitrev_launch(mono, n, mono, n, j.log_n, j.cols, stream);
  if (!e) e = mark();
  if (e) return e;
  const uint32_t log_ccap = j.log_cap - j.log_lde;
  const uint32_t layers = j.log_n - log_ccap + 1;
  CosetStreams *cs = nullptr;
  std::unique_lock<std::mutex> cs_lock;
  if (coset_parallel && f > 1) {
    e = coset_streams_get(f - 1, &cs);
    if (e) return e;
    cs_lock = std::unique_lock<std::mutex>(cs->mu);
    if ((e = (int)cudaEventRecord(cs->fork, stream))) return e;
  }
  for (uint32_t c = 0; c < f; c++) {
    if (cs && c > 0) {
      cur = cs->streams[c - 1];
      if ((e = (int)cudaStreamWaitEvent(cur, cs->fork, 0))) return e;
    }
    if ((e = mark())) return e;  // coset start (on the stream that runs this coset)
    uint64_t *dst = j.lde + (uint64_t)c * coset_elems;
    const uint32_t coset = brev_bits(c, j.log_lde);
    // Without a monomials buffer the last coset transforms the monomials in place: on parallel
    // streams it must wait until every other coset's NTT has read them.
    const bool mono_in_lde = !j.monomials;
    if (cs && mono_in_lde && c == f - 1)
      for (uint32_t d = 0; d + 1 < f; d++)
        if ((e = (int)cudaStreamWaitEvent(cur, cs->ntt_done[d], 0))) return e;
    e = ntt_launch(mono, dst, j.log_n, j.cols, n, n, false, false, j.log_lde, coset, cur, 0);
    if (!e && cs && mono_in_lde && c + 1 < f) e = (int)cudaEventRecord(cs->ntt_done[c], cur);
    if (!e) e = mark();
    if (e) return e;
    uint64_t *tree = j.trees + (uint64_t)c * 8 * n;
    e = p2_leaves_launch(dst, tree, 0, j.cols, n, false, false, cur);
    if (!e) e = mark();
    if (e) return e;
    if (layers > 1) {
      e = p2_tree_nodes_launch(tree, n, layers - 1, cur);
      if (e) return e;
    }
    e = mark();
    if (e) return e;
    if (cs && c > 0) {
      if ((e = (int)cudaEventRecord(cs->joins[c - 1], cur))) return e;
      if ((e = (int)cudaStreamWaitEvent(stream, cs->joins[c - 1], 0))) return e;
    }
  }
  cur = stream;
  const uint32_t ccap = 1u << log_ccap;
  const uint32_t total = 4 * ccap * f;
  gather_caps_kernel<<<(total + 127) / 128, 128, 0, stream>>>(j.trees, 8 * n, 8 * n - 8ull * ccap, ccap, f, j.cap);
  e = last_launch_error();
  if (!e) e = mark();
  return e;
}

}  // namespace glc

using namespace glc;

extern "C" glc_status glc_commit_profiled(const glc_commit_job *job, void *stream, void **events, uint32_t n_events) {
  if (!job || !events) return fail("commit: null job or events");
  int e = commit_check(*job);
  if (e) return e;
  if (n_events < 3 + 4 * (1u << job->log_lde)) return fail("commit: need 3 + 4 * 2^log_lde events");
  if (!current_tables()) return fail("commit: glc_context_create has not been called on this device");
  return commit_enqueue(*job, (cudaStream_t)stream, reinterpret_cast<cudaEvent_t *>(events), true);
}

extern "C" glc_status glc_commit(const glc_commit_job *job, void *stream) {
  if (!job) return fail("commit: null job");
  int e = commit_check(*job);
  if (e) return e;
  if (!current_tables()) return fail("commit: glc_context_create has not been called on this device");
  return commit_enqueue(*job, (cudaStream_t)stream, nullptr, true);
}
