// Commitment cap without any device allocation.
//
// Some callers cannot call cudaMalloc, or must not: a custom device allocator or an allocation
// callback that needs a commitment while it is itself serving an allocation (re-entering the
// allocator would deadlock or recurse), a plugin whose host framework owns all device memory
// through its own pool and forbids side allocations, or a process whose device memory is
// already reserved by another framework, so that a fresh cudaMalloc fails or forces a
// synchronising trim of that framework's cache.  glc_commit needs the caller to pass the LDE and
// tree buffers; glc_commit_cap_noalloc keeps them in a fixed array compiled into this library
// instead and returns only the cap.
//
// The array is 2^24 elements (128 MiB) and every GPU that loads the library holds it until the
// process exits.  A job fits when 2^log_lde * (cols + 8) * 2^log_n <= 2^24 (the LDE cosets plus
// the Merkle subtrees); larger jobs are rejected with an error message, never truncated.
//
// All calls share the array and it keeps the last call's contents.  Nothing in it has to start
// at zero: every element a job reads was written earlier in the same job (NTT outputs, leaf
// digests, node digests).  Two calls whose work overlaps on the GPU race on it (different
// streams, or different host threads, without an order between them); calls on one stream, or
// ordered by events, are safe.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "glc_internal.h"

namespace glc {

static constexpr uint64_t NOALLOC_ELEMS = 1ull << 24;

// Scratch for the LDE cosets and the subtrees of one job.  In host code this name is only a
// stand-in for the symbol, not a device address: host code passes the address obtained from
// cudaGetSymbolAddress below.
static __device__ __align__(256) uint64_t g_noalloc_scratch[NOALLOC_ELEMS];

static uint64_t *g_noalloc_ptr[MAX_DEVICES] = {};
static std::mutex g_noalloc_mu;

// Forgets the device address looked up on `dev`.  glc_context_destroy calls it: after a device
// reset (cudaDeviceReset) the caller has to create the context again, and the next call then
// looks the address up again instead of using one from the old context.
void noalloc_forget_device(int dev) {
  if (dev < 0 || dev >= MAX_DEVICES) return;
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  g_noalloc_ptr[dev] = nullptr;
}

// Device address of the array on the current device, looked up once per device (on the first
// call there after glc_context_create) with that device current.
static int noalloc_scratch(uint64_t **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  if (dev < 0 || dev >= MAX_DEVICES) return fail("commit_cap_noalloc: device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return (int)e;
    g_noalloc_ptr[dev] = static_cast<uint64_t *>(p);
  }
  *out = g_noalloc_ptr[dev];
  return 0;
}

}  // namespace glc

using namespace glc;

extern "C" glc_status glc_commit_cap_noalloc(const uint64_t *evals, uint64_t evals_stride, uint32_t log_n,
                                             uint32_t cols, uint32_t log_lde, uint32_t log_cap, uint64_t *cap,
                                             void *stream) {
  glc_commit_job j{};
  j.evals = evals;
  j.evals_stride = evals_stride;
  j.log_n = log_n;
  j.cols = cols;
  j.log_lde = log_lde;
  j.log_cap = log_cap;
  j.cap = cap;
  // placeholders so that commit_check validates the shape; replaced by the array below
  j.lde = j.trees = cap;
  int e = commit_check(j);
  if (e) return e;
  const uint64_t n = 1ull << log_n, f = 1ull << log_lde;
  const uint64_t need = f * ((uint64_t)cols + 8) * n;
  if (need > NOALLOC_ELEMS)
    return fail("commit_cap_noalloc: job needs " + std::to_string(need) +
                " scratch elements (2^log_lde * (cols + 8) * 2^log_n); the maximum is 2^24");
  if (!current_tables()) return fail("commit_cap_noalloc: glc_context_create has not been called on this device");
  uint64_t *scratch = nullptr;
  if ((e = noalloc_scratch(&scratch))) return e;
  j.lde = scratch;                              // f cosets x cols x 2^log_n
  j.trees = scratch + f * (uint64_t)cols * n;   // f subtrees x 8 x 2^log_n
  j.monomials = nullptr;                        // kept in the last coset's LDE slot
  return commit_enqueue(j, (cudaStream_t)stream, nullptr, false);
}
