// Per-device twiddle / power tables and error plumbing.
//
// Replaces boojum-cuda's Context (crates/boojum-cuda/src/context.rs:157-297,
// native/context.{cu,cuh}).  The reference splits every power table into fine x coarse parts
// held in __constant__ descriptors; here the hot NTT twiddles are one flat bit-reversed table in
// HBM (the prefix an NTT of size N touches, N/2 entries, stays in the 126 MB L2), and only the
// coset shifts use two-level tables.
#include <atomic>
#include <vector>

#include "glc_field.cuh"
#include "glc_internal.h"

namespace glc {

static thread_local std::string g_last_error;
static std::atomic<uint64_t> g_launches{0};

void count_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
uint64_t launches_issued() { return g_launches.load(std::memory_order_relaxed); }
static DeviceTables g_tables[MAX_DEVICES];
static std::mutex g_tables_mutex;

void set_error(const std::string &msg) { g_last_error = msg; }

int fail(const std::string &msg) {
  set_error(msg);
  return (int)cudaErrorInvalidValue;
}

const DeviceTables *current_tables() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) return nullptr;
  return g_tables[dev].ready ? &g_tables[dev] : nullptr;
}

static __device__ __forceinline__ uint32_t brev_bits(uint32_t x, uint32_t bits) { return __brev(x) >> (32 - bits); }

// T[x] = w_{2^30}^(bitrev_23(x) << 6) = w_{2^24}^bitrev_23(x); inverse uses w^-1.
__global__ void build_twiddles_kernel(uint64_t *tw_fwd, uint64_t *tw_inv, const uint64_t *w_lo, const uint64_t *w_hi,
                                      uint32_t count) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= count) return;
  const uint32_t y = brev_bits(x, MAX_LOG_N - 1) << (OMEGA_LOG_ORDER - MAX_LOG_N);
  const uint32_t yi = ((1u << OMEGA_LOG_ORDER) - y) & ((1u << OMEGA_LOG_ORDER) - 1);
  tw_fwd[x] = canon(mul(w_lo[y & 32767], w_hi[y >> 15]));
  tw_inv[x] = canon(mul(w_lo[yi & 32767], w_hi[yi >> 15]));
}

static void free_tables(DeviceTables &t) {
  uint64_t **ptrs[] = {&t.tw_fwd, &t.tw_inv, &t.g_lo, &t.g_hi, &t.gi_lo, &t.gi_hi, &t.w_lo, &t.w_hi};
  for (auto p : ptrs) {
    if (*p) cudaFree(*p);
    *p = nullptr;
  }
  t.ready = false;
}

static std::vector<uint64_t> powers(uint64_t base, size_t count) {
  std::vector<uint64_t> v(count);
  uint64_t x = 1;
  for (size_t i = 0; i < count; i++, x = h_mul(x, base)) v[i] = x;
  return v;
}

}  // namespace glc

using namespace glc;

extern "C" const char *glc_last_error_message(void) { return g_last_error.c_str(); }

extern "C" uint64_t glc_launch_count(void) { return launches_issued(); }

extern "C" glc_status glc_context_create(uint32_t powers_of_w_coarse_log_count, uint32_t powers_of_g_coarse_log_count) {
  // context.rs:175-176
  if (powers_of_w_coarse_log_count > OMEGA_LOG_ORDER || powers_of_g_coarse_log_count > OMEGA_LOG_ORDER)
    return fail("glc_context_create: coarse log counts must be <= 30");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  if (dev < 0 || dev >= MAX_DEVICES) return fail("glc_context_create: device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_tables_mutex);
  DeviceTables &t = g_tables[dev];
  free_tables(t);
  const size_t tw_count = size_t(1) << (MAX_LOG_N - 1);
  auto alloc = [&](uint64_t **p, size_t n) { return e == cudaSuccess ? (e = cudaMalloc(p, n * sizeof(uint64_t))) : e; };
  alloc(&t.tw_fwd, tw_count);
  alloc(&t.tw_inv, tw_count);
  alloc(&t.g_lo, 4096);
  alloc(&t.g_hi, 4096);
  alloc(&t.gi_lo, 4096);
  alloc(&t.gi_hi, 4096);
  alloc(&t.w_lo, 32768);
  alloc(&t.w_hi, 32768);
  if (e != cudaSuccess) {
    free_tables(t);
    return (int)e;
  }
  const uint64_t g = GENERATOR, gi = h_inv(GENERATOR);
  const uint64_t w = h_root_of_unity(OMEGA_LOG_ORDER);
  auto up = [&](uint64_t *dst, const std::vector<uint64_t> &src) {
    if (e == cudaSuccess) e = cudaMemcpy(dst, src.data(), src.size() * sizeof(uint64_t), cudaMemcpyHostToDevice);
  };
  up(t.g_lo, powers(g, 4096));
  up(t.g_hi, powers(h_pow(g, 4096), 4096));
  up(t.gi_lo, powers(gi, 4096));
  up(t.gi_hi, powers(h_pow(gi, 4096), 4096));
  up(t.w_lo, powers(w, 32768));
  up(t.w_hi, powers(h_pow(w, 32768), 32768));
  if (e == cudaSuccess) {
    build_twiddles_kernel<<<(unsigned)((tw_count + 255) / 256), 256>>>(t.tw_fwd, t.tw_inv, t.w_lo, t.w_hi,
                                                                       (uint32_t)tw_count);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  if (e == cudaSuccess) e = (cudaError_t)ntt_init_device();
  if (e != cudaSuccess) {
    free_tables(t);
    return (int)e;
  }
  const uint64_t two_inv = h_inv(2);
  uint64_t x = 1;
  for (uint32_t k = 0; k <= OMEGA_LOG_ORDER; k++, x = h_mul(x, two_inv)) t.inv_sizes[k] = x;
  t.w_coarse_log = powers_of_w_coarse_log_count;
  t.g_coarse_log = powers_of_g_coarse_log_count;
  t.ready = true;
  set_error("");
  return 0;
}

extern "C" glc_status glc_context_destroy(void) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return (int)e;
  if (dev < 0 || dev >= MAX_DEVICES) return fail("glc_context_destroy: device ordinal out of range");
  std::lock_guard<std::mutex> lock(g_tables_mutex);
  // cudaFree synchronises the device, so no kernel still reads the tables
  free_tables(g_tables[dev]);
  noalloc_forget_device(dev);
  fused_forget_device(dev);
  return 0;
}
