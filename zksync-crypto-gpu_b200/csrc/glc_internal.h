// Internal declarations shared by the translation units of libglc (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <functional>
#include <mutex>
#include <string>

#include "../../include/glc.h"

namespace glc {

// Largest NTT size the twiddle table covers (the reference plans stop at 2^24, ntt.rs:70-169).
static constexpr uint32_t MAX_LOG_N = 24;
// Roots of unity are powers of w_{2^30} (OMEGA_LOG_ORDER, crates/boojum-cuda/native/context.cuh:9).
static constexpr uint32_t OMEGA_LOG_ORDER = 30;
static constexpr int MAX_DEVICES = 64;

// Device-resident tables of one GPU (the reference keeps the same data in five __constant__
// descriptors plus device arrays, crates/boojum-cuda/native/context.cu:3-8).
struct DeviceTables {
  bool ready = false;
  uint32_t w_coarse_log = 0, g_coarse_log = 0;  // as passed by the caller (kept for reporting)
  // Flat bit-reversed twiddles T[x] = w_{2^24}^{bitrev_23(x)}, x < 2^23 (forward) and the same for w^-1.
  uint64_t *tw_fwd = nullptr, *tw_inv = nullptr;
  // Two-level power tables: g^j = g_lo[j & 4095] * g_hi[j >> 12] (j < 2^24), same for g^-1;
  // w_{2^30}^y = w_lo[y & 32767] * w_hi[y >> 15] (y < 2^30).
  uint64_t *g_lo = nullptr, *g_hi = nullptr, *gi_lo = nullptr, *gi_hi = nullptr;
  uint64_t *w_lo = nullptr, *w_hi = nullptr;
  uint64_t inv_sizes[OMEGA_LOG_ORDER + 1] = {};
};

// Tables of the current device, or nullptr when glc_context_create has not run on it.
const DeviceTables *current_tables();

// Thread-local message for the last contract violation.
void set_error(const std::string &msg);
int fail(const std::string &msg);  // set_error + return cudaErrorInvalidValue

// Kernel launches issued by this library (process-wide), for benchmark accounting.
void count_launches(uint64_t n);
uint64_t launches_issued();
// Called once after each kernel launch: counts it and returns the launch status.
inline int last_launch_error() {
  count_launches(1);
  return (int)cudaGetLastError();
}

// Launch choices of the NTT for one size (set by the autotuner, per device and log_n).
struct NttTuning {
  uint32_t radix_bits = 3;        // stages per register round: 2, 3 or 4
  uint32_t k1 = 0;                // stages in the strided pass of a two-pass plan (0: log_n / 2)
  uint32_t max_log_w = 5;         // at most 2^max_log_w contiguous elements per tile row
  uint32_t max_cols_per_cta = 8;  // columns one CTA walks with the same twiddles
  uint32_t l2_chunk_mb = 0;       // columns per L2-resident chunk of a two-pass NTT (0: all columns)
};
NttTuning &ntt_tuning(uint32_t log_n);

// Launch choices of the Poseidon2 leaf kernel (set by the autotuner, per device).
struct P2Tuning {
  uint32_t leaf_threads = 128;  // 64, 128 or 256
  uint32_t rolled = 2;          // 0: every round unrolled; 1: partial rounds in a loop; 2: all rounds in loops
  bool lazy = true;             // partial rounds keep s1..s11 partially reduced
  uint32_t min_blocks = 2;      // leaf kernel register cap: 2 -> 128, 3 -> 85, 5 -> 102 registers (<= 128 threads)
};
P2Tuning &p2_tuning();

// Round constants: installs rc (30*12 values) on the current device.
int p2_install_round_constants(const uint64_t *rc);
bool p2_constants_installed();

// Internal launchers reused by the commitment pipeline (all enqueue on `stream`).
int ntt_launch(const uint64_t *in, uint64_t *out, uint32_t log_n, uint32_t num_ntts, uint64_t in_stride,
               uint64_t out_stride, bool bitrev_inputs, bool inverse, uint32_t log_ext, uint32_t coset_idx,
               cudaStream_t stream, uint32_t l2_chunk_cols);
int bitrev_launch(const uint64_t *src, uint64_t src_stride, uint64_t *dst, uint64_t dst_stride, uint32_t log_rows,
                  uint32_t cols, cudaStream_t stream);
int p2_leaves_launch(const uint64_t *values, uint64_t *results, uint32_t rows, uint64_t cols, uint64_t count,
                     bool load_intermediate, bool store_intermediate, cudaStream_t stream);
int p2_nodes_launch(const uint64_t *values, uint64_t *results, uint64_t count, cudaStream_t stream);
// Node layers of a tree whose leaf layer ([4][leaves]) starts at `layer0`; writes layers 1..layers
// into the following part of the same buffer (reference layout, poseidon2.rs:276-314).
int p2_tree_nodes_launch(uint64_t *layer0, uint64_t leaves, uint32_t layers, cudaStream_t stream);

int ntt_init_device();  // kernel attributes; called by glc_context_create
void noalloc_forget_device(int dev);  // drops the cached scratch address; called by glc_context_destroy
void fused_forget_device(int dev);    // releases the fused batch's work-table pool; called by glc_context_destroy
double job_cost(const glc_commit_job &j);
int commit_check(const glc_commit_job &j);
// Enqueues one job; when `events` is given, records events[0] before the first stage, one after
// the monomials, then per coset {start, after NTT, after leaves, after nodes} on the stream that
// runs the coset, then one after the cap gather (3 + 4 * 2^log_lde events).
// coset_parallel: run the cosets on internal streams forked from `stream` (one call); the batch
// and serving runtimes pass false because they already spread jobs over streams.
int commit_enqueue(const glc_commit_job &j, cudaStream_t stream, cudaEvent_t *events = nullptr,
                   bool coset_parallel = false);

}  // namespace glc
