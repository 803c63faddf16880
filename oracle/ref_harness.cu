// Host driver for the reference's OWN CUDA kernels (crates/boojum-cuda/native), compiled from
// the reference sources by oracle/build_ref.py into oracle/_ref/libbcref.so.
//
// TEST INFRASTRUCTURE ONLY: it lets the GPU tests check the oracle and the product kernels
// against the reference kernels on the same inputs, and lets the benchmark time the reference's
// per-call form on the same B200.  The reference's Rust host code cannot be built here (no
// Rust toolchain), so this file restates, in C++, what that host code does before each launch:
//   - Context::create: table contents and the __constant__ descriptors (src/context.rs:171-282)
//   - batch_ntt_internal: per-size kernel plans and launch shapes (src/ntt.rs:70-291)
//   - launch_bit_reverse (src/ops_complex.rs:273-306)
//   - select with get_launch_dims (src/ops_complex.rs:27-29, 446-463)
//   - compute_leaf_hashes / compute_node_hashes / build_merkle_tree / gathers, with the
//     st-or-mt kernel choice by wave count (src/poseidon2.rs:143-380)
// Round constants for the Poseidon2 kernels are compiled in from a generated header
// (build_ref.py fills the reference's template with the same constants the product uses).
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <vector>

struct RefLayer {
  const uint64_t *values;
  unsigned mask;
  unsigned log_count;
};
struct RefPowers {
  RefLayer fine, coarse;
};
struct RefPtrStride {
  const uint64_t *ptr;
  size_t stride;
};

// symbols defined by the reference's native/context.cu (extern "C" __constant__)
extern "C" __device__ __constant__ RefPowers powers_data_w;
extern "C" __device__ __constant__ RefPowers powers_data_w_bitrev_for_ntt;
extern "C" __device__ __constant__ RefPowers powers_data_w_inv_bitrev_for_ntt;
extern "C" __device__ __constant__ RefPowers powers_data_g_f;
extern "C" __device__ __constant__ RefPowers powers_data_g_i;
extern "C" __device__ __constant__ uint64_t inv_sizes[31];

#define NTT_ARGS                                                                                                  \
  const uint64_t *, uint64_t *, unsigned, unsigned, unsigned, unsigned, unsigned, bool, unsigned, unsigned, unsigned
extern "C" __global__ void n2b_1_stage(NTT_ARGS);
extern "C" __global__ void b2n_1_stage(NTT_ARGS);
extern "C" __global__ void n2b_final_7_stages_warp(NTT_ARGS);
extern "C" __global__ void n2b_final_8_stages_warp(NTT_ARGS);
extern "C" __global__ void n2b_final_9_to_12_stages_block(NTT_ARGS);
extern "C" __global__ void n2b_nonfinal_7_or_8_stages_block(NTT_ARGS);
extern "C" __global__ void b2n_initial_7_stages_warp(NTT_ARGS);
extern "C" __global__ void b2n_initial_8_stages_warp(NTT_ARGS);
extern "C" __global__ void b2n_initial_9_to_12_stages_block(NTT_ARGS);
extern "C" __global__ void b2n_noninitial_7_or_8_stages_block(NTT_ARGS);
extern "C" __global__ void bit_reverse_naive_kernel(RefPtrStride, RefPtrStride, unsigned);
extern "C" __global__ void bit_reverse_kernel(RefPtrStride, RefPtrStride, unsigned);
extern "C" __global__ void poseidon2_gl_st_leaves_kernel(const uint64_t *, uint64_t *, unsigned, unsigned, unsigned, bool,
                                                         bool);
extern "C" __global__ void poseidon2_gl_mt_leaves_kernel(const uint64_t *, uint64_t *, unsigned, unsigned, unsigned, bool,
                                                         bool);
extern "C" __global__ void poseidon2_gl_st_nodes_kernel(const uint64_t *, uint64_t *, unsigned);
extern "C" __global__ void poseidon2_gl_mt_nodes_kernel(const uint64_t *, uint64_t *, unsigned);
extern "C" __global__ void poseidon2_gl_gather_rows_kernel(const unsigned *, unsigned, RefPtrStride, RefPtrStride);
extern "C" __global__ void poseidon2_gl_gather_merkle_paths_kernel(const unsigned *, unsigned, const uint64_t *, unsigned,
                                                                   uint64_t *);
extern "C" __global__ void select_kernel(const unsigned *, const uint64_t *, uint64_t *, unsigned);

namespace {

constexpr uint64_t P = 0xFFFFFFFF00000001ull;
constexpr unsigned OMEGA_LOG_ORDER = 30;

uint64_t hmul(uint64_t a, uint64_t b) { return (uint64_t)(((unsigned __int128)a * b) % P); }
uint64_t hpow(uint64_t a, uint64_t e) {
  uint64_t r = 1;
  a %= P;
  while (e) {
    if (e & 1) r = hmul(r, a);
    a = hmul(a, a);
    e >>= 1;
  }
  return r;
}
uint64_t hinv(uint64_t a) { return hpow(a, P - 2); }
// domain generator of size 2^k: 7^((p-1)/2^k)
uint64_t root(unsigned log_size) { return hpow(7, (P - 1) >> log_size); }

std::vector<uint64_t *> g_allocs;

int upload_powers(uint64_t base, size_t count, bool bitrev, const uint64_t **out) {
  std::vector<uint64_t> h(count);
  uint64_t x = 1;
  for (size_t i = 0; i < count; i++, x = hmul(x, base)) h[i] = x;
  if (bitrev && count > 1) {
    unsigned bits = 0;
    while ((size_t(1) << bits) < count) bits++;
    for (size_t i = 0; i < count; i++) {
      size_t r = 0;
      for (unsigned b = 0; b < bits; b++) r |= ((i >> b) & 1) << (bits - 1 - b);
      if (r > i) std::swap(h[i], h[r]);
    }
  }
  uint64_t *d = nullptr;
  cudaError_t e = cudaMalloc(&d, count * 8);
  if (e) return e;
  g_allocs.push_back(d);
  e = cudaMemcpy(d, h.data(), count * 8, cudaMemcpyHostToDevice);
  *out = d;
  return e;
}

RefPowers make(const uint64_t *fine, unsigned fine_log, const uint64_t *coarse, unsigned coarse_log) {
  return RefPowers{{fine, (1u << fine_log) - 1, fine_log}, {coarse, (1u << coarse_log) - 1, coarse_log}};
}

enum Kern { N2B_F7, N2B_F8, N2B_F9_12, N2B_NF, B2N_I7, B2N_I8, B2N_I9_12, B2N_NI, NONE };
struct Step {
  Kern k;
  unsigned stages;
};
// Plans for log_n = 16..24 (src/ntt.rs:70-169), [n2b, b2n][log_n - 16][step]
const Step PLANS[2][9][3] = {
    {{{N2B_NF, 8}, {N2B_F8, 8}, {NONE, 0}},
     {{N2B_NF, 8}, {N2B_F9_12, 9}, {NONE, 0}},
     {{N2B_NF, 8}, {N2B_F9_12, 10}, {NONE, 0}},
     {{N2B_NF, 8}, {N2B_F9_12, 11}, {NONE, 0}},
     {{N2B_NF, 8}, {N2B_F9_12, 12}, {NONE, 0}},
     {{N2B_NF, 7}, {N2B_NF, 7}, {N2B_F7, 7}},
     {{N2B_NF, 7}, {N2B_NF, 7}, {N2B_F8, 8}},
     {{N2B_NF, 7}, {N2B_NF, 8}, {N2B_F8, 8}},
     {{N2B_NF, 8}, {N2B_NF, 8}, {N2B_F8, 8}}},
    {{{B2N_I8, 8}, {B2N_NI, 8}, {NONE, 0}},
     {{B2N_I9_12, 9}, {B2N_NI, 8}, {NONE, 0}},
     {{B2N_I9_12, 10}, {B2N_NI, 8}, {NONE, 0}},
     {{B2N_I9_12, 11}, {B2N_NI, 8}, {NONE, 0}},
     {{B2N_I9_12, 12}, {B2N_NI, 8}, {NONE, 0}},
     {{B2N_I7, 7}, {B2N_NI, 7}, {B2N_NI, 7}},
     {{B2N_I8, 8}, {B2N_NI, 7}, {B2N_NI, 7}},
     {{B2N_I8, 8}, {B2N_NI, 8}, {B2N_NI, 7}},
     {{B2N_I8, 8}, {B2N_NI, 8}, {B2N_NI, 8}}},
};

int waves_count(const void *fn, unsigned block, unsigned grid) {
  int dev = 0, mpc = 0, maxb = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&mpc, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&maxb, fn, (int)block, 0);
  if (maxb <= 0) maxb = 1;
  return (int)((grid - 1) / (unsigned)(mpc * maxb) + 1);
}

}  // namespace

extern "C" int ref_context_create(unsigned w_coarse_log, unsigned g_coarse_log) {
  if (w_coarse_log > OMEGA_LOG_ORDER || g_coarse_log > OMEGA_LOG_ORDER) return 1;
  const uint64_t *wf, *wc, *wfb, *wcb, *wifb, *wicb, *gff, *gfc, *gif, *gic;
  int e = 0;
  const unsigned cw = w_coarse_log, cg = g_coarse_log;
  const uint64_t w30 = root(OMEGA_LOG_ORDER);
  e = e ? e : upload_powers(w30, size_t(1) << (OMEGA_LOG_ORDER - cw), false, &wf);
  e = e ? e : upload_powers(root(cw), size_t(1) << cw, false, &wc);
  e = e ? e : upload_powers(w30, size_t(1) << (OMEGA_LOG_ORDER - cw - 1), true, &wfb);
  e = e ? e : upload_powers(root(cw + 1), size_t(1) << cw, true, &wcb);
  e = e ? e : upload_powers(hinv(w30), size_t(1) << (OMEGA_LOG_ORDER - cw - 1), true, &wifb);
  e = e ? e : upload_powers(hinv(root(cw + 1)), size_t(1) << cw, true, &wicb);
  const size_t gfine = size_t(1) << (OMEGA_LOG_ORDER - cg);
  e = e ? e : upload_powers(7, gfine, false, &gff);
  e = e ? e : upload_powers(hpow(7, gfine), size_t(1) << cg, false, &gfc);
  e = e ? e : upload_powers(hinv(7), gfine, false, &gif);
  e = e ? e : upload_powers(hpow(hinv(7), gfine), size_t(1) << cg, false, &gic);
  if (e) return e;
  RefPowers d;
  d = make(wf, OMEGA_LOG_ORDER - cw, wc, cw);
  e = e ? e : cudaMemcpyToSymbol(powers_data_w, &d, sizeof(d));
  d = make(wfb, OMEGA_LOG_ORDER - cw - 1, wcb, cw);
  e = e ? e : cudaMemcpyToSymbol(powers_data_w_bitrev_for_ntt, &d, sizeof(d));
  d = make(wifb, OMEGA_LOG_ORDER - cw - 1, wicb, cw);
  e = e ? e : cudaMemcpyToSymbol(powers_data_w_inv_bitrev_for_ntt, &d, sizeof(d));
  d = make(gff, OMEGA_LOG_ORDER - cg, gfc, cg);
  e = e ? e : cudaMemcpyToSymbol(powers_data_g_f, &d, sizeof(d));
  d = make(gif, OMEGA_LOG_ORDER - cg, gic, cg);
  e = e ? e : cudaMemcpyToSymbol(powers_data_g_i, &d, sizeof(d));
  uint64_t inv[31];
  uint64_t x = 1, half = hinv(2);
  for (int k = 0; k < 31; k++, x = hmul(x, half)) inv[k] = x;
  e = e ? e : cudaMemcpyToSymbol(inv_sizes, inv, sizeof(inv));
  return e ? e : (int)cudaDeviceSynchronize();
}

extern "C" int ref_context_destroy() {
  for (auto p : g_allocs) cudaFree(p);
  g_allocs.clear();
  return 0;
}

// batch_ntt_internal (src/ntt.rs:179-291)
extern "C" int ref_batch_ntt(const uint64_t *in, uint64_t *out, unsigned log_n, unsigned num_ntts, unsigned in_stride,
                             unsigned out_stride, bool bitrev_inputs, bool inverse, unsigned log_ext, unsigned coset,
                             cudaStream_t stream) {
  if (log_n < 1 || log_n + log_ext > OMEGA_LOG_ORDER || log_n > 24) return 1;
  const unsigned n = 1u << log_n;
  if (n > in_stride || n > out_stride) return 1;
  if (coset > 0 && (log_ext == 0 || coset >= (1u << log_ext))) return 1;
  if (log_n < 16) {
    const unsigned threads = 128;
    const unsigned blocks_per_ntt = (n + 2 * threads - 1) / (2 * threads);
    const unsigned blocks = blocks_per_ntt * num_ntts;
    for (unsigned stage = 0; stage < log_n; stage++) {
      const uint64_t *ip = stage == 0 ? in : out;
      const unsigned is = stage == 0 ? in_stride : out_stride;
      if (bitrev_inputs)
        b2n_1_stage<<<blocks, threads, 0, stream>>>(ip, out, is, out_stride, stage, 1, log_n, inverse, blocks_per_ntt,
                                                    log_ext, coset);
      else
        n2b_1_stage<<<blocks, threads, 0, stream>>>(ip, out, is, out_stride, stage, 1, log_n, inverse, blocks_per_ntt,
                                                    log_ext, coset);
    }
    return (int)cudaGetLastError();
  }
  const Step *plan = PLANS[bitrev_inputs ? 1 : 0][log_n - 16];
  unsigned stage = 0;
  const unsigned chunks = (num_ntts + 7) / 8;  // NTTS_PER_BLOCK (src/ntt.rs:174)
  for (int s = 0; s < 3 && plan[s].k != NONE; s++) {
    const uint64_t *ip = stage == 0 ? in : out;
    const unsigned is = stage == 0 ? in_stride : out_stride;
    const unsigned start = stage;
    stage += plan[s].stages;
    void (*fn)(NTT_ARGS) = nullptr;
    unsigned gx = 0, bx = 0;
    switch (plan[s].k) {
      case N2B_F7: fn = n2b_final_7_stages_warp; gx = n / (4 * 128); bx = 128; break;
      case N2B_F8: fn = n2b_final_8_stages_warp; gx = n / (4 * 256); bx = 128; break;
      case N2B_F9_12: fn = n2b_final_9_to_12_stages_block; gx = n / 4096; bx = 512; break;
      case N2B_NF: fn = n2b_nonfinal_7_or_8_stages_block; gx = n / 4096; bx = 512; break;
      case B2N_I7: fn = b2n_initial_7_stages_warp; gx = n / (4 * 128); bx = 128; break;
      case B2N_I8: fn = b2n_initial_8_stages_warp; gx = n / (4 * 256); bx = 128; break;
      case B2N_I9_12: fn = b2n_initial_9_to_12_stages_block; gx = n / 4096; bx = 512; break;
      case B2N_NI: fn = b2n_noninitial_7_or_8_stages_block; gx = n / 4096; bx = 512; break;
      default: return 1;
    }
    fn<<<dim3(gx, chunks), bx, 0, stream>>>(ip, out, is, out_stride, start, plan[s].stages, log_n, inverse, num_ntts,
                                             log_ext, coset);
    const int e = (int)cudaGetLastError();
    if (e) return e;
  }
  return stage == log_n ? 0 : 1;
}

// launch_bit_reverse (src/ops_complex.rs:273-306)
extern "C" int ref_bit_reverse(const uint64_t *src, size_t src_stride, uint64_t *dst, size_t dst_stride, unsigned log_rows,
                               unsigned cols, cudaStream_t stream) {
  const RefPtrStride s{src, src_stride}, d{dst, dst_stride};
  const unsigned half = log_rows >> 1;
  if (half < 5) {
    const unsigned n = 1u << log_rows;
    const unsigned block = n < 128 ? n : 128;  // get_launch_dims: 128 threads per block
    bit_reverse_naive_kernel<<<dim3((n + block - 1) / block, cols), block, 0, stream>>>(s, d, log_rows);
  } else {
    const unsigned tiles = 1u << (half - 5);
    const unsigned gx = tiles * (tiles + 1) / 2, gy = log_rows - (half << 1) + 1;
    bit_reverse_kernel<<<dim3(gx, gy, cols), dim3(32, 2, 2), 0, stream>>>(s, d, log_rows);
  }
  return (int)cudaGetLastError();
}

// select_function_and_grid_block_dims (src/poseidon2.rs:143-158)
static void select_dims(const void *mt, unsigned count, bool &use_mt, dim3 &grid, dim3 &block) {
  unsigned bx = count < 32 ? count : 32;
  unsigned gx = (count + bx - 1) / bx;
  if (waves_count(mt, 32 * 3, gx) > 1) {
    use_mt = false;
    bx = count < 128 ? count : 128;
    grid = dim3((count + bx - 1) / bx);
    block = dim3(bx);
  } else {
    use_mt = true;
    grid = dim3(gx);
    block = dim3(bx, 3);
  }
}

// compute_leaf_hashes (src/poseidon2.rs:180-226)
extern "C" int ref_p2_leaves(const uint64_t *values, size_t values_len, uint64_t *results, size_t results_len,
                             unsigned log_rows_per_hash, bool load_int, bool store_int, cudaStream_t stream) {
  if (results_len % 4) return 1;
  const size_t count = results_len / 4;
  if (count == 0 || values_len % (count << log_rows_per_hash)) return 1;
  const size_t rows = size_t(1) << log_rows_per_hash, cols = values_len / (count << log_rows_per_hash);
  if (store_int && (rows * cols) % 8) return 1;
  bool mt;
  dim3 g, b;
  select_dims((const void *)poseidon2_gl_mt_leaves_kernel, (unsigned)count, mt, g, b);
  if (mt)
    poseidon2_gl_mt_leaves_kernel<<<g, b, 0, stream>>>(values, results, (unsigned)rows, (unsigned)cols, (unsigned)count,
                                                       load_int, store_int);
  else
    poseidon2_gl_st_leaves_kernel<<<g, b, 0, stream>>>(values, results, (unsigned)rows, (unsigned)cols, (unsigned)count,
                                                       load_int, store_int);
  return (int)cudaGetLastError();
}

// compute_node_hashes (src/poseidon2.rs:228-251)
extern "C" int ref_p2_nodes(const uint64_t *values, size_t values_len, uint64_t *results, size_t results_len,
                            cudaStream_t stream) {
  if (values_len % 8 || results_len % 4 || values_len != 2 * results_len) return 1;
  const unsigned count = (unsigned)(results_len / 4);
  if (count == 0) return 0;
  bool mt;
  dim3 g, b;
  select_dims((const void *)poseidon2_gl_mt_nodes_kernel, count, mt, g, b);
  if (mt)
    poseidon2_gl_mt_nodes_kernel<<<g, b, 0, stream>>>(values, results, count);
  else
    poseidon2_gl_st_nodes_kernel<<<g, b, 0, stream>>>(values, results, count);
  return (int)cudaGetLastError();
}

// build_merkle_tree (src/poseidon2.rs:297-314): leaves, then one node launch per layer
extern "C" int ref_p2_build_merkle_tree(const uint64_t *values, size_t values_len, uint64_t *results,
                                        size_t results_len, unsigned log_rows_per_hash, unsigned layers_count,
                                        cudaStream_t stream) {
  if (layers_count == 0 || results_len % 8) return 1;
  const size_t leaves = results_len / 8;
  if ((size_t(1) << (layers_count - 1)) > leaves || values_len % leaves) return 1;
  size_t half = results_len / 2;
  int e = ref_p2_leaves(values, values_len, results, half, log_rows_per_hash, false, false, stream);
  const uint64_t *layer = results;
  uint64_t *rest = results + half;
  size_t len = half;
  for (unsigned l = 1; l < layers_count && !e; l++) {
    e = ref_p2_nodes(layer, len, rest, len / 2, stream);
    layer = rest;
    rest += len / 2;
    len /= 2;
  }
  return e;
}

// gather_rows (src/poseidon2.rs:316-348)
extern "C" int ref_p2_gather_rows(const unsigned *indexes, unsigned indexes_count, unsigned log_rows_per_index,
                                  const uint64_t *values, size_t values_stride, uint64_t *results, size_t results_stride,
                                  unsigned cols, cudaStream_t stream) {
  const unsigned rows_per_index = 1u << log_rows_per_index;
  const unsigned per_block = 32u >> log_rows_per_index;
  const unsigned by = indexes_count < per_block ? indexes_count : per_block;
  if (by == 0) return 0;
  const unsigned gx = (indexes_count + by - 1) / by;
  poseidon2_gl_gather_rows_kernel<<<dim3(gx, cols), dim3(rows_per_index, by), 0, stream>>>(
      indexes, indexes_count, RefPtrStride{values, values_stride}, RefPtrStride{results, results_stride});
  return (int)cudaGetLastError();
}

// gather_merkle_paths (src/poseidon2.rs:350-380)
extern "C" int ref_p2_gather_merkle_paths(const unsigned *indexes, unsigned indexes_count, const uint64_t *values,
                                          size_t values_len, uint64_t *results, unsigned layers_count,
                                          cudaStream_t stream) {
  const size_t vc = values_len / 4;
  unsigned log_vc = 0;
  while ((size_t(1) << log_vc) < vc) log_vc++;
  const unsigned log_leaves = log_vc - 1;
  const unsigned bx = indexes_count < 32 ? indexes_count : 32;
  if (bx == 0 || layers_count == 0) return 0;
  poseidon2_gl_gather_merkle_paths_kernel<<<dim3((indexes_count + bx - 1) / bx, 4, layers_count), bx, 0, stream>>>(
      indexes, indexes_count, values, log_leaves, results);
  return (int)cudaGetLastError();
}

// ops_complex::select (src/ops_complex.rs:446-463): one thread per index, get_launch_dims = 128
// threads per block (WARP_SIZE * 4, ops_complex.rs:27-29).
extern "C" int ref_select(const unsigned *indexes, const uint64_t *src, uint64_t *dst, unsigned count,
                          cudaStream_t stream) {
  if (count == 0) return 0;
  const unsigned block = count < 128 ? count : 128;
  select_kernel<<<(count + block - 1) / block, block, 0, stream>>>(indexes, src, dst, count);
  return (int)cudaGetLastError();
}
