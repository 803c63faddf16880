/*
 * glc.h -- C ABI of libglc: Goldilocks NTT / coset LDE and Poseidon2 Merkle trees on B200 (sm_100a).
 *
 * Each entry point replaces one function of boojum-cuda's Rust API (matter-labs/zksync-crypto-gpu,
 * crates/boojum-cuda) and keeps its argument meaning, memory layout and checks, so that a caller
 * such as shivini can bind it as a drop-in.
 *
 * Conventions (as in the reference, crates/boojum-cuda/src/{ntt,poseidon2,context}.rs):
 *   - All buffers are device memory owned by the caller; field elements are uint64_t in [0, 2^64),
 *     not necessarily canonical (outputs of this library are canonical).
 *   - Every call enqueues work on `stream` (a cudaStream_t; NULL = legacy default stream) and
 *     returns without synchronising.
 *   - The return value is a cudaError_t value: 0 on success.  Where the reference panics through
 *     assert! on a contract violation, this library returns cudaErrorInvalidValue (1) without
 *     launching anything, and glc_last_error_message() describes the violated condition.
 *   - Column-major matrices: column k starts at base + k * stride.
 */
#ifndef GLC_H
#define GLC_H

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int glc_status;

/* Message of the last contract violation seen by the calling thread ("" if none). */
const char *glc_last_error_message(void);

/* ---------------------------------------------------------------------------------------------
 * Context: twiddle and power tables of the current device.
 * Replaces context::Context::create (crates/boojum-cuda/src/context.rs:171-282).  The coarse
 * log counts are validated as in the reference (<= 30) and recorded; the B200 layout keeps a
 * flat bit-reversed twiddle table for sizes up to 2^24 in HBM (128 MiB) plus two-level power
 * tables for the coset shifts.  Like the reference's __constant__ descriptors, the context is
 * one per device; creating it again replaces it.  Not thread-safe (same as the reference).
 */
glc_status glc_context_create(uint32_t powers_of_w_coarse_log_count, uint32_t powers_of_g_coarse_log_count);
/* Replaces context::Context::destroy (context.rs:284-296). */
glc_status glc_context_destroy(void);

/* ---------------------------------------------------------------------------------------------
 * Batched NTT / coset LDE (crates/boojum-cuda/src/ntt.rs).
 * num_ntts columns of 2^log_n elements; column k of the input starts at
 * inputs_matrix + inputs_offset + k * stride_between_input_arrays (same for outputs).
 * bitrev_inputs = false: natural-order input, bit-reversed output ("n2b");
 * bitrev_inputs = true: bit-reversed input, natural-order output ("b2n").
 * inverse: inverse transform including the 1/N factor.
 * log_extension_degree > 0 selects the coset s = 7 * w_{2^(log_n+log_extension_degree)}^coset_index:
 * forward multiplies coefficient j by s^j before the transform, inverse by s^-j after it.
 * Sizes: 1 <= log_n <= 24, log_n + log_extension_degree <= 30.
 */
/* Replaces ntt::batch_ntt_out_of_place (ntt.rs:294-335); inputs_len/outputs_len are the slice
 * lengths in elements; the two matrices must differ (ntt.rs:317,320). */
glc_status glc_batch_ntt_out_of_place(const uint64_t *inputs_matrix, size_t inputs_len, uint64_t *outputs_matrix,
                                      size_t outputs_len, uint32_t log_n, uint32_t num_ntts, uint32_t inputs_offset,
                                      uint32_t outputs_offset, uint32_t stride_between_input_arrays,
                                      uint32_t stride_between_output_arrays, bool bitrev_inputs, bool inverse,
                                      uint32_t log_extension_degree, uint32_t coset_index, void *stream);
/* Replaces ntt::batch_ntt_in_place (ntt.rs:338-369). */
glc_status glc_batch_ntt_in_place(uint64_t *inputs_matrix, size_t inputs_len, uint32_t log_n, uint32_t num_ntts,
                                  uint32_t inputs_offset, uint32_t stride_between_input_arrays, bool bitrev_inputs,
                                  bool inverse, uint32_t log_extension_degree, uint32_t coset_index, void *stream);

/* ---------------------------------------------------------------------------------------------
 * Bit reversal of the rows of a column-major matrix (rows a power of two).
 * Replaces ops_complex::bit_reverse (crates/boojum-cuda/src/ops_complex.rs:309-320) ... */
glc_status glc_bit_reverse(const uint64_t *src, uint64_t src_stride, uint64_t *dst, uint64_t dst_stride, uint32_t rows,
                           uint32_t cols, void *stream);
/* ... and ops_complex::bit_reverse_in_place (ops_complex.rs:322-331). */
glc_status glc_bit_reverse_in_place(uint64_t *values, uint64_t stride, uint32_t rows, uint32_t cols, void *stream);

/* ---------------------------------------------------------------------------------------------
 * Poseidon2 over Goldilocks, width 12, rate 8, capacity 4 (GLHasher,
 * crates/boojum-cuda/src/poseidon2.rs:383-441).  Digests are stored [4][count]: element j of
 * digest i at results[j * count + i].
 */
/* Installs the 30 x 12 round constants (round-major) on the current device.  The reference
 * generates them from boojum at build time (crates/boojum-cuda/build/poseidon2_gl.rs:3,34);
 * without this call the library uses its built-in placeholder set. */
glc_status glc_poseidon2_set_round_constants(const uint64_t *round_constants);
/* *out = 1 when glc_poseidon2_set_round_constants has installed constants on the current device,
 * 0 while every digest (leaves, nodes, trees, commitments, caps) still uses the built-in
 * placeholder set, which is not boojum's.  Host-side bookkeeping only; launches nothing. */
glc_status glc_poseidon2_round_constants_installed(uint32_t *out);
/* Replaces GpuTreeHasher::compute_leaf_hashes (poseidon2.rs:180-226). */
glc_status glc_poseidon2_compute_leaf_hashes(const uint64_t *values, size_t values_len, uint64_t *results,
                                             size_t results_len, uint32_t log_rows_per_hash, bool load_intermediate,
                                             bool store_intermediate, void *stream);
/* Replaces GpuTreeHasher::compute_node_hashes (poseidon2.rs:228-251). */
glc_status glc_poseidon2_compute_node_hashes(const uint64_t *values, size_t values_len, uint64_t *results,
                                             size_t results_len, void *stream);
/* Replaces GpuTreeHasher::build_merkle_tree_leaves (poseidon2.rs:253-274). */
glc_status glc_poseidon2_build_merkle_tree_leaves(const uint64_t *values, size_t values_len, uint64_t *results,
                                                  size_t results_len, uint32_t log_rows_per_hash,
                                                  bool load_intermediate, bool store_intermediate, void *stream);
/* Replaces GpuTreeHasher::build_merkle_tree_nodes (poseidon2.rs:276-295); values_len == results_len. */
glc_status glc_poseidon2_build_merkle_tree_nodes(const uint64_t *values, size_t values_len, uint64_t *results,
                                                 size_t results_len, uint32_t layers_count, void *stream);
/* Replaces GpuTreeHasher::build_merkle_tree (poseidon2.rs:297-314); results_len = 2 * 4 * leaves. */
glc_status glc_poseidon2_build_merkle_tree(const uint64_t *values, size_t values_len, uint64_t *results,
                                           size_t results_len, uint32_t log_rows_per_hash, uint32_t layers_count,
                                           void *stream);
/* Replaces GpuTreeHasher::gather_rows (poseidon2.rs:316-348): values is values_rows x cols with
 * column stride values_stride; results is (indexes_len << log_rows_per_index) x cols. */
glc_status glc_poseidon2_gather_rows(const uint32_t *indexes, size_t indexes_len, uint32_t log_rows_per_index,
                                     const uint64_t *values, uint64_t values_rows, uint64_t values_cols,
                                     uint64_t values_stride, uint64_t *results, uint64_t results_rows,
                                     uint64_t results_cols, uint64_t results_stride, void *stream);
/* Replaces GpuTreeHasher::gather_merkle_paths (poseidon2.rs:350-380). */
glc_status glc_poseidon2_gather_merkle_paths(const uint32_t *indexes, size_t indexes_len, const uint64_t *values,
                                             size_t values_len, uint64_t *results, size_t results_len,
                                             uint32_t layers_count, void *stream);

/* GoldilocksExt2 column layouts, replacing extension_field::convert (extension_field.rs:60-90,
 * kernels goldilocks_extension.cu:8-34).  Vectorized: extension column k is two base columns, c0 at
 * v[2k*v_stride + row] and c1 at v[(2k+1)*v_stride + row] (strides in base elements).  Tuples:
 * element (row, k) is the pair {c0, c1} at t[2*(k*t_stride + row)] (strides in extension
 * elements; the tuple matrix must be 16-byte aligned).  Strides >= rows. */
glc_status glc_ef_vectorized_to_tuples(const uint64_t *src, uint64_t src_stride, uint64_t *dst, uint64_t dst_stride,
                                       uint32_t rows, uint32_t cols, void *stream);
glc_status glc_ef_tuples_to_vectorized(const uint64_t *src, uint64_t src_stride, uint64_t *dst, uint64_t dst_stride,
                                       uint32_t rows, uint32_t cols, void *stream);

/* ops_complex::select (crates/boojum-cuda/src/ops_complex.rs:446-463, kernel native/ops_complex.cu:
 * 158-164): dst[i] = indexes[i] has bit 31 set ? 0 : src[indexes[i]] for i < indexes_len.  Every
 * length must fit in 32 bits and dst must hold indexes_len elements.  An index at or past src_len
 * (other than a placeholder) yields 0 (the reference reads whatever lies there). */
glc_status glc_select(const uint32_t *indexes, uint64_t indexes_len, const uint64_t *src, uint64_t src_len,
                      uint64_t *dst, uint64_t dst_len, void *stream);

/* GenericTraceStorage::fill_from_remote_witness_data (crates/shivini/src/data_structures/trace.rs:
 * 108-193): the trace matrix of a commitment from the witness values, column-major with
 * domain_size rows: num_variable_cols columns selected by variable_indexes, then num_witness_cols
 * columns selected by witness_indexes (glc_select on `values`), then num_multiplicity_cols (0 or 1)
 * column of the lookup multiplicities (u32, as field elements) zero-padded to domain_size.  Same
 * checks as the reference: variable_indexes_len = num_variable_cols * domain_size,
 * witness_indexes_len = num_witness_cols * domain_size, trace_len = columns * domain_size,
 * multiplicities_len <= domain_size.  All buffers are device buffers (the reference copies the
 * values and multiplicities from the host first). */
glc_status glc_trace_fill_from_witness(const uint32_t *variable_indexes, uint64_t variable_indexes_len,
                                       const uint32_t *witness_indexes, uint64_t witness_indexes_len,
                                       const uint64_t *values, uint64_t values_len, const uint32_t *multiplicities,
                                       uint64_t multiplicities_len, uint64_t *trace, uint64_t trace_len,
                                       uint32_t num_variable_cols, uint32_t num_witness_cols,
                                       uint32_t num_multiplicity_cols, uint64_t domain_size, void *stream);

/* ---------------------------------------------------------------------------------------------
 * Commitment jobs (no single counterpart in boojum-cuda: this is the sequence shivini runs for one
 * trace / argument / quotient commitment, crates/shivini/src/data_structures/storage.rs:155-330,
 * cache.rs:353-418, oracle.rs:62-88, built from the calls above).
 */
typedef struct glc_commit_job {
  const uint64_t *evals;  /* cols columns of 2^log_n natural-order evaluations (device) */
  uint64_t evals_stride;  /* elements between columns, >= 2^log_n */
  uint32_t log_n;         /* 1..24 */
  uint32_t cols;          /* >= 1; extension-field columns count as two adjacent base columns */
  uint32_t log_lde;       /* log2 of the LDE factor f, 0..4 */
  uint32_t log_cap;       /* log2 of the cap; log_lde <= log_cap <= log_n + log_lde */
  uint64_t *monomials;    /* optional (NULL = not kept): cols x 2^log_n natural-order coefficients */
  uint64_t *lde;          /* f cosets x cols x 2^log_n, coset-major; coset c holds the bit-reversed
                             evaluations on 7 * w_{f*2^log_n}^bitrev(c) * <w_{2^log_n}> */
  uint64_t *trees;        /* f subtrees x (2 * 4 * 2^log_n) digests, build_merkle_tree layout,
                             each with cap 2^(log_cap - log_lde) */
  uint64_t *cap;          /* [4][2^log_cap]: the subtree caps concatenated coset by coset */
} glc_commit_job;

/* One commitment on one stream (the plain per-call form).  Its digests use the round constants
 * of glc_poseidon2_set_round_constants (glc_poseidon2_round_constants_installed tells whether the
 * placeholder set is still in use). */
glc_status glc_commit(const glc_commit_job *job, void *stream);

/* glc_commit that also records CUDA events (cudaEvent_t, created by the caller) at the stage
 * boundaries: events[0] before the first stage, events[1] after the monomials, for each coset c
 * events[2+4c .. 5+4c] at its start, after its NTT, after its leaf hashes and after its node
 * layers (cosets may run on parallel internal streams), then one after the cap gather
 * (n_events >= 3 + 4 * 2^log_lde).  For per-stage timing of a live run. */
glc_status glc_commit_profiled(const glc_commit_job *job, void *stream, void **events, uint32_t n_events);

/* The cap of one commitment, computed without allocating any device memory (no counterpart in
 * the reference).  For callers that cannot call cudaMalloc: a device allocator or allocation
 * callback that needs a commitment while serving an allocation, a plugin whose host framework
 * owns all device memory, a process whose memory another framework has already reserved.  The
 * LDE cosets and subtrees live in one 2^24-element (128 MiB) array compiled into the library,
 * held by every GPU that loads it: jobs with 2^log_lde * (cols + 8) * 2^log_n > 2^24 are rejected.
 * evals, stride, sizes and cap ([4][2^log_cap], device) mean what they mean in glc_commit_job.
 * The first call on a device looks up the array's device address (cudaGetSymbolAddress), so make
 * it before any stream capture on that device.  Calls share the array: calls that overlap on the
 * GPU race; calls ordered on one stream or by events do not.  Needs glc_context_create; the
 * digests use the round constants installed by glc_poseidon2_set_round_constants (otherwise the
 * built-in placeholder set).  glc_context_destroy forgets the looked-up address, so after a
 * device reset create the context again and the next call looks it up anew. */
glc_status glc_commit_cap_noalloc(const uint64_t *evals, uint64_t evals_stride, uint32_t log_n, uint32_t cols,
                                  uint32_t log_lde, uint32_t log_cap, uint64_t *cap, void *stream);

/* Many commitments as one unit on `stream`: the jobs run concurrently on n_streams internal
 * streams (0 = 8), largest first, balanced by estimated cost; `stream` waits for all of them.
 * Capturable into a CUDA graph. */
glc_status glc_commit_batch(const glc_commit_job *jobs, uint32_t n_jobs, uint32_t n_streams, void *stream);

/* Many commitments (log_n <= 22 each) in ONE launch: a persistent grid (launched
 * cooperatively, so all its CTAs are resident) takes work items of every stage of every job
 * (inverse NTT tiles, bit reversal, coset NTT tiles, leaves, node layers, caps) from a global
 * counter in stage order; each item waits (bounded, about 1 s) only for the items it reads from,
 * so different jobs' stages overlap.  Same results as glc_commit on each job.  Allocates
 * (stream-ordered) and copies a small work table per call; not for use inside stream capture.
 * No counterpart in the reference, whose per-call form launches one kernel per NTT stage
 * (log_n < 16) and per tree layer (crates/boojum-cuda/src/ntt.rs:201-241, src/poseidon2.rs:276-295). */
glc_status glc_commit_batch_fused(const glc_commit_job *jobs, uint32_t n_jobs, void *stream);
/* glc_commit_batch_fused with a per-item trace: item i of the launch (items are numbered in
 * stage order, heaviest first within a stage) writes trace[4i .. 4i+3] = {the GPU global timer
 * in ns when its CTA claimed it, when its producers were done and it started, when it ended,
 * (SM id << 40) | (CTA index << 8) | kind}, kind 0 NTT tile, 1 bit reversal, 2 leaves, 3 nodes,
 * 4 cap entries.  Items from trace_items on are not recorded; the caller clears the buffer (a
 * device buffer of 4 * trace_items words) to tell unwritten records apart.  No counterpart in the
 * reference (its tracing is NVTX ranges around whole calls, shivini test.rs:2155-2181). */
glc_status glc_commit_batch_fused_traced(const glc_commit_job *jobs, uint32_t n_jobs, uint64_t *trace,
                                         uint64_t trace_items, void *stream);
/* glc_commit_batch_fused that a host can stop: before each item (and every 64 polls while an item
 * waits for its producers) the launch reads the 32-bit word at `cancel` (a device-readable
 * address: a word from glc_mapped_word_create, or device memory).  Once it reads non-zero, no
 * CTA claims or starts another item and every wait ends, so the launch returns after the items
 * already running; the outputs are then incomplete.  If `status` is not null, the last CTA to
 * leave writes 1 there when every item ran, 2 when the cancel skipped some.  A watchdog for the
 * persistent grid; the reference has no persistent kernel and no counterpart. */
glc_status glc_commit_batch_fused_cancellable(const glc_commit_job *jobs, uint32_t n_jobs, const uint32_t *cancel,
                                              uint32_t *status, void *stream);
/* A zeroed 32-bit word of page-locked host memory mapped into the device: the host reads and
 * writes *host, kernels use *device (for glc_commit_batch_fused_cancellable's cancel and status).
 * Released with glc_mapped_word_destroy(host). */
glc_status glc_mapped_word_create(uint32_t **host, uint32_t **device);
glc_status glc_mapped_word_destroy(uint32_t *host);
/* Waits of glc_commit_batch_fused that expired on the current device since the library was
 * loaded (0 unless something is wrong; a launch with an expired wait computes wrong results).
 * Synchronous. */
glc_status glc_commit_batch_fused_timeouts(uint64_t *out);

/* A batch captured once into a CUDA graph and replayed with one launch.  The graph keeps the
 * buffer addresses of the jobs it was created with. */
typedef struct glc_graph glc_graph;
glc_status glc_commit_graph_create(const glc_commit_job *jobs, uint32_t n_jobs, uint32_t n_streams, glc_graph **out);
glc_status glc_commit_graph_launch(glc_graph *graph, void *stream);
glc_status glc_commit_graph_destroy(glc_graph *graph);

/* ---------------------------------------------------------------------------------------------
 * Serving (no counterpart in boojum-cuda): commitment requests arrive over time; a worker thread
 * admits them by HBM footprint and in-flight slots and runs them concurrently on a stream pool
 * (continuous batching).  Host buffers are read and written by the device: pinned memory gives
 * asynchronous copies.  The context must exist on the device current at glc_server_create.
 */
typedef struct glc_server glc_server;
typedef struct glc_server_config {
  uint64_t hbm_budget_bytes; /* admission limit on the device memory held by admitted requests */
  uint32_t max_inflight;     /* at most this many requests on the device at once */
  uint32_t streams;          /* streams the requests run on (0 = 8) */
  uint32_t flat_priority;    /* 0: smaller requests run on higher-priority streams (their blocks are
                                scheduled first as SMs free up); 1: all streams at one priority */
} glc_server_config;
typedef struct glc_serve_request {
  const uint64_t *host_evals; /* cols x 2^log_n natural-order evaluations (host) */
  uint32_t log_n, cols, log_lde, log_cap;
  uint64_t *host_cap;         /* output: [4][2^log_cap] cap (host) */
  uint32_t keep_resident;     /* 1: keep the LDE and trees on the device until glc_server_release */
} glc_serve_request;
typedef struct glc_serve_result {
  uint64_t ticket;
  int status;           /* 0, or the error of this request */
  double queue_s;       /* submit -> admitted */
  double latency_s;     /* submit -> result on the host */
  uint64_t *device_lde; /* keep_resident only: f x cols x 2^log_n, as glc_commit_job.lde */
  uint64_t *device_trees;
} glc_serve_result;
typedef struct glc_server_stats {
  uint64_t completed, rejected, pending, inflight, used_bytes, peak_bytes, peak_inflight;
} glc_server_stats;
glc_status glc_server_create(const glc_server_config *config, glc_server **out);
/* Rejects (cudaErrorInvalidValue) a request whose footprint exceeds the budget. */
glc_status glc_server_submit(glc_server *server, const glc_serve_request *request, uint64_t *ticket);
/* Cancels a request that has not started. */
glc_status glc_server_cancel(glc_server *server, uint64_t ticket);
/* Waits up to timeout_s (< 0: forever) for a request; cudaErrorNotReady on timeout. */
glc_status glc_server_wait(glc_server *server, uint64_t ticket, double timeout_s, glc_serve_result *out);
/* Frees the device buffers of a finished keep_resident request. */
glc_status glc_server_release(glc_server *server, uint64_t ticket);
glc_status glc_server_get_stats(glc_server *server, glc_server_stats *out);
/* Finishes admitted and pending requests, then frees everything. */
glc_status glc_server_destroy(glc_server *server);

/* ---------------------------------------------------------------------------------------------
 * Launch tuning (no counterpart in boojum-cuda, whose plans are fixed tables, ntt.rs:70-169).
 * Values are per device; glc_autotune times candidates on the current device and installs the
 * fastest per NTT size and for the leaf kernel.  Launches read the values without a lock: set
 * them (or autotune) before other host threads launch work on that device.  Every choice
 * computes the same bits.
 */
typedef struct glc_ntt_tuning {
  uint32_t radix_bits;       /* stages per register round: 2, 3 or 4 */
  uint32_t k1;               /* stages in the strided pass of a two-pass NTT (0 = log_n / 2) */
  uint32_t max_log_w;        /* tile rows hold up to 2^max_log_w contiguous elements (<= 5) */
  uint32_t max_cols_per_cta; /* columns one CTA walks with the same twiddles (1..64) */
  uint32_t l2_chunk_mb;      /* a two-pass NTT runs both passes per chunk of this many MiB; 0: one chunk */
} glc_ntt_tuning;
typedef struct glc_p2_tuning {
  uint32_t leaf_threads; /* 64, 128 or 256 (leaf and wide node-layer kernels) */
  uint32_t rolled;       /* 0: fully unrolled, 1: partial rounds in a loop, 2: full rounds too */
  uint32_t lazy;         /* 1: partial rounds keep 11 of 12 state words partially reduced */
  uint32_t min_blocks;   /* leaf kernel register cap: 2 -> 128 registers, 3 -> 85 registers,
                            5 -> 102 registers (leaf_threads <= 128) */
} glc_p2_tuning;
glc_status glc_tuning_get_ntt(uint32_t log_n, glc_ntt_tuning *out);
glc_status glc_tuning_set_ntt(uint32_t log_n, const glc_ntt_tuning *tuning);
glc_status glc_tuning_get_p2(glc_p2_tuning *out);
glc_status glc_tuning_set_p2(const glc_p2_tuning *tuning);
/* Times the candidates for log_n in [log_n_min, log_n_max] on `cols` columns, or with cols = 0 on
 * 128 columns capped at 2^28 elements per size (synchronous; allocates and frees one scratch
 * buffer of the largest batch, at least 132 x 2^19 elements). */
glc_status glc_autotune(uint32_t log_n_min, uint32_t log_n_max, uint32_t cols, uint32_t reps);
glc_status glc_tuning_save(const char *path);
glc_status glc_tuning_load(const char *path);

/* ---------------------------------------------------------------------------------------------
 * Utilities (no counterpart in boojum-cuda).
 */
/* Elements offset .. offset+count of the seeded synthetic stream: ChaCha20 (RFC 8439) keyed by
 * key32, little-endian u64 words, a word >= p redrawn from the nonce-1 stream (uniform in [0, p)). */
glc_status glc_fill_random(uint64_t *dst, uint64_t count, uint64_t offset, const uint8_t *key32, void *stream);
/* Number of kernel launches this library has issued in this process (all devices). */
uint64_t glc_launch_count(void);
/* Modular-multiply throughput probe: blocks x 256 threads, 8 independent chains of `iters`
 * multiplies each (scratch: blocks * 256 elements). */
glc_status glc_modmul_probe(uint64_t *scratch, uint32_t blocks, uint32_t iters, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* GLC_H */
