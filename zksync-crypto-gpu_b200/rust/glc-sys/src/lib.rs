//! Raw FFI declarations of libglc, one per C function of `include/glc.h`, with the same names,
//! argument order and C types.  Every function returns a `cudaError_t` value as `GlcStatus`
//! (0 = success; contract violations return 1, cudaErrorInvalidValue, and
//! `glc_last_error_message` names the violated condition).  Device buffers are raw device
//! pointers owned by the caller; `stream` is a `cudaStream_t` (null = the legacy default stream).
//!
//! Not compiled in this repository's build environment (it has no Rust toolchain).
#![allow(non_camel_case_types)]

use std::ffi::CStr;
use std::os::raw::{c_char, c_int, c_void};

pub type GlcStatus = c_int;
pub type Stream = *mut c_void;

/// One commitment (include/glc.h `glc_commit_job`): device buffers and the job's shape.
#[repr(C)]
#[derive(Debug, Clone, Copy)]
pub struct glc_commit_job {
    pub evals: *const u64,
    pub evals_stride: u64,
    pub log_n: u32,
    pub cols: u32,
    pub log_lde: u32,
    pub log_cap: u32,
    pub monomials: *mut u64,
    pub lde: *mut u64,
    pub trees: *mut u64,
    pub cap: *mut u64,
}

#[repr(C)]
pub struct glc_graph {
    _private: [u8; 0],
}

#[repr(C)]
pub struct glc_server {
    _private: [u8; 0],
}

#[repr(C)]
#[derive(Debug, Clone, Copy, Default)]
pub struct glc_server_config {
    pub hbm_budget_bytes: u64,
    pub max_inflight: u32,
    pub streams: u32,
    pub flat_priority: u32,
}

#[repr(C)]
#[derive(Debug, Clone, Copy)]
pub struct glc_serve_request {
    pub host_evals: *const u64,
    pub log_n: u32,
    pub cols: u32,
    pub log_lde: u32,
    pub log_cap: u32,
    pub host_cap: *mut u64,
    pub keep_resident: u32,
}

#[repr(C)]
#[derive(Debug, Clone, Copy)]
pub struct glc_serve_result {
    pub ticket: u64,
    pub status: c_int,
    pub queue_s: f64,
    pub latency_s: f64,
    pub device_lde: *mut u64,
    pub device_trees: *mut u64,
}

#[repr(C)]
#[derive(Debug, Clone, Copy, Default)]
pub struct glc_server_stats {
    pub completed: u64,
    pub rejected: u64,
    pub pending: u64,
    pub inflight: u64,
    pub used_bytes: u64,
    pub peak_bytes: u64,
    pub peak_inflight: u64,
}

#[repr(C)]
#[derive(Debug, Clone, Copy, Default)]
pub struct glc_ntt_tuning {
    pub radix_bits: u32,
    pub k1: u32,
    pub max_log_w: u32,
    pub max_cols_per_cta: u32,
    pub l2_chunk_mb: u32,
}

#[repr(C)]
#[derive(Debug, Clone, Copy, Default)]
pub struct glc_p2_tuning {
    pub leaf_threads: u32,
    pub rolled: u32,
    pub lazy: u32,
    pub min_blocks: u32,
}

#[link(name = "glc")]
extern "C" {
    pub fn glc_last_error_message() -> *const c_char;

    // context::Context::create / destroy (crates/boojum-cuda/src/context.rs:171-297)
    pub fn glc_context_create(powers_of_w_coarse_log_count: u32, powers_of_g_coarse_log_count: u32) -> GlcStatus;
    pub fn glc_context_destroy() -> GlcStatus;

    // ntt::batch_ntt_out_of_place / batch_ntt_in_place (crates/boojum-cuda/src/ntt.rs:294-369)
    pub fn glc_batch_ntt_out_of_place(inputs_matrix: *const u64, inputs_len: usize, outputs_matrix: *mut u64,
        outputs_len: usize, log_n: u32, num_ntts: u32, inputs_offset: u32, outputs_offset: u32,
        stride_between_input_arrays: u32, stride_between_output_arrays: u32, bitrev_inputs: bool, inverse: bool,
        log_extension_degree: u32, coset_index: u32, stream: Stream) -> GlcStatus;
    pub fn glc_batch_ntt_in_place(inputs_matrix: *mut u64, inputs_len: usize, log_n: u32, num_ntts: u32,
        inputs_offset: u32, stride_between_input_arrays: u32, bitrev_inputs: bool, inverse: bool,
        log_extension_degree: u32, coset_index: u32, stream: Stream) -> GlcStatus;

    // ops_complex::bit_reverse / bit_reverse_in_place (crates/boojum-cuda/src/ops_complex.rs:309-331)
    pub fn glc_bit_reverse(src: *const u64, src_stride: u64, dst: *mut u64, dst_stride: u64, rows: u32, cols: u32,
        stream: Stream) -> GlcStatus;
    pub fn glc_bit_reverse_in_place(values: *mut u64, stride: u64, rows: u32, cols: u32, stream: Stream) -> GlcStatus;

    // GpuTreeHasher for GLHasher (crates/boojum-cuda/src/poseidon2.rs:180-380)
    pub fn glc_poseidon2_set_round_constants(round_constants: *const u64) -> GlcStatus;
    pub fn glc_poseidon2_round_constants_installed(out: *mut u32) -> GlcStatus;
    pub fn glc_poseidon2_compute_leaf_hashes(values: *const u64, values_len: usize, results: *mut u64,
        results_len: usize, log_rows_per_hash: u32, load_intermediate: bool, store_intermediate: bool,
        stream: Stream) -> GlcStatus;
    pub fn glc_poseidon2_compute_node_hashes(values: *const u64, values_len: usize, results: *mut u64,
        results_len: usize, stream: Stream) -> GlcStatus;
    pub fn glc_poseidon2_build_merkle_tree_leaves(values: *const u64, values_len: usize, results: *mut u64,
        results_len: usize, log_rows_per_hash: u32, load_intermediate: bool, store_intermediate: bool,
        stream: Stream) -> GlcStatus;
    pub fn glc_poseidon2_build_merkle_tree_nodes(values: *const u64, values_len: usize, results: *mut u64,
        results_len: usize, layers_count: u32, stream: Stream) -> GlcStatus;
    pub fn glc_poseidon2_build_merkle_tree(values: *const u64, values_len: usize, results: *mut u64,
        results_len: usize, log_rows_per_hash: u32, layers_count: u32, stream: Stream) -> GlcStatus;
    pub fn glc_poseidon2_gather_rows(indexes: *const u32, indexes_len: usize, log_rows_per_index: u32,
        values: *const u64, values_rows: u64, values_cols: u64, values_stride: u64, results: *mut u64,
        results_rows: u64, results_cols: u64, results_stride: u64, stream: Stream) -> GlcStatus;
    pub fn glc_poseidon2_gather_merkle_paths(indexes: *const u32, indexes_len: usize, values: *const u64,
        values_len: usize, results: *mut u64, results_len: usize, layers_count: u32, stream: Stream) -> GlcStatus;

    // extension_field::convert (crates/boojum-cuda/src/extension_field.rs:60-90)
    pub fn glc_ef_vectorized_to_tuples(src: *const u64, src_stride: u64, dst: *mut u64, dst_stride: u64, rows: u32,
        cols: u32, stream: Stream) -> GlcStatus;
    pub fn glc_ef_tuples_to_vectorized(src: *const u64, src_stride: u64, dst: *mut u64, dst_stride: u64, rows: u32,
        cols: u32, stream: Stream) -> GlcStatus;

    // ops_complex::select (crates/boojum-cuda/src/ops_complex.rs:446-463) and shivini's
    // fill_from_remote_witness_data (crates/shivini/src/data_structures/trace.rs:108-193)
    pub fn glc_select(indexes: *const u32, indexes_len: u64, src: *const u64, src_len: u64, dst: *mut u64,
        dst_len: u64, stream: Stream) -> GlcStatus;
    pub fn glc_trace_fill_from_witness(variable_indexes: *const u32, variable_indexes_len: u64,
        witness_indexes: *const u32, witness_indexes_len: u64, values: *const u64, values_len: u64,
        multiplicities: *const u32, multiplicities_len: u64, trace: *mut u64, trace_len: u64, num_variable_cols: u32,
        num_witness_cols: u32, num_multiplicity_cols: u32, domain_size: u64, stream: Stream) -> GlcStatus;

    // commitment jobs (shivini's per-commitment sequence as one call)
    pub fn glc_commit(job: *const glc_commit_job, stream: Stream) -> GlcStatus;
    pub fn glc_commit_profiled(job: *const glc_commit_job, stream: Stream, events: *mut *mut c_void,
        n_events: u32) -> GlcStatus;
    pub fn glc_commit_cap_noalloc(evals: *const u64, evals_stride: u64, log_n: u32, cols: u32, log_lde: u32,
        log_cap: u32, cap: *mut u64, stream: Stream) -> GlcStatus;
    pub fn glc_commit_batch(jobs: *const glc_commit_job, n_jobs: u32, n_streams: u32, stream: Stream) -> GlcStatus;
    pub fn glc_commit_batch_fused(jobs: *const glc_commit_job, n_jobs: u32, stream: Stream) -> GlcStatus;
    pub fn glc_commit_batch_fused_traced(jobs: *const glc_commit_job, n_jobs: u32, trace: *mut u64,
        trace_items: u64, stream: Stream) -> GlcStatus;
    pub fn glc_commit_batch_fused_cancellable(jobs: *const glc_commit_job, n_jobs: u32, cancel: *const u32,
        status: *mut u32, stream: Stream) -> GlcStatus;
    pub fn glc_mapped_word_create(host: *mut *mut u32, device: *mut *mut u32) -> GlcStatus;
    pub fn glc_mapped_word_destroy(host: *mut u32) -> GlcStatus;
    pub fn glc_commit_batch_fused_timeouts(out: *mut u64) -> GlcStatus;
    pub fn glc_commit_graph_create(jobs: *const glc_commit_job, n_jobs: u32, n_streams: u32,
        out: *mut *mut glc_graph) -> GlcStatus;
    pub fn glc_commit_graph_launch(graph: *mut glc_graph, stream: Stream) -> GlcStatus;
    pub fn glc_commit_graph_destroy(graph: *mut glc_graph) -> GlcStatus;

    // serving
    pub fn glc_server_create(config: *const glc_server_config, out: *mut *mut glc_server) -> GlcStatus;
    pub fn glc_server_submit(server: *mut glc_server, request: *const glc_serve_request, ticket: *mut u64)
        -> GlcStatus;
    pub fn glc_server_cancel(server: *mut glc_server, ticket: u64) -> GlcStatus;
    pub fn glc_server_wait(server: *mut glc_server, ticket: u64, timeout_s: f64, out: *mut glc_serve_result)
        -> GlcStatus;
    pub fn glc_server_release(server: *mut glc_server, ticket: u64) -> GlcStatus;
    pub fn glc_server_get_stats(server: *mut glc_server, out: *mut glc_server_stats) -> GlcStatus;
    pub fn glc_server_destroy(server: *mut glc_server) -> GlcStatus;

    // launch tuning
    pub fn glc_tuning_get_ntt(log_n: u32, out: *mut glc_ntt_tuning) -> GlcStatus;
    pub fn glc_tuning_set_ntt(log_n: u32, tuning: *const glc_ntt_tuning) -> GlcStatus;
    pub fn glc_tuning_get_p2(out: *mut glc_p2_tuning) -> GlcStatus;
    pub fn glc_tuning_set_p2(tuning: *const glc_p2_tuning) -> GlcStatus;
    pub fn glc_autotune(log_n_min: u32, log_n_max: u32, cols: u32, reps: u32) -> GlcStatus;
    pub fn glc_tuning_save(path: *const c_char) -> GlcStatus;
    pub fn glc_tuning_load(path: *const c_char) -> GlcStatus;

    // utilities
    pub fn glc_fill_random(dst: *mut u64, count: u64, offset: u64, key32: *const u8, stream: Stream) -> GlcStatus;
    pub fn glc_launch_count() -> u64;
    pub fn glc_modmul_probe(scratch: *mut u64, blocks: u32, iters: u32, stream: Stream) -> GlcStatus;
}

/// The message of the calling thread's last contract violation ("" if none).
pub fn last_error_message() -> String {
    unsafe {
        let p = glc_last_error_message();
        if p.is_null() {
            String::new()
        } else {
            CStr::from_ptr(p).to_string_lossy().into_owned()
        }
    }
}

/// `Ok(())` for status 0, else the status and the library's message.
pub fn check(status: GlcStatus) -> Result<(), (GlcStatus, String)> {
    if status == 0 {
        Ok(())
    } else {
        Err((status, last_error_message()))
    }
}
