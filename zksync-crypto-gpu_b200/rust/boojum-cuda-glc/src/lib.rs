//! boojum-cuda's commitment-path entry points with their reference signatures, implemented over
//! libglc.  The bodies of crates/boojum-cuda/src/ntt.rs:294-369 (batch NTTs),
//! src/poseidon2.rs:180-380 (GpuTreeHasher for GLHasher), src/ops_complex.rs:309-331 and 446-463
//! (bit reversal, select) and src/context.rs:171-297 (Context) become calls into libglc; the contract checks
//! stay the reference's `assert!`s, so a caller sees the same panics, and libglc re-checks them
//! (returning cudaErrorInvalidValue).  shivini switches by importing these paths instead of
//! boojum_cuda's.
//!
//! Not compiled in this repository's build environment (it has no Rust toolchain);
//! tests/test_rust_shim_cpu.py checks the extern block below against include/glc.h.

use boojum::field::goldilocks::GoldilocksField;
use era_cudart::result::{CudaResult, CudaResultWrap};
use era_cudart::slice::DeviceSlice;
use era_cudart::stream::CudaStream;
use era_cudart_sys::{cudaStream_t, CudaError};

type GL = GoldilocksField;

/// libglc's functions typed for boojum: field-element pointers, `cudaStream_t`, `CudaError`
/// results (libglc returns cudaError_t values only).
mod ffi {
    use super::*;
    #[link(name = "glc")]
    extern "C" {
        pub fn glc_context_create(powers_of_w_coarse_log_count: u32, powers_of_g_coarse_log_count: u32) -> CudaError;
        pub fn glc_context_destroy() -> CudaError;
        pub fn glc_batch_ntt_out_of_place(inputs_matrix: *const GL, inputs_len: usize, outputs_matrix: *mut GL,
            outputs_len: usize, log_n: u32, num_ntts: u32, inputs_offset: u32, outputs_offset: u32,
            stride_between_input_arrays: u32, stride_between_output_arrays: u32, bitrev_inputs: bool,
            inverse: bool, log_extension_degree: u32, coset_index: u32, stream: cudaStream_t) -> CudaError;
        pub fn glc_batch_ntt_in_place(inputs_matrix: *mut GL, inputs_len: usize, log_n: u32, num_ntts: u32,
            inputs_offset: u32, stride_between_input_arrays: u32, bitrev_inputs: bool, inverse: bool,
            log_extension_degree: u32, coset_index: u32, stream: cudaStream_t) -> CudaError;
        pub fn glc_bit_reverse(src: *const GL, src_stride: u64, dst: *mut GL, dst_stride: u64, rows: u32,
            cols: u32, stream: cudaStream_t) -> CudaError;
        pub fn glc_bit_reverse_in_place(values: *mut GL, stride: u64, rows: u32, cols: u32,
            stream: cudaStream_t) -> CudaError;
        pub fn glc_select(indexes: *const u32, indexes_len: u64, src: *const GL, src_len: u64, dst: *mut GL,
            dst_len: u64, stream: cudaStream_t) -> CudaError;
        pub fn glc_poseidon2_set_round_constants(round_constants: *const u64) -> CudaError;
        pub fn glc_poseidon2_compute_leaf_hashes(values: *const GL, values_len: usize, results: *mut GL,
            results_len: usize, log_rows_per_hash: u32, load_intermediate: bool, store_intermediate: bool,
            stream: cudaStream_t) -> CudaError;
        pub fn glc_poseidon2_compute_node_hashes(values: *const GL, values_len: usize, results: *mut GL,
            results_len: usize, stream: cudaStream_t) -> CudaError;
        pub fn glc_poseidon2_build_merkle_tree_leaves(values: *const GL, values_len: usize, results: *mut GL,
            results_len: usize, log_rows_per_hash: u32, load_intermediate: bool, store_intermediate: bool,
            stream: cudaStream_t) -> CudaError;
        pub fn glc_poseidon2_build_merkle_tree_nodes(values: *const GL, values_len: usize, results: *mut GL,
            results_len: usize, layers_count: u32, stream: cudaStream_t) -> CudaError;
        pub fn glc_poseidon2_build_merkle_tree(values: *const GL, values_len: usize, results: *mut GL,
            results_len: usize, log_rows_per_hash: u32, layers_count: u32, stream: cudaStream_t) -> CudaError;
        pub fn glc_poseidon2_gather_rows(indexes: *const u32, indexes_len: usize, log_rows_per_index: u32,
            values: *const GL, values_rows: u64, values_cols: u64, values_stride: u64, results: *mut GL,
            results_rows: u64, results_cols: u64, results_stride: u64, stream: cudaStream_t) -> CudaError;
        pub fn glc_poseidon2_gather_merkle_paths(indexes: *const u32, indexes_len: usize, values: *const GL,
            values_len: usize, results: *mut GL, results_len: usize, layers_count: u32,
            stream: cudaStream_t) -> CudaError;
    }
}

pub mod context {
    use super::*;
    use boojum::field::U64Representable;
    use boojum::implementations::poseidon_goldilocks_params::ALL_ROUND_CONSTANTS_AS_FIELD_ELEMENTS;

    /// context::Context (crates/boojum-cuda/src/context.rs:171-297): twiddle and power tables of
    /// the current device, plus boojum's Poseidon2 round constants installed once.
    pub struct Context {
        _private: (),
    }

    impl Context {
        pub fn create(powers_of_w_coarse_log_count: u32, powers_of_g_coarse_log_count: u32) -> CudaResult<Self> {
            assert!(powers_of_w_coarse_log_count <= 30);
            assert!(powers_of_g_coarse_log_count <= 30);
            unsafe { ffi::glc_context_create(powers_of_w_coarse_log_count, powers_of_g_coarse_log_count) }.wrap()?;
            let rc: Vec<u64> = ALL_ROUND_CONSTANTS_AS_FIELD_ELEMENTS.iter().map(|x| x.as_u64()).collect();
            assert_eq!(rc.len(), 30 * 12);
            unsafe { ffi::glc_poseidon2_set_round_constants(rc.as_ptr()) }.wrap()?;
            Ok(Self { _private: () })
        }

        pub fn destroy(self) -> CudaResult<()> {
            unsafe { ffi::glc_context_destroy() }.wrap()
        }
    }
}

pub mod ntt {
    use super::*;

    /// ntt::batch_ntt_out_of_place (crates/boojum-cuda/src/ntt.rs:294-335).
    #[allow(clippy::too_many_arguments)]
    pub fn batch_ntt_out_of_place(inputs_matrix: &DeviceSlice<GL>, outputs_matrix: &mut DeviceSlice<GL>, log_n: u32,
        num_ntts: u32, inputs_offset: u32, outputs_offset: u32, stride_between_input_arrays: u32,
        stride_between_output_arrays: u32, bitrev_inputs: bool, inverse: bool, log_extension_degree: u32,
        coset_index: u32, stream: &CudaStream) -> CudaResult<()> {
        let n = 1u32 << log_n;
        assert!(inputs_offset + n <= stride_between_input_arrays);
        assert!(outputs_offset + n <= stride_between_output_arrays);
        assert!(inputs_matrix.len() >= (num_ntts * stride_between_input_arrays) as usize);
        assert!(outputs_matrix.len() >= (num_ntts * stride_between_output_arrays) as usize);
        assert!(inputs_matrix.as_ptr() != outputs_matrix.as_ptr() as *const GL);
        unsafe {
            ffi::glc_batch_ntt_out_of_place(inputs_matrix.as_ptr(), inputs_matrix.len(), outputs_matrix.as_mut_ptr(),
                outputs_matrix.len(), log_n, num_ntts, inputs_offset, outputs_offset, stride_between_input_arrays,
                stride_between_output_arrays, bitrev_inputs, inverse, log_extension_degree, coset_index,
                stream.into())
        }
        .wrap()
    }

    /// ntt::batch_ntt_in_place (crates/boojum-cuda/src/ntt.rs:338-369).
    #[allow(clippy::too_many_arguments)]
    pub fn batch_ntt_in_place(inputs_matrix: &mut DeviceSlice<GL>, log_n: u32, num_ntts: u32, inputs_offset: u32,
        stride_between_input_arrays: u32, bitrev_inputs: bool, inverse: bool, log_extension_degree: u32,
        coset_index: u32, stream: &CudaStream) -> CudaResult<()> {
        let n = 1u32 << log_n;
        assert!(inputs_offset + n <= stride_between_input_arrays);
        assert!(inputs_matrix.len() >= (num_ntts * stride_between_input_arrays) as usize);
        unsafe {
            ffi::glc_batch_ntt_in_place(inputs_matrix.as_mut_ptr(), inputs_matrix.len(), log_n, num_ntts,
                inputs_offset, stride_between_input_arrays, bitrev_inputs, inverse, log_extension_degree,
                coset_index, stream.into())
        }
        .wrap()
    }
}

pub mod ops_complex {
    use super::*;

    /// ops_complex::bit_reverse (crates/boojum-cuda/src/ops_complex.rs:309-320), with the
    /// matrix chunks given as (slice, stride between columns, rows, cols).
    pub fn bit_reverse(src: &DeviceSlice<GL>, src_stride: usize, dst: &mut DeviceSlice<GL>, dst_stride: usize,
        rows: usize, cols: usize, stream: &CudaStream) -> CudaResult<()> {
        assert!(rows.is_power_of_two() && rows <= u32::MAX as usize && cols <= u32::MAX as usize);
        assert!(src.len() >= (cols - 1) * src_stride + rows && dst.len() >= (cols - 1) * dst_stride + rows);
        unsafe {
            ffi::glc_bit_reverse(src.as_ptr(), src_stride as u64, dst.as_mut_ptr(), dst_stride as u64, rows as u32,
                cols as u32, stream.into())
        }
        .wrap()
    }

    /// ops_complex::bit_reverse_in_place (crates/boojum-cuda/src/ops_complex.rs:322-331).
    pub fn bit_reverse_in_place(values: &mut DeviceSlice<GL>, stride: usize, rows: usize, cols: usize,
        stream: &CudaStream) -> CudaResult<()> {
        assert!(rows.is_power_of_two() && rows <= u32::MAX as usize && cols <= u32::MAX as usize);
        assert!(values.len() >= (cols - 1) * stride + rows);
        unsafe { ffi::glc_bit_reverse_in_place(values.as_mut_ptr(), stride as u64, rows as u32, cols as u32, stream.into()) }
            .wrap()
    }

    /// ops_complex::select (crates/boojum-cuda/src/ops_complex.rs:446-463): dst[i] = src[indexes[i]],
    /// or zero where bit 31 of the index is set.
    pub fn select(indexes: &DeviceSlice<u32>, src: &DeviceSlice<GL>, dst: &mut DeviceSlice<GL>, stream: &CudaStream)
        -> CudaResult<()> {
        assert!(indexes.len() <= u32::MAX as usize);
        assert!(src.len() <= u32::MAX as usize);
        assert!(dst.len() <= u32::MAX as usize);
        unsafe {
            ffi::glc_select(indexes.as_ptr(), indexes.len() as u64, src.as_ptr(), src.len() as u64, dst.as_mut_ptr(),
                dst.len() as u64, stream.into())
        }
        .wrap()
    }
}

pub mod poseidon2 {
    //! GpuTreeHasher for GLHasher (crates/boojum-cuda/src/poseidon2.rs:180-380): digests are
    //! stored [4][count], element j of digest i at results[j * count + i].
    use super::*;
    const RATE: usize = 8;
    const CAPACITY: usize = 4;

    pub fn compute_leaf_hashes(values: &DeviceSlice<GL>, results: &mut DeviceSlice<GL>, log_rows_per_hash: u32,
        load_intermediate: bool, store_intermediate: bool, stream: &CudaStream) -> CudaResult<()> {
        assert_eq!(results.len() % CAPACITY, 0);
        let count = results.len() / CAPACITY;
        assert_eq!(values.len() % (count << log_rows_per_hash), 0);
        let cols = values.len() / (count << log_rows_per_hash);
        assert!(!store_intermediate || ((cols << log_rows_per_hash) % RATE == 0));
        unsafe {
            ffi::glc_poseidon2_compute_leaf_hashes(values.as_ptr(), values.len(), results.as_mut_ptr(), results.len(),
                log_rows_per_hash, load_intermediate, store_intermediate, stream.into())
        }
        .wrap()
    }

    pub fn compute_node_hashes(values: &DeviceSlice<GL>, results: &mut DeviceSlice<GL>, stream: &CudaStream)
        -> CudaResult<()> {
        assert_eq!(values.len() % RATE, 0);
        assert_eq!(results.len() % CAPACITY, 0);
        assert_eq!(values.len(), results.len() * 2);
        unsafe {
            ffi::glc_poseidon2_compute_node_hashes(values.as_ptr(), values.len(), results.as_mut_ptr(), results.len(),
                stream.into())
        }
        .wrap()
    }

    pub fn build_merkle_tree_leaves(values: &DeviceSlice<GL>, results: &mut DeviceSlice<GL>, log_rows_per_hash: u32,
        load_intermediate: bool, store_intermediate: bool, stream: &CudaStream) -> CudaResult<()> {
        assert_eq!(results.len() % CAPACITY, 0);
        assert_eq!(values.len() % (results.len() / CAPACITY), 0);
        unsafe {
            ffi::glc_poseidon2_build_merkle_tree_leaves(values.as_ptr(), values.len(), results.as_mut_ptr(),
                results.len(), log_rows_per_hash, load_intermediate, store_intermediate, stream.into())
        }
        .wrap()
    }

    pub fn build_merkle_tree_nodes(values: &DeviceSlice<GL>, results: &mut DeviceSlice<GL>, layers_count: u32,
        stream: &CudaStream) -> CudaResult<()> {
        if layers_count == 0 {
            return Ok(());
        }
        assert_eq!(values.len() % RATE, 0);
        assert_eq!(values.len(), results.len());
        unsafe {
            ffi::glc_poseidon2_build_merkle_tree_nodes(values.as_ptr(), values.len(), results.as_mut_ptr(),
                results.len(), layers_count, stream.into())
        }
        .wrap()
    }

    pub fn build_merkle_tree(values: &DeviceSlice<GL>, results: &mut DeviceSlice<GL>, log_rows_per_hash: u32,
        stream: &CudaStream, layers_count: u32) -> CudaResult<()> {
        assert_ne!(layers_count, 0);
        assert_eq!(results.len() % (2 * CAPACITY), 0);
        let leaves_count = results.len() / (2 * CAPACITY);
        assert!(1 << (layers_count - 1) <= leaves_count);
        assert_eq!(values.len() % leaves_count, 0);
        unsafe {
            ffi::glc_poseidon2_build_merkle_tree(values.as_ptr(), values.len(), results.as_mut_ptr(), results.len(),
                log_rows_per_hash, layers_count, stream.into())
        }
        .wrap()
    }

    /// gather_rows with the matrix chunks given as (slice, rows, cols, stride between columns).
    #[allow(clippy::too_many_arguments)]
    pub fn gather_rows(indexes: &DeviceSlice<u32>, log_rows_per_index: u32, values: &DeviceSlice<GL>,
        values_rows: usize, values_cols: usize, values_stride: usize, results: &mut DeviceSlice<GL>,
        results_rows: usize, results_cols: usize, results_stride: usize, stream: &CudaStream) -> CudaResult<()> {
        assert!(log_rows_per_index < 32);
        assert_eq!(results_cols, values_cols);
        assert_eq!(results_rows, indexes.len() << log_rows_per_index);
        unsafe {
            ffi::glc_poseidon2_gather_rows(indexes.as_ptr(), indexes.len(), log_rows_per_index, values.as_ptr(),
                values_rows as u64, values_cols as u64, values_stride as u64, results.as_mut_ptr(),
                results_rows as u64, results_cols as u64, results_stride as u64, stream.into())
        }
        .wrap()
    }

    pub fn gather_merkle_paths(indexes: &DeviceSlice<u32>, values: &DeviceSlice<GL>, results: &mut DeviceSlice<GL>,
        layers_count: u32, stream: &CudaStream) -> CudaResult<()> {
        assert_eq!(values.len() % CAPACITY, 0);
        let values_count = values.len() / CAPACITY;
        assert!(values_count.is_power_of_two());
        let log_leaves_count = values_count.trailing_zeros() - 1;
        assert!(layers_count <= log_leaves_count);
        assert_eq!(indexes.len() * layers_count as usize * CAPACITY, results.len());
        unsafe {
            ffi::glc_poseidon2_gather_merkle_paths(indexes.as_ptr(), indexes.len(), values.as_ptr(), values.len(),
                results.as_mut_ptr(), results.len(), layers_count, stream.into())
        }
        .wrap()
    }
}
