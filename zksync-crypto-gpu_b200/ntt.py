"""Batched NTT / coset LDE: the counterpart of boojum-cuda's ntt module
(crates/boojum-cuda/src/ntt.rs:294-369).  Same argument names and meaning; buffers are torch
CUDA tensors of 8-byte elements (or DevicePtr), streams are torch streams (None = current)."""
from __future__ import annotations

from ._buffers import as_slice, stream_handle
from ._lib import call

NTTS_PER_BLOCK = 8  # kept for callers that size batches like the reference (ntt.rs:174)


def batch_ntt_out_of_place(inputs_matrix, outputs_matrix, log_n: int, num_ntts: int, inputs_offset: int,
                           outputs_offset: int, stride_between_input_arrays: int, stride_between_output_arrays: int,
                           bitrev_inputs: bool, inverse: bool, log_extension_degree: int, coset_index: int,
                           stream=None) -> None:
    """ntt::batch_ntt_out_of_place (ntt.rs:294)."""
    ip, il = as_slice(inputs_matrix)
    op, ol = as_slice(outputs_matrix)
    call("glc_batch_ntt_out_of_place", ip, il, op, ol, log_n, num_ntts, inputs_offset, outputs_offset,
         stride_between_input_arrays, stride_between_output_arrays, bool(bitrev_inputs), bool(inverse),
         log_extension_degree, coset_index, stream_handle(stream))


def batch_ntt_in_place(inputs_matrix, log_n: int, num_ntts: int, inputs_offset: int, stride_between_input_arrays: int,
                       bitrev_inputs: bool, inverse: bool, log_extension_degree: int, coset_index: int,
                       stream=None) -> None:
    """ntt::batch_ntt_in_place (ntt.rs:338)."""
    ip, il = as_slice(inputs_matrix)
    call("glc_batch_ntt_in_place", ip, il, log_n, num_ntts, inputs_offset, stride_between_input_arrays,
         bool(bitrev_inputs), bool(inverse), log_extension_degree, coset_index, stream_handle(stream))
