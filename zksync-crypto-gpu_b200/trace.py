"""The trace matrix of a commitment from the prover's witness: the counterpart of shivini's
GenericTraceStorage::fill_from_remote_witness_data (crates/shivini/src/data_structures/
trace.rs:108-193) over device buffers (glc_trace_fill_from_witness)."""
from __future__ import annotations

from ._buffers import as_slice, stream_handle
from ._lib import call


def fill_from_remote_witness_data(variable_indexes, witness_indexes, values, multiplicities, trace,
                                  num_variable_cols: int, num_witness_cols: int, num_multiplicity_cols: int,
                                  domain_size: int, stream=None) -> None:
    """trace (column-major, domain_size rows) = the variable columns selected from `values` by
    variable_indexes, the witness columns selected by witness_indexes (bit 31 set: zero), then at
    most one column of the lookup multiplicities (u32) zero-padded to domain_size.  Index and
    multiplicity buffers hold 4-byte elements (torch int32 tensors carry the u32 bit patterns);
    `witness_indexes` / `multiplicities` may be None when their columns are absent."""
    vp, vl = as_slice(variable_indexes, 4) if variable_indexes is not None else (None, 0)
    wp, wl = as_slice(witness_indexes, 4) if witness_indexes is not None else (None, 0)
    xp, xl = as_slice(values)
    mp, ml = as_slice(multiplicities, 4) if multiplicities is not None else (None, 0)
    tp, tl = as_slice(trace)
    call("glc_trace_fill_from_witness", vp, vl, wp, wl, xp, xl, mp, ml, tp, tl, num_variable_cols, num_witness_cols,
         num_multiplicity_cols, domain_size, stream_handle(stream))
