"""Row bit reversal of column-major matrices and the index gather: the counterparts of boojum-cuda's
ops_complex::bit_reverse / bit_reverse_in_place (crates/boojum-cuda/src/ops_complex.rs:309-331)
and ops_complex::select (ops_complex.rs:446-463).  A matrix is given as (buffer, rows, cols,
stride) like the reference's DeviceMatrixChunk."""
from __future__ import annotations

from ._buffers import as_slice, stream_handle
from ._lib import call


def bit_reverse(src, dst, rows: int, cols: int, src_stride: int | None = None, dst_stride: int | None = None,
                stream=None) -> None:
    sp, sl = as_slice(src)
    dp, dl = as_slice(dst)
    src_stride = rows if src_stride is None else src_stride
    dst_stride = rows if dst_stride is None else dst_stride
    if cols and (sl < (cols - 1) * src_stride + rows or dl < (cols - 1) * dst_stride + rows):
        raise ValueError("bit_reverse: buffer shorter than the matrix")
    call("glc_bit_reverse", sp, src_stride, dp, dst_stride, rows, cols, stream_handle(stream))


def bit_reverse_in_place(values, rows: int, cols: int, stride: int | None = None, stream=None) -> None:
    vp_, vl = as_slice(values)
    stride = rows if stride is None else stride
    if cols and vl < (cols - 1) * stride + rows:
        raise ValueError("bit_reverse_in_place: buffer shorter than the matrix")
    call("glc_bit_reverse_in_place", vp_, stride, rows, cols, stream_handle(stream))


def select(indexes, src, dst, stream=None) -> None:
    """ops_complex::select (ops_complex.rs:446-463): dst[i] = src[indexes[i]] for i < len(indexes),
    0 where bit 31 of the index is set.  `indexes`: a device buffer of 4-byte elements (a torch
    int32 tensor holds the u32 bit patterns)."""
    ip, il = as_slice(indexes, 4)
    sp, sl = as_slice(src)
    dp, dl = as_slice(dst)
    call("glc_select", ip, il, sp, sl, dp, dl, stream_handle(stream))
