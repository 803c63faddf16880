"""GoldilocksExt2 column layouts: the counterpart of boojum-cuda's extension_field::convert
(crates/boojum-cuda/src/extension_field.rs:60-90) for VectorizedExtensionField <-> ExtensionField.

A vectorized matrix of `cols` extension columns is 2*cols base columns (c0 then c1 of each
extension column), `v_stride` base elements apart; a tuple matrix stores element (row, k) as the
pair {c0, c1} at pair index k*t_stride + row.  Buffers are u64 device tensors or DevicePtr."""
from __future__ import annotations

from ._buffers import as_slice, stream_handle
from ._lib import call


def _check(name, v_len, t_len, rows, cols, v_stride, t_stride):
    if cols and (v_len < (2 * cols - 1) * v_stride + rows or t_len < 2 * ((cols - 1) * t_stride + rows)):
        raise ValueError("%s: buffer shorter than the matrix" % name)


def vectorized_to_tuples(src, dst, rows: int, cols: int, src_stride: int | None = None, dst_stride: int | None = None,
                         stream=None) -> None:
    sp, sl = as_slice(src)
    dp, dl = as_slice(dst)
    src_stride = rows if src_stride is None else src_stride
    dst_stride = rows if dst_stride is None else dst_stride
    _check("vectorized_to_tuples", sl, dl, rows, cols, src_stride, dst_stride)
    call("glc_ef_vectorized_to_tuples", sp, src_stride, dp, dst_stride, rows, cols, stream_handle(stream))


def tuples_to_vectorized(src, dst, rows: int, cols: int, src_stride: int | None = None, dst_stride: int | None = None,
                         stream=None) -> None:
    sp, sl = as_slice(src)
    dp, dl = as_slice(dst)
    src_stride = rows if src_stride is None else src_stride
    dst_stride = rows if dst_stride is None else dst_stride
    _check("tuples_to_vectorized", dl, sl, rows, cols, dst_stride, src_stride)
    call("glc_ef_tuples_to_vectorized", sp, src_stride, dp, dst_stride, rows, cols, stream_handle(stream))
