"""Poseidon2-Goldilocks tree hashing: the counterpart of boojum-cuda's GpuTreeHasher for
GLHasher (crates/boojum-cuda/src/poseidon2.rs:165-441).  Digests are [4][count]."""
from __future__ import annotations

import ctypes as C

from ._buffers import as_slice, stream_handle
from ._lib import call


def set_round_constants(round_constants) -> None:
    """Installs 30 x 12 round constants (round-major) on the current device."""
    vals = [int(v) for v in round_constants]
    if len(vals) != 360:
        raise ValueError("expected 360 round constants")
    arr = (C.c_uint64 * 360)(*vals)
    call("glc_poseidon2_set_round_constants", C.addressof(arr))


def round_constants_installed() -> bool:
    """True once set_round_constants has run on the current device; until then every digest uses
    the library's built-in placeholder constants (glc_poseidon2_round_constants_installed)."""
    v = C.c_uint32()
    call("glc_poseidon2_round_constants_installed", C.byref(v))
    return bool(v.value)


class GLHasher:
    RATE = 8
    CAPACITY = 4
    CHUNKING = 1

    @staticmethod
    def compute_leaf_hashes(values, results, log_rows_per_hash: int, load_intermediate: bool,
                            store_intermediate: bool, stream=None) -> None:
        vp_, vl = as_slice(values)
        rp, rl = as_slice(results)
        call("glc_poseidon2_compute_leaf_hashes", vp_, vl, rp, rl, log_rows_per_hash, bool(load_intermediate),
             bool(store_intermediate), stream_handle(stream))

    @staticmethod
    def compute_node_hashes(values, results, stream=None) -> None:
        vp_, vl = as_slice(values)
        rp, rl = as_slice(results)
        call("glc_poseidon2_compute_node_hashes", vp_, vl, rp, rl, stream_handle(stream))

    @staticmethod
    def build_merkle_tree_leaves(values, results, log_rows_per_hash: int, load_intermediate: bool,
                                 store_intermediate: bool, stream=None) -> None:
        vp_, vl = as_slice(values)
        rp, rl = as_slice(results)
        call("glc_poseidon2_build_merkle_tree_leaves", vp_, vl, rp, rl, log_rows_per_hash, bool(load_intermediate),
             bool(store_intermediate), stream_handle(stream))

    @staticmethod
    def build_merkle_tree_nodes(values, results, layers_count: int, stream=None) -> None:
        vp_, vl = as_slice(values)
        rp, rl = as_slice(results)
        call("glc_poseidon2_build_merkle_tree_nodes", vp_, vl, rp, rl, layers_count, stream_handle(stream))

    @staticmethod
    def build_merkle_tree(values, results, log_rows_per_hash: int, stream=None, layers_count: int = 1) -> None:
        vp_, vl = as_slice(values)
        rp, rl = as_slice(results)
        call("glc_poseidon2_build_merkle_tree", vp_, vl, rp, rl, log_rows_per_hash, layers_count,
             stream_handle(stream))

    @staticmethod
    def gather_rows(indexes, log_rows_per_index: int, values, values_rows: int, values_cols: int, result,
                    result_rows: int, result_cols: int, values_stride: int | None = None,
                    result_stride: int | None = None, stream=None) -> None:
        ip, il = as_slice(indexes, 4)
        vp_, vl = as_slice(values)
        rp, rl = as_slice(result)
        values_stride = values_rows if values_stride is None else values_stride
        result_stride = result_rows if result_stride is None else result_stride
        if values_cols and vl < (values_cols - 1) * values_stride + values_rows:
            raise ValueError("gather_rows: values buffer shorter than the matrix")
        if result_cols and rl < (result_cols - 1) * result_stride + result_rows:
            raise ValueError("gather_rows: result buffer shorter than the matrix")
        call("glc_poseidon2_gather_rows", ip, il, log_rows_per_index, vp_, values_rows, values_cols, values_stride,
             rp, result_rows, result_cols, result_stride, stream_handle(stream))

    @staticmethod
    def gather_merkle_paths(indexes, values, results, layers_count: int, stream=None) -> None:
        ip, il = as_slice(indexes, 4)
        vp_, vl = as_slice(values)
        rp, rl = as_slice(results)
        call("glc_poseidon2_gather_merkle_paths", ip, il, vp_, vl, rp, rl, layers_count, stream_handle(stream))
