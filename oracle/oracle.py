"""ctypes front end of the CPU oracle (glc_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the CPU-baseline leg
of bench.py, always as the checker or the timed CPU baseline, never as a product path.
Arrays are numpy uint64 (contiguous); results are canonical field elements.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libglc_oracle.so")
P = 0xFFFFFFFF00000001

_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        u64p = C.POINTER(C.c_uint64)
        u32p = C.POINTER(C.c_uint32)
        sz = C.c_size_t
        L.or_mul.restype = C.c_uint64
        L.or_mul.argtypes = [C.c_uint64, C.c_uint64]
        L.or_root_of_unity.restype = C.c_uint64
        L.or_root_of_unity.argtypes = [C.c_uint32]
        ntt_args = [u64p, u64p, C.c_uint32, C.c_uint32, C.c_uint64, C.c_uint64, C.c_int, C.c_int, C.c_uint32, C.c_uint32]
        L.or_batch_ntt.argtypes = ntt_args + [C.c_int]
        L.or_batch_ntt_naive.argtypes = ntt_args
        L.or_bit_reverse.argtypes = [u64p, C.c_uint64, u64p, C.c_uint64, C.c_uint32, C.c_uint32]
        L.or_ef_vectorized_to_tuples.argtypes = [u64p, C.c_uint64, u64p, C.c_uint64, C.c_uint32, C.c_uint32]
        L.or_ef_tuples_to_vectorized.argtypes = [u64p, C.c_uint64, u64p, C.c_uint64, C.c_uint32, C.c_uint32]
        L.or_p2_set_round_constants.argtypes = [u64p]
        L.or_p2_permutation.argtypes = [u64p]
        L.or_p2_leaves.argtypes = [u64p, sz, u64p, sz, C.c_uint32, C.c_int, C.c_int, C.c_int]
        L.or_p2_nodes.argtypes = [u64p, sz, u64p, sz, C.c_int]
        L.or_p2_build_merkle_tree.argtypes = [u64p, sz, u64p, sz, C.c_uint32, C.c_uint32, C.c_int]
        L.or_p2_gather_rows.argtypes = [u32p, C.c_uint32, C.c_uint32, u64p, C.c_uint64, C.c_uint32, u64p, C.c_uint64]
        L.or_p2_gather_merkle_paths.argtypes = [u32p, C.c_uint32, u64p, sz, C.c_uint32, u64p, sz]
        L.or_p2_find_opening.restype = C.c_int64
        L.or_p2_find_opening.argtypes = [u64p, C.c_uint32, u64p, C.c_uint32, u64p, C.c_uint32]
        L.or_select.argtypes = [u32p, C.c_uint64, u64p, C.c_uint64, u64p]
        L.or_trace_fill.argtypes = [u32p, u32p, u64p, C.c_uint64, u32p, C.c_uint64, u64p, C.c_uint32, C.c_uint32,
                                    C.c_uint32, C.c_uint64]
        L.or_commit.argtypes = [u64p, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, u64p, u64p, u64p, u64p, C.c_int]
        _lib = L
    return _lib


def _p(a):
    if a is None:
        return None
    assert a.dtype == np.uint64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_uint64))


def _p32(a):
    assert a.dtype == np.uint32 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_uint32))


def canon(a: np.ndarray) -> np.ndarray:
    a = np.asarray(a, dtype=np.uint64)
    return np.where(a >= np.uint64(P), a - np.uint64(P), a)


def set_round_constants(rc) -> None:
    arr = np.ascontiguousarray(np.asarray(rc, dtype=np.uint64).reshape(-1))
    assert arr.size == 360
    lib().or_p2_set_round_constants(_p(arr))


def permutation(state) -> np.ndarray:
    s = np.ascontiguousarray(np.asarray(state, dtype=np.uint64).copy())
    lib().or_p2_permutation(_p(s))
    return s


def batch_ntt(inp, log_n, num_ntts, in_stride, out_stride, bitrev_inputs, inverse, log_ext, coset_idx,
              out=None, threads=os.cpu_count() or 1, naive=False):
    """Returns `out` (allocated as zeros of num_ntts*out_stride when None)."""
    if out is None:
        out = np.zeros(num_ntts * out_stride, dtype=np.uint64)
    if naive:
        rc = lib().or_batch_ntt_naive(_p(inp), _p(out), log_n, num_ntts, in_stride, out_stride, int(bitrev_inputs),
                                      int(inverse), log_ext, coset_idx)
    else:
        rc = lib().or_batch_ntt(_p(inp), _p(out), log_n, num_ntts, in_stride, out_stride, int(bitrev_inputs),
                                int(inverse), log_ext, coset_idx, threads)
    if rc:
        raise ValueError("or_batch_ntt: contract violation")
    return out


def bit_reverse(src, log_rows, cols, src_stride=None, dst=None, dst_stride=None):
    n = 1 << log_rows
    src_stride = n if src_stride is None else src_stride
    dst_stride = n if dst_stride is None else dst_stride
    if dst is None:
        dst = np.zeros(cols * dst_stride, dtype=np.uint64)
    lib().or_bit_reverse(_p(src), src_stride, _p(dst), dst_stride, log_rows, cols)
    return dst


def ef_vectorized_to_tuples(v, v_stride, rows, cols, t_stride=None):
    """GoldilocksExt2 columns: vectorized (c0 column, c1 column) -> {c0, c1} pairs."""
    t_stride = rows if t_stride is None else t_stride
    t = np.zeros(2 * cols * t_stride, dtype=np.uint64)
    lib().or_ef_vectorized_to_tuples(_p(v), v_stride, _p(t), t_stride, rows, cols)
    return t


def ef_tuples_to_vectorized(t, t_stride, rows, cols, v_stride=None):
    v_stride = rows if v_stride is None else v_stride
    v = np.zeros(2 * cols * v_stride, dtype=np.uint64)
    lib().or_ef_tuples_to_vectorized(_p(t), t_stride, _p(v), v_stride, rows, cols)
    return v


def select(indexes, src):
    """ops_complex::select: src[indexes[i]], 0 where bit 31 is set (or the index is past src)."""
    idx = np.ascontiguousarray(indexes, dtype=np.uint32)
    src = np.ascontiguousarray(src, dtype=np.uint64)
    out = np.zeros(idx.size, dtype=np.uint64)
    lib().or_select(_p32(idx), idx.size, _p(src), src.size, _p(out))
    return out


def trace_fill(variable_indexes, witness_indexes, values, multiplicities, nv, nw, nm, n):
    """fill_from_remote_witness_data: the (nv + nw + nm) x n trace."""
    vi = np.ascontiguousarray(variable_indexes, dtype=np.uint32)
    wi = np.ascontiguousarray(witness_indexes if witness_indexes is not None else [], dtype=np.uint32)
    vals = np.ascontiguousarray(values, dtype=np.uint64)
    mult = np.ascontiguousarray(multiplicities if multiplicities is not None else [], dtype=np.uint32)
    assert vi.size == nv * n and wi.size == nw * n and nm <= 1 and mult.size <= n * nm
    out = np.zeros((nv + nw + nm) * n, dtype=np.uint64)
    lib().or_trace_fill(_p32(vi), _p32(wi), _p(vals), vals.size, _p32(mult), mult.size, _p(out), nv, nw, nm, n)
    return out


def leaves(values, results_len, log_rows_per_hash=0, load_intermediate=False, store_intermediate=False,
           results=None, threads=os.cpu_count() or 1):
    if results is None:
        results = np.zeros(results_len, dtype=np.uint64)
    if lib().or_p2_leaves(_p(values), values.size, _p(results), results.size, log_rows_per_hash,
                          int(load_intermediate), int(store_intermediate), threads):
        raise ValueError("or_p2_leaves: contract violation")
    return results


def nodes(values, threads=os.cpu_count() or 1):
    results = np.zeros(values.size // 2, dtype=np.uint64)
    if lib().or_p2_nodes(_p(values), values.size, _p(results), results.size, threads):
        raise ValueError("or_p2_nodes: contract violation")
    return results


def build_merkle_tree(values, results_len, log_rows_per_hash, layers_count, threads=os.cpu_count() or 1):
    results = np.zeros(results_len, dtype=np.uint64)
    if lib().or_p2_build_merkle_tree(_p(values), values.size, _p(results), results.size, log_rows_per_hash,
                                     layers_count, threads):
        raise ValueError("or_p2_build_merkle_tree: contract violation")
    return results


def gather_rows(indexes, log_rows_per_index, values, values_stride, cols):
    idx = np.ascontiguousarray(indexes, dtype=np.uint32)
    rows = idx.size << log_rows_per_index
    out = np.zeros(rows * cols, dtype=np.uint64)
    lib().or_p2_gather_rows(_p32(idx), idx.size, log_rows_per_index, _p(values), values_stride, cols, _p(out), rows)
    return out


def gather_merkle_paths(indexes, values, layers_count):
    idx = np.ascontiguousarray(indexes, dtype=np.uint32)
    out = np.zeros(idx.size * layers_count * 4, dtype=np.uint64)
    if lib().or_p2_gather_merkle_paths(_p32(idx), idx.size, _p(values), values.size, layers_count, _p(out), out.size):
        raise ValueError("or_p2_gather_merkle_paths: contract violation")
    return out


def find_opening(leaf, path, cap) -> int:
    leaf = np.ascontiguousarray(leaf, dtype=np.uint64)
    path = np.ascontiguousarray(path, dtype=np.uint64).reshape(-1)
    cap = np.ascontiguousarray(cap, dtype=np.uint64).reshape(-1)
    return int(lib().or_p2_find_opening(_p(leaf), leaf.size, _p(path), path.size // 4, _p(cap), cap.size // 4))


def commit(evals, log_n, cols, log_lde, log_cap, threads=os.cpu_count() or 1):
    """Returns (monomials, lde, trees, cap) as in or_commit."""
    n = 1 << log_n
    f = 1 << log_lde
    mono = np.zeros(cols * n, dtype=np.uint64)
    lde = np.zeros(f * cols * n, dtype=np.uint64)
    trees = np.zeros(f * 8 * n, dtype=np.uint64)
    cap = np.zeros(4 << log_cap, dtype=np.uint64)
    if lib().or_commit(_p(evals), log_n, cols, log_lde, log_cap, _p(mono), _p(lde), _p(trees), _p(cap), threads):
        raise ValueError("or_commit: contract violation")
    return mono, lde, trees, cap
