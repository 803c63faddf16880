"""ctypes binding of libglc.so (the C ABI declared in include/glc.h).

The library must have been built (build.py); loading fails loudly otherwise: there is no CPU
fallback for any entry point.  GLC_LIBRARY names another build of the same library to load
instead of _build/libglc.so.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("GLC_LIBRARY") or os.path.join(HERE, "_build", "libglc.so")


class GlcError(RuntimeError):
    """A non-zero glc_status: a CUDA error code, or cudaErrorInvalidValue (1) for a violated
    argument contract (where boojum-cuda would panic through assert!)."""

    def __init__(self, status: int, where: str, message: str):
        self.status = status
        super().__init__("%s failed with status %d%s" % (where, status, (": " + message) if message else ""))


_lib = None

u64p = C.c_void_p
u32p = C.c_void_p
sz = C.c_size_t
u32 = C.c_uint32
u64 = C.c_uint64
vp = C.c_void_p
b = C.c_bool

SIGNATURES = {
    "glc_last_error_message": (C.c_char_p, []),
    "glc_context_create": (C.c_int, [u32, u32]),
    "glc_context_destroy": (C.c_int, []),
    "glc_batch_ntt_out_of_place": (C.c_int, [u64p, sz, u64p, sz, u32, u32, u32, u32, u32, u32, b, b, u32, u32, vp]),
    "glc_batch_ntt_in_place": (C.c_int, [u64p, sz, u32, u32, u32, u32, b, b, u32, u32, vp]),
    "glc_bit_reverse": (C.c_int, [u64p, u64, u64p, u64, u32, u32, vp]),
    "glc_bit_reverse_in_place": (C.c_int, [u64p, u64, u32, u32, vp]),
    "glc_poseidon2_set_round_constants": (C.c_int, [u64p]),
    "glc_poseidon2_round_constants_installed": (C.c_int, [vp]),
    "glc_poseidon2_compute_leaf_hashes": (C.c_int, [u64p, sz, u64p, sz, u32, b, b, vp]),
    "glc_poseidon2_compute_node_hashes": (C.c_int, [u64p, sz, u64p, sz, vp]),
    "glc_poseidon2_build_merkle_tree_leaves": (C.c_int, [u64p, sz, u64p, sz, u32, b, b, vp]),
    "glc_poseidon2_build_merkle_tree_nodes": (C.c_int, [u64p, sz, u64p, sz, u32, vp]),
    "glc_poseidon2_build_merkle_tree": (C.c_int, [u64p, sz, u64p, sz, u32, u32, vp]),
    "glc_poseidon2_gather_rows": (C.c_int, [u32p, sz, u32, u64p, u64, u64, u64, u64p, u64, u64, u64, vp]),
    "glc_poseidon2_gather_merkle_paths": (C.c_int, [u32p, sz, u64p, sz, u64p, sz, u32, vp]),
    "glc_ef_vectorized_to_tuples": (C.c_int, [u64p, u64, u64p, u64, u32, u32, vp]),
    "glc_ef_tuples_to_vectorized": (C.c_int, [u64p, u64, u64p, u64, u32, u32, vp]),
    "glc_select": (C.c_int, [u32p, u64, u64p, u64, u64p, u64, vp]),
    "glc_trace_fill_from_witness": (C.c_int, [u32p, u64, u32p, u64, u64p, u64, u32p, u64, u64p, u64, u32, u32, u32, u64, vp]),
    "glc_commit": (C.c_int, [vp, vp]),
    "glc_commit_profiled": (C.c_int, [vp, vp, vp, u32]),
    "glc_commit_cap_noalloc": (C.c_int, [u64p, u64, u32, u32, u32, u32, u64p, vp]),
    "glc_launch_count": (C.c_uint64, []),
    "glc_commit_batch": (C.c_int, [vp, u32, u32, vp]),
    "glc_commit_batch_fused": (C.c_int, [vp, u32, vp]),
    "glc_commit_batch_fused_traced": (C.c_int, [vp, u32, u64p, u64, vp]),
    "glc_commit_batch_fused_cancellable": (C.c_int, [vp, u32, vp, vp, vp]),
    "glc_mapped_word_create": (C.c_int, [vp, vp]),
    "glc_mapped_word_destroy": (C.c_int, [vp]),
    "glc_commit_batch_fused_timeouts": (C.c_int, [vp]),
    "glc_commit_graph_create": (C.c_int, [vp, u32, u32, vp]),
    "glc_commit_graph_launch": (C.c_int, [vp, vp]),
    "glc_commit_graph_destroy": (C.c_int, [vp]),
    "glc_tuning_get_ntt": (C.c_int, [u32, vp]),
    "glc_tuning_set_ntt": (C.c_int, [u32, vp]),
    "glc_tuning_get_p2": (C.c_int, [vp]),
    "glc_tuning_set_p2": (C.c_int, [vp]),
    "glc_autotune": (C.c_int, [u32, u32, u32, u32]),
    "glc_tuning_save": (C.c_int, [C.c_char_p]),
    "glc_tuning_load": (C.c_int, [C.c_char_p]),
    "glc_fill_random": (C.c_int, [u64p, u64, u64, C.c_char_p, vp]),
    "glc_modmul_probe": (C.c_int, [u64p, u32, u32, vp]),
}


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libglc.so is not built (run %s/build.py)" % HERE)
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status: int, where: str) -> None:
    if status != 0:
        msg = lib().glc_last_error_message()
        raise GlcError(status, where, msg.decode() if msg else "")


def call(name: str, *args) -> None:
    check(getattr(lib(), name)(*args), name)
