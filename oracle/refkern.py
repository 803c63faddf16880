"""ctypes front end of oracle/_ref/libbcref.so: the reference's own CUDA kernels driven by
oracle/ref_harness.cu.  TEST INFRASTRUCTURE ONLY (parity checks and the reference-kernel timing
leg of the benchmark).  Buffers are raw device addresses (ints)."""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libbcref.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        vp, u32, sz, b = C.c_void_p, C.c_uint32, C.c_size_t, C.c_bool
        sig = {
            "ref_context_create": [u32, u32],
            "ref_context_destroy": [],
            "ref_batch_ntt": [vp, vp, u32, u32, u32, u32, b, b, u32, u32, vp],
            "ref_bit_reverse": [vp, sz, vp, sz, u32, u32, vp],
            "ref_p2_leaves": [vp, sz, vp, sz, u32, b, b, vp],
            "ref_p2_nodes": [vp, sz, vp, sz, vp],
            "ref_p2_build_merkle_tree": [vp, sz, vp, sz, u32, u32, vp],
            "ref_p2_gather_rows": [vp, u32, u32, vp, sz, vp, sz, u32, vp],
            "ref_p2_gather_merkle_paths": [vp, u32, vp, sz, vp, u32, vp],
            "ref_select": [vp, vp, vp, u32, vp],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.restype = C.c_int
            f.argtypes = args
        _lib = L
    return _lib


def call(name, *args):
    rc = getattr(lib(), name)(*args)
    if rc:
        raise RuntimeError("%s failed with %d" % (name, rc))
