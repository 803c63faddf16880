"""Launch tuning of the NTT and leaf kernels (glc_tuning_*, glc_autotune)."""
from __future__ import annotations

import ctypes as C

from ._lib import call


class NttTuning(C.Structure):
    _fields_ = [("radix_bits", C.c_uint32), ("k1", C.c_uint32), ("max_log_w", C.c_uint32),
                ("max_cols_per_cta", C.c_uint32), ("l2_chunk_mb", C.c_uint32)]


class P2Tuning(C.Structure):
    _fields_ = [("leaf_threads", C.c_uint32), ("rolled", C.c_uint32), ("lazy", C.c_uint32), ("min_blocks", C.c_uint32)]


def get_ntt(log_n: int) -> NttTuning:
    t = NttTuning()
    call("glc_tuning_get_ntt", log_n, C.byref(t))
    return t


def set_ntt(log_n: int, radix_bits=3, k1=0, max_log_w=5, max_cols_per_cta=8, l2_chunk_mb=0) -> None:
    t = NttTuning(radix_bits, k1, max_log_w, max_cols_per_cta, l2_chunk_mb)
    call("glc_tuning_set_ntt", log_n, C.byref(t))


def get_p2() -> P2Tuning:
    t = P2Tuning()
    call("glc_tuning_get_p2", C.byref(t))
    return t


def set_p2(leaf_threads=256, rolled=1, lazy=0, min_blocks=2) -> None:
    t = P2Tuning(leaf_threads, rolled, lazy, min_blocks)
    call("glc_tuning_set_p2", C.byref(t))


def autotune(log_n_min: int, log_n_max: int, cols: int = 0, reps: int = 3) -> None:
    """Time the launch candidates on this device and install the fastest (cols = 0: 128 columns,
    capped at 2^28 elements per size)."""
    call("glc_autotune", log_n_min, log_n_max, cols, reps)


def save(path: str) -> None:
    call("glc_tuning_save", path.encode())


def load(path: str) -> None:
    call("glc_tuning_load", path.encode())
