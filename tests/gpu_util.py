"""Device-buffer helpers for the GPU tests (torch supplies memory and streams only)."""
import numpy as np


def torch():
    import torch as T
    return T


def to_dev(a):
    T = torch()
    a = np.ascontiguousarray(a, dtype=np.uint64)
    return T.from_numpy(a.view(np.int64).copy()).cuda()


def zeros_dev(n):
    T = torch()
    return T.zeros(int(n), dtype=T.int64, device="cuda")


def from_dev(t):
    torch().cuda.synchronize()
    return t.cpu().numpy().view(np.uint64)


class _RawDevice:
    """A raw device address seen through __cuda_array_interface__ (int64 elements)."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (int(n),), "typestr": "<i8", "data": (int(ptr), False),
                                         "version": 3}


def raw_to_host(ptr, n):
    """Copies n u64 elements from a raw device address (e.g. a resident serving buffer) to numpy."""
    T = torch()
    T.cuda.synchronize()
    return T.as_tensor(_RawDevice(ptr, n), device="cuda").cpu().numpy().view(np.uint64)
