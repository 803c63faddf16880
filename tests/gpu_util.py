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
