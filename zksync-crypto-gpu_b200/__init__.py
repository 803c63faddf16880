"""B200-native Goldilocks LDE + Poseidon2 Merkle commitment (sm_100a CUDA behind a C ABI).

Python mirror of boojum-cuda's ntt::, poseidon2:: and ops_complex:: call surface, plus the
batched commitment and serving runtime.  Import name: the directory is not a valid Python
identifier, so load it with importlib.import_module("zksync-crypto-gpu_b200").
"""
from __future__ import annotations

from . import _lib
from ._buffers import DevicePtr
from ._lib import GlcError, LIB_PATH

_lib.lib()  # load libglc.so now: fail loudly at import when it is not built

from . import commit, context, extension_field, ntt, ops_complex, poseidon2, serve, trace, tuning  # noqa: E402
from .commit import CommitGraph, CommitJob  # noqa: E402
from .context import Context  # noqa: E402
from .poseidon2 import GLHasher  # noqa: E402

__all__ = ["Context", "GLHasher", "GlcError", "DevicePtr", "LIB_PATH", "CommitJob", "CommitGraph", "commit",
           "context", "extension_field", "ntt", "ops_complex", "poseidon2", "serve", "trace", "tuning"]
