import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

P = 0xFFFFFFFF00000001


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def load_package():
    return importlib.import_module("zksync-crypto-gpu_b200")


def load_synthetic():
    return importlib.import_module("zksync-crypto-gpu_b200.synthetic")


def load_constants_module():
    return importlib.import_module("zksync-crypto-gpu_b200.p2_constants")


@pytest.fixture(scope="session")
def oracle():
    import oracle as O
    O.build()
    consts = load_constants_module()
    rc = consts.env_round_constants() or consts.grain_lfsr_round_constants()
    O.set_round_constants(rc)
    return O


@pytest.fixture(scope="session")
def round_constants():
    consts = load_constants_module()
    return consts.env_round_constants() or consts.grain_lfsr_round_constants()


@pytest.fixture(scope="session")
def syn():
    return load_synthetic()


def rand_elems(n, seed, noncanonical=False):
    """Seeded u64 test inputs; with noncanonical=True some values land in [p, 2^64)."""
    rng = np.random.default_rng(seed)
    if noncanonical:
        x = rng.integers(0, 2**64, size=n, dtype=np.uint64)
        # force a sprinkle of the edge values
        edges = np.array([0, 1, P - 1, P, P + 1, 2**64 - 1, 2**63], dtype=np.uint64)
        if n >= len(edges):
            x[rng.choice(n, size=len(edges), replace=False)] = edges
        return x
    return rng.integers(0, P, size=n, dtype=np.uint64)


def canon(a):
    a = np.asarray(a, dtype=np.uint64)
    return np.where(a >= np.uint64(P), a - np.uint64(P), a)
