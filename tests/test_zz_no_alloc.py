"""glc_commit_cap_noalloc: the commitment cap for callers that cannot allocate device memory
(an allocator or allocation callback that needs a commitment while serving an allocation, a
plugin whose host framework owns all device memory, a process whose memory another framework
has reserved).  Its LDE and subtrees live in a fixed 2^24-element array inside the library.

Called through the C ABI and compared bit for bit (integer results: no tolerance) with the cap
that glc_commit computes from caller-allocated buffers and with the oracle's cap, on calls in a
row: each call finds the previous one's data in the shared array and must not depend on it.
Covers the exact size limit (accepted), one column more (rejected), LDE factors 1 and 16.
This file is collected last."""
import ctypes as C

import pytest

from conftest import load_package
from gpu_util import from_dev, to_dev, zeros_dev

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def glc(round_constants):
    g = load_package()
    ctx = g.Context.create(15, 15)
    g.poseidon2.set_round_constants(round_constants)
    yield g
    ctx.destroy()


def _cap_via_commit(glc, ev_dev, log_n, cols, log_lde, log_cap):
    sz = glc.CommitJob.sizes(log_n, cols, log_lde, log_cap)
    job = glc.CommitJob(evals=ev_dev, log_n=log_n, cols=cols, log_lde=log_lde, log_cap=log_cap,
                        lde=zeros_dev(sz["lde"]), trees=zeros_dev(sz["trees"]), cap=zeros_dev(sz["cap"]))
    glc.commit.commit(job)
    return from_dev(job.cap)


def _cap_noalloc(glc, ev_dev, log_n, cols, log_lde, log_cap):
    import torch
    cap = zeros_dev(4 << log_cap)
    lib = glc._lib.lib()
    st = lib.glc_commit_cap_noalloc(ev_dev.data_ptr(), 1 << log_n, log_n, cols, log_lde, log_cap, cap.data_ptr(),
                                    C.c_void_p(torch.cuda.current_stream().cuda_stream))
    glc._lib.check(st, "glc_commit_cap_noalloc")
    return from_dev(cap)


# (log_n, cols, log_lde, log_cap): two ordinary shapes, the exact limit 2^0 * (248 + 8) * 2^16 =
# 2^24 (the monomials sit in place in coset 0), and LDE x16
SHAPES = [(14, 64, 1, 4), (13, 40, 2, 4), (16, 248, 0, 4), (12, 8, 4, 4)]


def test_noalloc_cap_equals_commit_cap_and_oracle(glc, syn, oracle):
    import numpy as np
    for log_n, cols, log_lde, log_cap in SHAPES:
        assert (1 << log_lde) * (cols + 8) << log_n <= 1 << 24
        ev = syn.random_field_elements("noalloc-%d-%d" % (log_n, cols), cols << log_n)
        ev_dev = to_dev(ev)
        want = _cap_via_commit(glc, ev_dev, log_n, cols, log_lde, log_cap)
        got = _cap_noalloc(glc, ev_dev, log_n, cols, log_lde, log_cap)
        assert (got == want).all(), "cap differs from glc_commit for %s" % ((log_n, cols, log_lde, log_cap),)
        cap = oracle.commit(np.ascontiguousarray(ev), log_n, cols, log_lde, log_cap)[3]
        assert (got == cap).all(), "cap differs from the oracle for %s" % ((log_n, cols, log_lde, log_cap),)


def test_noalloc_limit(glc):
    ev = zeros_dev(249 << 16)
    cap = zeros_dev(64)
    lib = glc._lib.lib()
    # one column past the limit: 2^0 * (249 + 8) * 2^16 > 2^24
    st = lib.glc_commit_cap_noalloc(ev.data_ptr(), 1 << 16, 16, 249, 0, 4, cap.data_ptr(), None)
    assert st != 0
    assert b"maximum" in lib.glc_last_error_message()
    # far past it: 2^1 * (120 + 8) * 2^20 = 2^28
    ev = zeros_dev(120 << 20)
    st = lib.glc_commit_cap_noalloc(ev.data_ptr(), 1 << 20, 20, 120, 1, 4, cap.data_ptr(), None)
    assert st != 0
    assert b"maximum" in lib.glc_last_error_message()
