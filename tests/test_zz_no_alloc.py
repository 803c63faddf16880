"""glc_commit_cap_noalloc: the commitment cap for callers that cannot allocate device memory
(an allocator or allocation callback that needs a commitment while serving an allocation, a
plugin whose host framework owns all device memory, a process whose memory another framework
has reserved).  Its LDE and subtrees live in a fixed 2^24-element array inside the library.

Called through the C ABI and compared bit for bit (integer results: no tolerance) with the cap
that glc_commit computes from caller-allocated buffers, on two calls in a row: the second call
finds the first one's data in the shared array and must not depend on it.  This file is
collected last."""
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


def test_noalloc_cap_equals_commit_cap(glc, syn):
    # two calls in a row with different shapes; the second overwrites part of what the first left
    for log_n, cols, log_lde, log_cap in [(14, 64, 1, 4), (13, 40, 2, 4)]:
        ev = to_dev(syn.random_field_elements("noalloc-%d-%d" % (log_n, cols), cols << log_n))
        want = _cap_via_commit(glc, ev, log_n, cols, log_lde, log_cap)
        got = _cap_noalloc(glc, ev, log_n, cols, log_lde, log_cap)
        assert (got == want).all(), "cap differs from glc_commit for %s" % ((log_n, cols, log_lde, log_cap),)


def test_noalloc_rejects_jobs_beyond_the_array(glc):
    ev = zeros_dev(1 << 20)
    cap = zeros_dev(64)
    lib = glc._lib.lib()
    # 2^1 * (120 + 8) * 2^20 = 2^28 elements > 2^24
    st = lib.glc_commit_cap_noalloc(ev.data_ptr(), 1 << 20, 20, 120, 1, 4, cap.data_ptr(), None)
    assert st != 0
    assert b"maximum" in lib.glc_last_error_message()
