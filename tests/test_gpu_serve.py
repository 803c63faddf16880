"""Serving: continuous batching of commitment requests; each result is bit-identical alone and
in the mix; admission by HBM footprint; host-side failures (bad sizes, over budget, cancel,
timeouts) without any GPU fault."""
import numpy as np
import pytest

from conftest import canon, load_package, load_synthetic

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def glc(round_constants):
    g = load_package()
    ctx = g.Context.create(15, 15)
    g.poseidon2.set_round_constants(round_constants)
    yield g
    ctx.destroy()


def inp(i, log_n, cols):
    return load_synthetic().random_field_elements("serve-%d" % i, cols << log_n)


@pytest.mark.parametrize("size_priority", [True, False])
def test_mix_equals_alone(glc, oracle, size_priority):
    # the first job runs long enough that the small ones arrive while it is on the device; with
    # size priorities the small ones run on higher-priority streams than the first
    jobs = [(18, 64, 1, 4), (12, 8, 1, 4), (14, 24, 2, 4), (13, 16, 1, 4), (12, 40, 2, 4), (15, 8, 1, 4),
            (12, 130, 1, 1)]
    with glc.serve.Server(hbm_budget_bytes=8 << 30, max_inflight=4, streams=4, size_priority=size_priority) as srv:
        res = glc.serve.poisson_load(srv, jobs, rate_per_s=0, make_input=inp)
        st = srv.stats()
    assert st["completed"] >= len(jobs) and st["peak_inflight"] > 1, st
    for i, (j, cap) in enumerate(zip(jobs, res["caps"])):
        _, _, _, want = oracle.commit(inp(i, j[0], j[1]), j[0], j[1], j[2], j[3])
        assert (canon(cap) == want).all(), ("in the mix", j)
    # each job alone
    with glc.serve.Server(hbm_budget_bytes=8 << 30, max_inflight=1, streams=1) as srv:
        for i, j in enumerate(jobs):
            t = srv.submit(inp(i, j[0], j[1]), *j)
            cap, _ = srv.wait(t)
            assert (cap == res["caps"][i]).all(), ("alone", j)


def test_admission_by_footprint(glc):
    # budget for about two 2^14 x 32 jobs at a time
    jobs = [(14, 32, 1, 4)] * 6
    one = 8 * ((32 << 14) * 3 + 2 * 8 * (1 << 14) + 64)
    with glc.serve.Server(hbm_budget_bytes=2 * one + 1024, max_inflight=8, streams=4) as srv:
        res = glc.serve.poisson_load(srv, jobs, rate_per_s=0, make_input=inp)
        st = srv.stats()
    assert st["peak_bytes"] <= 2 * one + 1024 and st["peak_inflight"] <= 2
    assert res["jobs"] == 6


def test_rejections_and_cancel(glc):
    with glc.serve.Server(hbm_budget_bytes=1 << 20, max_inflight=1, streams=1) as srv:
        with pytest.raises(glc.GlcError):  # footprint over the budget
            srv.submit(inp(0, 14, 32), 14, 32, 1, 4)
        with pytest.raises(glc.GlcError):  # bad size
            srv.submit(np.zeros(8 << 2, dtype=np.uint64), 2, 8, 5, 5)
        assert srv.stats()["rejected"] == 1
    with glc.serve.Server(hbm_budget_bytes=1 << 30, max_inflight=1, streams=1) as srv:
        t1 = srv.submit(inp(1, 16, 64), 16, 64, 1, 4)
        t2 = srv.submit(inp(2, 12, 8), 12, 8, 1, 4)
        try:
            srv.cancel(t2)
            cancelled = True
        except glc.GlcError:  # it may already have started
            cancelled = False
        srv.wait(t1)
        if cancelled:
            with pytest.raises(glc.GlcError):
                srv.wait(t2)
        else:
            srv.wait(t2)


def test_wait_timeout_and_resident(glc, oracle):
    import torch
    with glc.serve.Server(hbm_budget_bytes=4 << 30, max_inflight=2, streams=2) as srv:
        t = srv.submit(inp(3, 16, 128), 16, 128, 1, 4, keep_resident=True)
        try:
            srv.wait(t, timeout_s=0.0)
            done_early = True
        except glc.GlcError as e:
            assert e.status == 600  # cudaErrorNotReady: still running
            done_early = False
        if not done_early:
            cap, r = srv.wait(t)
        else:
            cap, r = None, None
        if r is not None:
            assert r.device_lde
            srv.release(t)
