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
    """A zero-timeout wait either returns the finished request or reports cudaErrorNotReady; the
    LDE and trees kept resident on the device equal the oracle's either way."""
    from gpu_util import raw_to_host
    log_n, cols, log_lde, log_cap = 16, 128, 1, 4
    ev = inp(3, log_n, cols)
    with glc.serve.Server(hbm_budget_bytes=4 << 30, max_inflight=2, streams=2) as srv:
        t = srv.submit(ev, log_n, cols, log_lde, log_cap, keep_resident=True)
        try:
            cap, r = srv.wait(t, timeout_s=0.0)  # already finished
        except glc.GlcError as e:
            assert e.status == 600  # cudaErrorNotReady: still running
            cap, r = srv.wait(t)
        assert r.device_lde and r.device_trees
        n, f = 1 << log_n, 1 << log_lde
        _, lde, trees, want_cap = oracle.commit(ev, log_n, cols, log_lde, log_cap)
        assert (canon(cap) == want_cap).all(), "cap"
        assert (canon(raw_to_host(r.device_lde, f * cols * n)) == lde).all(), "resident LDE"
        assert (canon(raw_to_host(r.device_trees, f * 8 * n)) == trees).all(), "resident trees"
        srv.release(t)


def test_submit_does_not_wait_for_copies(glc):
    """submit() returns within milliseconds while the worker copies a large request's pageable
    input to the device (2 GiB: that copy takes about 100 ms or more); the small requests
    submitted meanwhile still finish."""
    import time
    log_n, cols = 23, 32
    big = np.full(cols << log_n, 3, dtype=np.uint64)  # pageable, pages touched
    small = [inp(10 + i, 12, 8) for i in range(8)]
    with glc.serve.Server(hbm_budget_bytes=32 << 30, max_inflight=4, streams=2) as srv:
        t_big = srv.submit(big, log_n, cols, 1, 4)
        time.sleep(0.02)  # the worker admits it and starts the copy
        took, tickets = [], []
        for x in small:
            t0 = time.perf_counter()
            tickets.append(srv.submit(x, 12, 8, 1, 4))
            took.append(time.perf_counter() - t0)
            time.sleep(0.005)
        srv.wait(t_big)
        for t in tickets:
            srv.wait(t)
    assert max(took) < 0.02, "submit waited %.1f ms" % (max(took) * 1e3)
