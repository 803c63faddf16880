"""Commitment jobs (plain, batched, CUDA graph), tuning invariance and the device-side input
generator, against the oracle."""
import numpy as np
import pytest

from conftest import canon, load_package, load_synthetic
from gpu_util import from_dev, to_dev, zeros_dev

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def glc(round_constants):
    g = load_package()
    ctx = g.Context.create(15, 15)
    g.poseidon2.set_round_constants(round_constants)
    yield g
    ctx.destroy()


def make_job(glc, syn, log_n, cols, log_lde, log_cap, seed, keep_monomials=True):
    sz = glc.CommitJob.sizes(log_n, cols, log_lde, log_cap)
    ev = syn.random_field_elements(seed, sz["evals"])
    job = glc.CommitJob(evals=to_dev(ev), log_n=log_n, cols=cols, log_lde=log_lde, log_cap=log_cap,
                        lde=zeros_dev(sz["lde"]), trees=zeros_dev(sz["trees"]), cap=zeros_dev(sz["cap"]),
                        monomials=zeros_dev(sz["monomials"]) if keep_monomials else None)
    return job, ev


def check_job(oracle, job, ev):
    mono, lde, trees, cap = oracle.commit(ev, job.log_n, job.cols, job.log_lde, job.log_cap)
    if job.monomials is not None:
        assert (canon(from_dev(job.monomials)) == mono).all(), "monomials"
    assert (canon(from_dev(job.lde)) == lde).all(), "lde"
    assert (canon(from_dev(job.trees)) == trees).all(), "trees"
    assert (canon(from_dev(job.cap)) == cap).all(), "cap"


@pytest.mark.parametrize("log_n,cols,log_lde,log_cap", [(12, 8, 1, 4), (13, 9, 2, 4), (16, 16, 1, 4), (5, 3, 2, 2),
                                                         (14, 24, 0, 0), (10, 130, 1, 1),
                                                         # edges: one row pair, one column, the cap is
                                                         # the whole leaf layer (no node layer), LDE x16
                                                         (1, 1, 0, 0), (1, 3, 1, 2), (3, 1, 4, 4), (6, 17, 3, 9),
                                                         (11, 1, 4, 6)])
def test_commit_plain(glc, oracle, syn, log_n, cols, log_lde, log_cap):
    job, ev = make_job(glc, syn, log_n, cols, log_lde, log_cap, "plain-%d-%d" % (log_n, cols))
    glc.commit.commit(job)
    check_job(oracle, job, ev)


@pytest.mark.parametrize("log_n,cols,log_lde", [(12, 8, 2), (14, 64, 1), (13, 40, 2)])
def test_commit_without_monomials(glc, oracle, syn, log_n, cols, log_lde):
    # the monomials then live in the last coset's LDE slot, which that coset transforms in place
    # while the other cosets (on parallel streams) read them: the sizes are large enough for the
    # cosets to overlap on the device
    job, ev = make_job(glc, syn, log_n, cols, log_lde, 4, "nomono-%d-%d" % (log_n, cols), keep_monomials=False)
    for _ in range(3):
        glc.commit.commit(job)
    check_job(oracle, job, ev)


def test_commit_batch_uneven_and_alone(glc, oracle, syn):
    shapes = [(12, 8, 1), (15, 16, 2), (13, 32, 1), (12, 64, 2), (16, 8, 1), (14, 16, 2), (12, 128, 1)]
    jobs = [make_job(glc, syn, l, c, e, 4, "batch-%d" % i) for i, (l, c, e) in enumerate(shapes)]
    glc.commit.commit_batch([j for j, _ in jobs], n_streams=4)
    for j, ev in jobs:
        check_job(oracle, j, ev)
    # the same job alone gives the same bits as in the mix
    j0, ev0 = make_job(glc, syn, *shapes[1], 4, "batch-1")
    glc.commit.commit(j0)
    assert (from_dev(j0.cap) == from_dev(jobs[1][0].cap)).all()
    assert (from_dev(j0.lde) == from_dev(jobs[1][0].lde)).all()


def test_commit_batch_fused(glc, oracle, syn):
    """The fused batch (one cooperative launch for every stage of every job) on uneven small jobs:
    1-pass and 2-pass NTT sizes, LDE x1..x16, with and without a monomials buffer, caps from one
    entry per coset to the whole leaf layer; each equals the oracle's commitment."""
    shapes = [(12, 8, 1, 4, True), (13, 9, 2, 4, False), (16, 16, 1, 4, True), (5, 3, 2, 2, False),
              (14, 24, 0, 0, False), (10, 130, 1, 1, True), (1, 1, 0, 0, True), (3, 1, 4, 4, False),
              (15, 40, 2, 6, False), (12, 64, 3, 5, True), (11, 1, 4, 15, False), (16, 8, 2, 4, False)]
    jobs = [make_job(glc, syn, l, c, e, cap, "fused-%d" % i, keep_monomials=m)
            for i, (l, c, e, cap, m) in enumerate(shapes)]
    glc.commit.commit_batch_fused([j for j, _ in jobs])
    for j, ev in jobs:
        check_job(oracle, j, ev)
    # again on the same buffers (the work table is rebuilt per call), after zeroing the outputs
    for j, _ in jobs:
        j.cap.zero_()
        j.trees.zero_()
    glc.commit.commit_batch_fused([j for j, _ in jobs])
    for j, ev in jobs:
        check_job(oracle, j, ev)
    assert glc.commit.fused_timeouts() == 0


def test_commit_batch_fused_many_jobs(glc, syn):
    """80 seeded random small jobs in one launch: every cap equals glc_commit's (the per-call
    form, itself checked against the oracle), and no dependency wait expired."""
    rng = np.random.default_rng(77)
    jobs = []
    for t in range(80):
        l = int(rng.integers(8, 17))
        e = int(rng.integers(0, 3))
        jobs.append(make_job(glc, syn, l, int(rng.integers(1, 40)), e, int(rng.integers(e, e + 5)), "fmany-%d" % t,
                             keep_monomials=bool(rng.integers(0, 2)))[0])
    glc.commit.commit_batch_fused(jobs)
    got = [from_dev(j.cap).copy() for j in jobs]
    for j in jobs:
        glc.commit.commit(j)
    for j, g in zip(jobs, got):
        assert (from_dev(j.cap) == g).all(), (j.log_n, j.cols, j.log_lde, j.log_cap)
    assert glc.commit.fused_timeouts() == 0


def test_commit_batch_fused_traced(glc, oracle, syn):
    """The traced fused launch gives the oracle's commitments, and its trace is consistent: one
    record per item up to the buffer's size (the rest stays zero), claim <= start <= end, every
    item kind present, leaves starting after the first NTT tile and caps ending last."""
    import torch
    shapes = [(12, 8, 1, 4, True), (14, 24, 2, 4, False), (16, 16, 1, 4, False), (9, 3, 0, 2, True)]
    jobs = [make_job(glc, syn, l, c, e, cap, "ftrace-%d" % i, keep_monomials=m)
            for i, (l, c, e, cap, m) in enumerate(shapes)]
    trace = torch.zeros(4 << 16, dtype=torch.int64, device="cuda")
    glc.commit.commit_batch_fused([j for j, _ in jobs], trace=trace)
    for j, ev in jobs:
        check_job(oracle, j, ev)
    r = trace.cpu().numpy().view(np.uint64).reshape(-1, 4)
    n = int((r[:, 2] > 0).sum())
    assert 0 < n < len(r) and (r[n:] == 0).all() and (r[:n, 2] > 0).all()
    r = r[:n]
    assert (r[:, 0] <= r[:, 1]).all() and (r[:, 1] <= r[:, 2]).all()
    kinds = r[:, 3] & np.uint64(0xFF)
    assert set(kinds.tolist()) == {0, 1, 2, 3, 4}
    assert r[kinds == 2, 1].min() > r[kinds == 0, 1].min()
    assert r[kinds == 4, 2].max() == r[:, 2].max()
    s = glc.commit.fused_trace_summary(r)
    assert s["items"] == n and s["leaves"]["work_cta_ms"] > 0
    # a buffer smaller than the launch keeps only the first items
    small = torch.zeros(4 * 10, dtype=torch.int64, device="cuda")
    glc.commit.commit_batch_fused([j for j, _ in jobs], trace=small)
    assert (small.cpu().numpy().reshape(-1, 4)[:, 2] != 0).all()
    assert glc.commit.fused_timeouts() == 0


def test_commit_batch_fused_cancellable(glc, syn):
    """The cancellable fused launch: never cancelled, it equals the plain fused launch and reports
    1; cancelled before it starts, it runs no item (caps untouched) and reports 2; cancelled by the
    host while it runs, it ends early (status 2) or had already finished (status 1).  Every later
    launch is unaffected and no wait expires."""
    import time
    import torch
    shapes = [(15, 128, 2, 4)] * 12 + [(13, 16, 1, 4)] * 8
    jobs = [make_job(glc, syn, l, c, e, cap, "fcancel-%d" % i, keep_monomials=False)[0]
            for i, (l, c, e, cap) in enumerate(shapes)]
    glc.commit.commit_batch_fused(jobs)
    want = [from_dev(j.cap).copy() for j in jobs]
    cancel, status = glc.commit.MappedWord(), glc.commit.MappedWord()
    # never cancelled
    for j in jobs:
        j.cap.zero_()
    glc.commit.commit_batch_fused_cancellable(jobs, cancel, status)
    torch.cuda.synchronize()
    assert status.value == 1 and all((from_dev(j.cap) == w).all() for j, w in zip(jobs, want))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    glc.commit.commit_batch_fused_cancellable(jobs, cancel, status)
    e1.record()
    torch.cuda.synchronize()
    full_ms = e0.elapsed_time(e1)
    # cancelled before the launch: nothing runs
    for j in jobs:
        j.cap.zero_()
    status.value = 0
    cancel.value = 1
    e0.record()
    glc.commit.commit_batch_fused_cancellable(jobs, cancel, status)
    e1.record()
    torch.cuda.synchronize()
    assert status.value == 2 and e0.elapsed_time(e1) < full_ms / 4
    assert all((from_dev(j.cap) == 0).all() for j in jobs)
    # cancelled while running
    cancel.value = 0
    status.value = 0
    e0.record()
    glc.commit.commit_batch_fused_cancellable(jobs, cancel, status)
    e1.record()
    time.sleep(full_ms / 4e3)
    cancel.value = 1
    torch.cuda.synchronize()
    assert status.value in (1, 2)
    if status.value == 2:
        assert e0.elapsed_time(e1) < full_ms
    # the next launch is whole again
    cancel.value = 0
    for j in jobs:
        j.cap.zero_()
    glc.commit.commit_batch_fused(jobs)
    assert all((from_dev(j.cap) == w).all() for j, w in zip(jobs, want))
    assert glc.commit.fused_timeouts() == 0
    cancel.close()
    status.close()


def test_commit_batch_fused_large_jobs(glc, syn):
    """Jobs of 2^17..2^22 rows (strided first passes of 5..10 stages on 2^12-element tiles) mixed
    with small ones in one launch: every LDE, tree and cap equals glc_commit's."""
    shapes = [(22, 8, 1, 4), (20, 24, 2, 4), (17, 40, 1, 4), (19, 8, 2, 5), (12, 16, 1, 4), (21, 9, 1, 3)]
    jobs = [make_job(glc, syn, l, c, e, cap, "flarge-%d" % i, keep_monomials=(i % 2 == 0))[0]
            for i, (l, c, e, cap) in enumerate(shapes)]
    glc.commit.commit_batch_fused(jobs)
    got = [(from_dev(j.lde).copy(), from_dev(j.trees).copy(), from_dev(j.cap).copy()) for j in jobs]
    for j in jobs:
        j.cap.zero_()
        j.trees.zero_()
        glc.commit.commit(j)
    for j, (lde, trees, cap) in zip(jobs, got):
        n, f = 1 << j.log_n, 1 << j.log_lde
        computed = 8 * n - 4 * (1 << (j.log_cap - j.log_lde))  # the tree prefix below the cap
        t = from_dev(j.trees).reshape(f, 8 * n)[:, :computed]
        assert (canon(from_dev(j.lde)) == canon(lde)).all(), (j.log_n, "lde")
        assert (canon(t) == canon(trees.reshape(f, 8 * n)[:, :computed])).all(), (j.log_n, "trees")
        assert (from_dev(j.cap) == cap).all(), (j.log_n, "cap")
    assert glc.commit.fused_timeouts() == 0


def test_commit_batch_fused_contract(glc, syn):
    job, _ = make_job(glc, syn, 23, 1, 1, 4, "fused-big")
    with pytest.raises(glc.GlcError):
        glc.commit.commit_batch_fused([job])
    glc.commit.commit_batch_fused([])  # nothing to do


def test_commit_graph_replay(glc, oracle, syn):
    shapes = [(12, 8, 1), (13, 16, 2), (12, 32, 1)]
    jobs = [make_job(glc, syn, l, c, e, 4, "graph-%d" % i) for i, (l, c, e) in enumerate(shapes)]
    g = glc.CommitGraph([j for j, _ in jobs], n_streams=3)
    g.launch()
    for j, ev in jobs:
        check_job(oracle, j, ev)
        j.cap.zero_()
        j.lde.zero_()
    g.launch()
    for j, ev in jobs:
        check_job(oracle, j, ev)
    g.close()


def test_commit_contract(glc, syn):
    job, _ = make_job(glc, syn, 12, 8, 1, 0, "bad")  # cap smaller than the coset count
    with pytest.raises(glc.GlcError):
        glc.commit.commit(job)
    job, _ = make_job(glc, syn, 12, 8, 5, 5, "bad2")  # log_lde > 4
    with pytest.raises(glc.GlcError):
        glc.commit.commit(job)


@pytest.mark.parametrize("radix,k1,lw,cpc,mb", [(2, 0, 5, 8, 8), (3, 7, 3, 1, 8), (4, 12, 4, 4, 0), (3, 10, 5, 64, 0),
                                                (4, 9, 3, 8, 0)])
def test_ntt_tuning_invariance(glc, oracle, radix, k1, lw, cpc, mb):
    """Every tuning choice computes the same transform (bit-exact)."""
    log_n = 20 if k1 != 7 else 14
    n = 1 << log_n
    cols = 3
    saved = glc.tuning.get_ntt(log_n)
    glc.tuning.set_ntt(log_n, radix, k1, lw, cpc, mb)
    try:
        x = syn_x = load_synthetic().random_field_elements("tune-%d" % radix, cols * n)
        for bitrev_inputs, inverse, e, c in ((False, False, 1, 1), (True, True, 2, 3)):
            d_in, d_out = to_dev(x), zeros_dev(cols * n)
            glc.ntt.batch_ntt_out_of_place(d_in, d_out, log_n, cols, 0, 0, n, n, bitrev_inputs, inverse, e, c)
            assert (canon(from_dev(d_out)) == oracle.batch_ntt(syn_x, log_n, cols, n, n, bitrev_inputs, inverse, e, c)).all()
    finally:
        glc.tuning.set_ntt(log_n, saved.radix_bits, saved.k1, saved.max_log_w, saved.max_cols_per_cta, saved.l2_chunk_mb)


@pytest.mark.parametrize("threads,rolled,lazy,minb", [(64, 0, 0, 2), (128, 1, 1, 3), (256, 0, 1, 2), (256, 1, 0, 3),
                                                     (128, 0, 0, 3), (256, 1, 1, 2), (256, 2, 1, 3), (128, 2, 0, 2),
                                                     (64, 2, 1, 2), (256, 2, 0, 3), (128, 2, 1, 5), (64, 1, 0, 5)])
def test_leaf_tuning_invariance(glc, oracle, threads, rolled, lazy, minb):
    saved = glc.tuning.get_p2()
    glc.tuning.set_p2(threads, rolled, lazy, minb)
    try:
        count, cols = 1 << 10, 11
        vals = load_synthetic().random_field_elements("leaf-tune", cols * count)
        d_res = zeros_dev(4 * count)
        glc.GLHasher.compute_leaf_hashes(to_dev(vals), d_res, 0, False, False)
        assert (canon(from_dev(d_res)) == oracle.leaves(vals, 4 * count, 0)).all()
        d_tree = zeros_dev(8 * count)
        glc.GLHasher.build_merkle_tree(to_dev(vals), d_tree, 0, None, 11)
        assert (canon(from_dev(d_tree)) == oracle.build_merkle_tree(vals, 8 * count, 0, 11)).all()
    finally:
        glc.tuning.set_p2(saved.leaf_threads, saved.rolled, saved.lazy, saved.min_blocks)


def test_autotune_keeps_results(glc, oracle, tmp_path):
    glc.tuning.autotune(10, 12, cols=4, reps=1)
    path = str(tmp_path / "tuning.txt")
    glc.tuning.save(path)
    glc.tuning.load(path)
    job, ev = make_job(glc, load_synthetic(), 12, 8, 1, 4, "after-tune")
    glc.commit.commit(job)
    check_job(oracle, job, ev)


@pytest.mark.parametrize("count,offset", [(1, 0), (1000, 3), (1 << 16, 12345)])
def test_device_random_matches_python(glc, syn, count, offset):
    d = zeros_dev(count)
    syn.fill_device(d, "fill-seed", offset)
    assert (from_dev(d) == syn.random_field_elements("fill-seed", count, offset)).all()


def test_commit_random_shapes(glc, oracle, syn):
    # seeded random shapes across the contract: every output equals the oracle's
    rng = np.random.default_rng(2024)
    for t in range(10):
        log_n = int(rng.integers(1, 15))
        cols = int(rng.integers(1, 41))
        log_lde = int(rng.integers(0, 4))
        log_cap = int(rng.integers(log_lde, log_lde + log_n + 1))
        job, ev = make_job(glc, syn, log_n, cols, log_lde, log_cap, "random-%d" % t,
                           keep_monomials=bool(rng.integers(0, 2)))
        glc.commit.commit(job)
        check_job(oracle, job, ev)
