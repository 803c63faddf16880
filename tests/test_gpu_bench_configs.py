"""The benchmarked commitments, run exactly as bench.py runs them (the shipped B200 tuning table,
glc_commit with coset-parallel streams), checked bit for bit against the reference's own
kernels (crates/boojum-cuda/native compiled for sm_100a, driven with the reference's launch
plans: src/ntt.rs:70-169, src/poseidon2.rs:297-314) on the same inputs, and, for the
128 x 2^20 case, against the oracle's CPU commitment.

Shapes:
  * 128 columns x 2^20 rows, LDE x2, cap 16 (single-size batch);
  * 176 base columns x 2^22 rows (128 base + 24 extension columns stored as adjacent c0/c1
    base columns), LDE x2, cap 16 (the large commitment, ~42 GB on the device for both sides).
"""
import os

import numpy as np
import pytest

from conftest import ROOT, canon, load_package, load_synthetic
from gpu_util import from_dev

pytestmark = pytest.mark.gpu

refkern = pytest.importorskip("refkern")
if not refkern.available():
    pytest.skip("reference kernels not built (oracle/build_ref.py)", allow_module_level=True)

P_SIGNED = -4294967295  # p = 2^64 - 2^32 + 1 read as int64


def canon_dev(t):
    """x mod p for int64-viewed u64 values: x >= p exactly when -(2^32 - 1) <= x < 0 as int64."""
    import torch
    return torch.where((t < 0) & (t >= P_SIGNED), t + 4294967295, t)


@pytest.fixture(scope="module")
def env(round_constants):
    import torch
    g = load_package()
    ctx = g.Context.create(15, 15)
    g.poseidon2.set_round_constants(round_constants)
    saved_ntt = {l: g.tuning.get_ntt(l) for l in range(1, 25)}
    saved_p2 = g.tuning.get_p2()
    g.tuning.load(os.path.join(ROOT, "zksync-crypto-gpu_b200", "tuning_b200.txt"))
    refkern.call("ref_context_create", 15, 15)
    yield g, torch
    refkern.call("ref_context_destroy")
    for l, t in saved_ntt.items():
        g.tuning.set_ntt(l, t.radix_bits, t.k1, t.max_log_w, t.max_cols_per_cta, t.l2_chunk_mb)
    g.tuning.set_p2(saved_p2.leaf_threads, saved_p2.rolled, saved_p2.lazy, saved_p2.min_blocks)
    ctx.destroy()


def reference_commit(torch, evals, log_n, cols, log_lde, log_cap):
    """The commitment sequence shivini runs (storage.rs:155-330, cache.rs:353-418) on the
    reference's kernels: iNTT + bit reversal to monomials, one forward coset NTT and one
    subtree per coset (kernel coset bitrev(c)); returns (lde, trees, cap) device tensors."""
    n, f = 1 << log_n, 1 << log_lde
    s = torch.cuda.current_stream().cuda_stream
    mono = torch.empty(cols * n, dtype=torch.int64, device="cuda")
    lde = torch.empty(f * cols * n, dtype=torch.int64, device="cuda")
    trees = torch.empty(f * 8 * n, dtype=torch.int64, device="cuda")
    refkern.call("ref_batch_ntt", evals.data_ptr(), mono.data_ptr(), log_n, cols, n, n, False, True, 0, 0, s)
    refkern.call("ref_bit_reverse", mono.data_ptr(), n, mono.data_ptr(), n, log_n, cols, s)
    log_ccap = log_cap - log_lde
    layers = log_n - log_ccap + 1
    for c in range(f):
        coset = int(format(c, "0%db" % log_lde)[::-1], 2) if log_lde else 0
        dst = lde.data_ptr() + c * cols * n * 8
        refkern.call("ref_batch_ntt", mono.data_ptr(), dst, log_n, cols, n, n, False, False, log_lde, coset, s)
        refkern.call("ref_p2_build_merkle_tree", dst, cols * n, trees.data_ptr() + c * 8 * n * 8, 8 * n, 0, layers, s)
    del mono
    ccap = 1 << log_ccap
    cap = torch.empty(4 << log_cap, dtype=torch.int64, device="cuda")
    for c in range(f):
        sub = trees[c * 8 * n + 8 * n - 8 * ccap: c * 8 * n + 8 * n - 4 * ccap].view(4, ccap)
        cap.view(4, f * ccap)[:, c * ccap:(c + 1) * ccap] = sub
    torch.cuda.synchronize()
    return lde, trees, cap


def ours_commit(g, torch, evals, log_n, cols, log_lde, log_cap):
    sz = g.CommitJob.sizes(log_n, cols, log_lde, log_cap)
    dev = lambda k: torch.empty(sz[k], dtype=torch.int64, device="cuda")
    # trees zeroed: the tail of each subtree buffer past its cap is never written, and the oracle
    # leaves it at zero
    job = g.CommitJob(evals=evals, log_n=log_n, cols=cols, log_lde=log_lde, log_cap=log_cap, lde=dev("lde"),
                      trees=torch.zeros(sz["trees"], dtype=torch.int64, device="cuda"), cap=dev("cap"),
                      monomials=dev("monomials"))
    g.commit.commit(job)
    torch.cuda.synchronize()
    return job


def assert_same(torch, a, b, what, chunk=1 << 27):
    assert a.numel() == b.numel()
    for i in range(0, a.numel(), chunk):
        x, y = canon_dev(a[i:i + chunk]), canon_dev(b[i:i + chunk])
        if not torch.equal(x, y):
            bad = i + int((x != y).nonzero()[0].item())
            pytest.fail("%s differs from the reference kernels first at element %d" % (what, bad))


@pytest.mark.parametrize("log_n,cols", [(20, 128), (22, 176)], ids=["128x2^20", "176x2^22"])
def test_benchmarked_commitment_vs_reference_kernels(env, log_n, cols):
    g, torch = env
    log_lde, log_cap = 1, 4
    evals = torch.empty(cols << log_n, dtype=torch.int64, device="cuda")
    load_synthetic().fill_device(evals, "bench-parity-%d-%d" % (log_n, cols))
    job = ours_commit(g, torch, evals, log_n, cols, log_lde, log_cap)
    r_lde, r_trees, r_cap = reference_commit(torch, evals, log_n, cols, log_lde, log_cap)
    assert_same(torch, job.cap, r_cap, "cap")
    # each coset's subtree: the layers up to the cap (8 * 2^log_n - 4 * cap/f digests elements);
    # the tail of the buffer past the cap is written by neither side
    n, f, ccap = 1 << log_n, 1 << log_lde, 1 << (log_cap - log_lde)
    for c in range(f):
        lo, hi = c * 8 * n, c * 8 * n + 8 * n - 4 * ccap
        assert_same(torch, job.trees[lo:hi], r_trees[lo:hi], "trees of coset %d" % c)
    del r_trees
    assert_same(torch, job.lde, r_lde, "LDE")
    del r_lde, job
    torch.cuda.empty_cache()


def test_benchmarked_commitment_vs_oracle(env, oracle, syn):
    """128 x 2^20, LDE x2, cap 16 against the oracle's C commitment on the host cores."""
    g, torch = env
    log_n, cols, log_lde, log_cap = 20, 128, 1, 4
    d_ev = torch.empty(cols << log_n, dtype=torch.int64, device="cuda")
    syn.fill_device(d_ev, "bench-oracle")  # same values as syn.random_field_elements (tested elsewhere)
    ev = np.ascontiguousarray(from_dev(d_ev))
    job = ours_commit(g, torch, d_ev, log_n, cols, log_lde, log_cap)
    mono, lde, trees, cap = oracle.commit(ev, log_n, cols, log_lde, log_cap)
    assert (canon(from_dev(job.cap)) == cap).all(), "cap"
    assert (canon(from_dev(job.trees)) == trees).all(), "trees"
    assert (canon(from_dev(job.monomials)) == mono).all(), "monomials"
    assert (canon(from_dev(job.lde)) == lde).all(), "LDE"
