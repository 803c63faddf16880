"""Witness-to-trace fill: glc_select (ops_complex::select, ops_complex.rs:446-463) against the
oracle and the reference's own select kernel, glc_trace_fill_from_witness
(fill_from_remote_witness_data, trace.rs:108-193) against the oracle, and the fill feeding a
commitment whose cap equals the oracle's commitment of the oracle's trace."""
import sys
import os

import numpy as np
import pytest

from conftest import ROOT, load_package, rand_elems
from gpu_util import from_dev, to_dev, zeros_dev

pytestmark = pytest.mark.gpu

PH = np.uint32(1 << 31)


@pytest.fixture(scope="module")
def glc(round_constants):
    g = load_package()
    ctx = g.Context.create(15, 15)
    g.poseidon2.set_round_constants(round_constants)
    yield g
    ctx.destroy()


def idx_dev(a):
    import torch
    a = np.ascontiguousarray(a, dtype=np.uint32)
    return torch.from_numpy(a.view(np.int32).copy()).cuda()


def rand_indexes(n, src_len, seed, placeholders=0.05, out_of_range=0.0):
    rng = np.random.default_rng(seed)
    ix = rng.integers(0, src_len, size=n, dtype=np.uint32)
    ph = rng.random(n) < placeholders
    ix[ph] |= PH
    if out_of_range:
        oor = rng.random(n) < out_of_range
        ix[oor & ~ph] = np.uint32(src_len) + rng.integers(0, 1000, size=int((oor & ~ph).sum()), dtype=np.uint32)
    return ix


@pytest.mark.parametrize("count,src_len", [(1, 1), (3, 10), (4, 4), (5, 100), (1000, 333), (4099, 1 << 16),
                                           ((1 << 20) + 3, 1 << 22)])
def test_select_vs_oracle_and_reference(glc, oracle, count, src_len):
    src = rand_elems(src_len, seed=count, noncanonical=True)
    ix = rand_indexes(count, src_len, seed=count + 1)
    want = oracle.select(ix, src)
    assert (want[(ix & PH) != 0] == 0).all() and (want[(ix & PH) == 0] == src[ix[(ix & PH) == 0]]).all()
    d_dst = zeros_dev(count)
    glc.ops_complex.select(idx_dev(ix), to_dev(src), d_dst)
    assert (from_dev(d_dst) == want).all()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refkern
    if refkern.available():
        d_ref = zeros_dev(count)
        d_ix, d_src = idx_dev(ix), to_dev(src)
        refkern.call("ref_select", d_ix.data_ptr(), d_src.data_ptr(), d_ref.data_ptr(), count, None)
        assert (from_dev(d_ref) == want).all()


@pytest.mark.parametrize("ioff,doff", [(1, 0), (0, 1), (3, 2)])
def test_select_unaligned_and_out_of_range(glc, oracle, ioff, doff):
    """4-byte and 8-byte offsets (no 16-byte vectors) and indexes past the source (read as 0)."""
    import torch
    count, src_len = 10007, 5000
    src = rand_elems(src_len, seed=ioff * 7 + doff)
    ix = rand_indexes(count, src_len, seed=ioff + 10 * doff, out_of_range=0.1)
    want = oracle.select(ix, src)
    d_ix = torch.zeros(count + ioff, dtype=torch.int32, device="cuda")
    d_ix[ioff:] = idx_dev(ix)
    d_dst = zeros_dev(count + doff)
    glc.ops_complex.select(d_ix[ioff:], to_dev(src), d_dst[doff:])
    got = from_dev(d_dst)
    assert (got[doff:] == want).all() and (got[:doff] == 0).all()


@pytest.mark.parametrize("nv,nw,nm,log_n,n_mult", [(3, 2, 1, 12, 1000), (5, 0, 0, 10, 0), (2, 3, 1, 8, 256),
                                                   (1, 1, 1, 1, 0), (16, 4, 1, 16, 40000)])
def test_trace_fill_vs_oracle(glc, oracle, nv, nw, nm, log_n, n_mult):
    n = 1 << log_n
    n_values = 3 * n + 17
    values = rand_elems(n_values, seed=nv * 100 + log_n)
    vi = rand_indexes(nv * n, n_values, seed=log_n)
    wi = rand_indexes(nw * n, n_values, seed=log_n + 1)
    mult = np.random.default_rng(log_n).integers(0, 1 << 32, size=n_mult, dtype=np.uint32)
    want = oracle.trace_fill(vi, wi, values, mult, nv, nw, nm, n)
    d_trace = zeros_dev((nv + nw + nm) * n)
    d_trace.fill_(-1)  # every element is written, padding included
    glc.trace.fill_from_remote_witness_data(idx_dev(vi), idx_dev(wi) if nw else None, to_dev(values),
                                            idx_dev(mult) if n_mult else None, d_trace, nv, nw, nm, n)
    assert (from_dev(d_trace) == want).all()


def test_trace_fill_contract(glc):
    L = glc._lib.lib()
    n = 64
    vi, vals, tr = idx_dev(np.zeros(2 * n, np.uint32)), to_dev(np.ones(10, np.uint64)), zeros_dev(3 * n)
    fill = lambda nv, nw, nm, tl, nvals=10, ml=0: L.glc_trace_fill_from_witness(
        vi.data_ptr(), nv * n, None, nw * n, vals.data_ptr(), nvals, vi.data_ptr(), ml, tr.data_ptr(), tl, nv, nw, nm,
        n, None)
    assert fill(2, 0, 1, 3 * n) == 0
    assert L.glc_trace_fill_from_witness(vi.data_ptr(), 2 * n - 1, None, 0, vals.data_ptr(), 10, None, 0,
                                         tr.data_ptr(), 3 * n, 2, 0, 1, n, None) == 1
    assert b"variable_indexes_len" in L.glc_last_error_message()
    assert fill(2, 0, 2, 4 * n) == 1 and b"multiplicity" in L.glc_last_error_message()
    assert fill(2, 0, 1, 3 * n + 1) == 1 and b"trace_len" in L.glc_last_error_message()
    assert fill(2, 0, 1, 3 * n, nvals=0) == 1 and b"witness values" in L.glc_last_error_message()
    assert fill(2, 0, 1, 3 * n, ml=n + 1) == 1 and b"multiplicities" in L.glc_last_error_message()
    assert L.glc_select(vi.data_ptr(), 2 * n, vals.data_ptr(), 10, tr.data_ptr(), 2 * n - 1, None) == 1
    assert b"dst shorter" in L.glc_last_error_message()


def test_witness_to_cap(glc, oracle):
    """Witness -> trace (fill) -> commitment on the GPU equals the oracle's fill and commitment."""
    import torch
    log_n, nv, nw, nm, log_lde, log_cap = 12, 6, 2, 1, 1, 4
    n, cols = 1 << log_n, nv + nw + nm
    values = rand_elems(5 * n, seed=99)
    vi = rand_indexes(nv * n, values.size, seed=5)
    wi = rand_indexes(nw * n, values.size, seed=6)
    mult = np.arange(n - 100, dtype=np.uint32)
    trace = oracle.trace_fill(vi, wi, values, mult, nv, nw, nm, n)
    _, _, _, want_cap = oracle.commit(trace, log_n, cols, log_lde, log_cap)
    sz = glc.CommitJob.sizes(log_n, cols, log_lde, log_cap)
    dev = lambda k: torch.zeros(sz[k], dtype=torch.int64, device="cuda")
    job = glc.CommitJob(evals=dev("evals"), log_n=log_n, cols=cols, log_lde=log_lde, log_cap=log_cap, lde=dev("lde"),
                        trees=dev("trees"), cap=dev("cap"))
    glc.trace.fill_from_remote_witness_data(idx_dev(vi), idx_dev(wi), to_dev(values), idx_dev(mult), job.evals, nv,
                                            nw, nm, n)
    glc.commit.commit(job)
    assert (from_dev(job.evals) == trace).all()
    assert (from_dev(job.cap) == want_cap).all()
