"""libglc against the REFERENCE's own kernels (crates/boojum-cuda/native compiled for sm_100a,
oracle/_ref/libbcref.so) on the same inputs, same twiddle definition and same round constants:
the product must reproduce the reference bit for bit (after canonicalisation)."""
import numpy as np
import pytest

from conftest import canon, load_package, rand_elems
from gpu_util import from_dev, to_dev, zeros_dev

pytestmark = pytest.mark.gpu

refkern = pytest.importorskip("refkern")
if not refkern.available():
    pytest.skip("reference kernels not built (oracle/build_ref.py)", allow_module_level=True)


@pytest.fixture(scope="module")
def both(round_constants):
    import torch
    g = load_package()
    ctx = g.Context.create(12, 12)
    g.poseidon2.set_round_constants(round_constants)
    refkern.call("ref_context_create", 12, 12)
    yield g, torch.cuda.current_stream().cuda_stream
    refkern.call("ref_context_destroy")
    ctx.destroy()


@pytest.mark.parametrize("log_n", [1, 4, 9, 12, 13, 15, 16, 18, 20, 21, 22, 24])
@pytest.mark.parametrize("bitrev_inputs", [False, True])
@pytest.mark.parametrize("inverse,log_ext,coset", [(False, 0, 0), (True, 0, 0), (False, 2, 1), (True, 2, 3)])
def test_ntt_vs_reference(both, log_n, bitrev_inputs, inverse, log_ext, coset):
    g, s = both
    n = 1 << log_n
    cols = max(1, min(11, (1 << 22) >> log_n))
    x = rand_elems(cols * n, log_n * 7 + bitrev_inputs, noncanonical=True)
    d_in = to_dev(x)
    d_ref, d_ours = zeros_dev(cols * n), zeros_dev(cols * n)
    refkern.call("ref_batch_ntt", d_in.data_ptr(), d_ref.data_ptr(), log_n, cols, n, n, bitrev_inputs, inverse, log_ext,
                 coset, s)
    g.ntt.batch_ntt_out_of_place(d_in, d_ours, log_n, cols, 0, 0, n, n, bitrev_inputs, inverse, log_ext, coset)
    assert (canon(from_dev(d_ours)) == canon(from_dev(d_ref))).all()


@pytest.mark.parametrize("log_rows", [3, 10, 11, 14])
def test_bitrev_vs_reference(both, log_rows):
    g, s = both
    n = 1 << log_rows
    x = rand_elems(4 * n, log_rows)
    d_in, d_ref, d_ours = to_dev(x), zeros_dev(4 * n), zeros_dev(4 * n)
    refkern.call("ref_bit_reverse", d_in.data_ptr(), n, d_ref.data_ptr(), n, log_rows, 4, s)
    g.ops_complex.bit_reverse(d_in, d_ours, n, 4)
    assert (from_dev(d_ours) == from_dev(d_ref)).all()


@pytest.mark.parametrize("log_n,cols,log_rows", [(4, 9, 1), (12, 9, 1), (14, 16, 0), (16, 3, 0), (5, 130, 0)])
def test_leaves_vs_reference(both, log_n, cols, log_rows):
    g, s = both
    count = 1 << log_n
    x = rand_elems(cols * count << log_rows, log_n + cols, noncanonical=True)
    d_in, d_ref, d_ours = to_dev(x), zeros_dev(4 * count), zeros_dev(4 * count)
    refkern.call("ref_p2_leaves", d_in.data_ptr(), x.size, d_ref.data_ptr(), 4 * count, log_rows, False, False, s)
    g.GLHasher.compute_leaf_hashes(d_in, d_ours, log_rows, False, False)
    assert (canon(from_dev(d_ours)) == canon(from_dev(d_ref))).all()


@pytest.mark.parametrize("log_n,cols,cap_log", [(12, 9, 0), (16, 8, 4), (18, 4, 3)])
def test_tree_vs_reference(both, log_n, cols, cap_log):
    g, s = both
    n = 1 << log_n
    layers = log_n - cap_log + 1
    x = rand_elems(cols * n, log_n, noncanonical=True)
    d_in, d_ref, d_ours = to_dev(x), zeros_dev(8 * n), zeros_dev(8 * n)
    refkern.call("ref_p2_build_merkle_tree", d_in.data_ptr(), x.size, d_ref.data_ptr(), 8 * n, 0, layers, s)
    g.GLHasher.build_merkle_tree(d_in, d_ours, 0, None, layers)
    assert (canon(from_dev(d_ours)) == canon(from_dev(d_ref))).all()


def test_gathers_vs_reference(both):
    import torch
    g, s = both
    log_leaves, n_idx = 12, 42
    tree = rand_elems(4 << (log_leaves + 1), 2)
    idx = np.random.default_rng(4).integers(0, 1 << log_leaves, size=n_idx).astype(np.uint32)
    d_idx = torch.from_numpy(idx.view(np.int32)).cuda()
    d_tree = to_dev(tree)
    d_ref, d_ours = zeros_dev(4 * n_idx * log_leaves), zeros_dev(4 * n_idx * log_leaves)
    refkern.call("ref_p2_gather_merkle_paths", d_idx.data_ptr(), n_idx, d_tree.data_ptr(), tree.size, d_ref.data_ptr(),
                 log_leaves, s)
    g.GLHasher.gather_merkle_paths(d_idx, d_tree, d_ours, log_leaves)
    assert (from_dev(d_ours) == from_dev(d_ref)).all()
    vals = rand_elems(16 << 12, 1)
    ridx = (idx % 2048).astype(np.uint32)
    d_ridx = torch.from_numpy(ridx.view(np.int32)).cuda()
    rows = n_idx << 1
    d_v = to_dev(vals)
    d_ref, d_ours = zeros_dev(rows * 16), zeros_dev(rows * 16)
    refkern.call("ref_p2_gather_rows", d_ridx.data_ptr(), n_idx, 1, d_v.data_ptr(), 1 << 12, d_ref.data_ptr(), rows, 16, s)
    g.GLHasher.gather_rows(d_ridx, 1, d_v, 1 << 12, 16, d_ours, rows, 16)
    assert (from_dev(d_ours) == from_dev(d_ref)).all()
