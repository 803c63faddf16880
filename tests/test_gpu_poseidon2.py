"""Poseidon2 / Merkle / bit-reverse parity: libglc against the oracle over the reference test
matrix (crates/boojum-cuda/src/poseidon2.rs:850-937, ops_complex.rs:1628-1680)."""
import numpy as np
import pytest

from conftest import canon, load_package, rand_elems
from gpu_util import from_dev, to_dev, zeros_dev

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def glc(round_constants):
    g = load_package()
    ctx = g.Context.create(12, 12)
    g.poseidon2.set_round_constants(round_constants)
    yield g
    ctx.destroy()


def test_round_constants_installed(glc):
    """After set_round_constants the device reports its constants installed."""
    assert glc.poseidon2.round_constants_installed() is True


@pytest.mark.parametrize("log_n", [0, 4, 12])
@pytest.mark.parametrize("checkpointed", [False, True])
@pytest.mark.parametrize("cols,log_rows", [(9, 1), (8, 0), (1, 0), (17, 0), (3, 3)])
def test_leaves(glc, oracle, log_n, checkpointed, cols, log_rows):
    count = 1 << log_n
    rows = 1 << log_rows
    vals = rand_elems(cols * count * rows, log_n * 10 + cols, noncanonical=True)
    want = oracle.leaves(vals, 4 * count, log_rows)
    d_vals = to_dev(vals)
    d_res = zeros_dev(4 * count)
    H = glc.GLHasher
    if not checkpointed:
        H.compute_leaf_hashes(d_vals, d_res, log_rows, False, False)
    else:
        chunk = 8  # RATE * CHUNKING columns per slab, as the reference test
        if (chunk * rows) % 8:
            pytest.skip("slab does not fill whole rate chunks")
        for c0 in range(0, cols, chunk):
            c1 = min(cols, c0 + chunk)
            slab = d_vals[c0 * count * rows:c1 * count * rows]
            H.compute_leaf_hashes(slab, d_res, log_rows, c0 != 0, c1 != cols)
    assert (canon(from_dev(d_res)) == want).all()


@pytest.mark.parametrize("log_n", [0, 4, 12, 16])
def test_nodes(glc, oracle, log_n):
    count = 1 << log_n
    vals = rand_elems(8 * count, 100 + log_n, noncanonical=True)
    d_res = zeros_dev(4 * count)
    glc.GLHasher.compute_node_hashes(to_dev(vals), d_res)
    assert (canon(from_dev(d_res)) == oracle.nodes(vals)).all()


@pytest.mark.parametrize("log_n,cols,cap_log", [(12, 9, 0), (12, 9, 4), (10, 1, 3), (17, 16, 4), (5, 3, 0), (0, 4, 0)])
def test_merkle_tree(glc, oracle, log_n, cols, cap_log):
    n = 1 << log_n
    layers = log_n - cap_log + 1
    vals = rand_elems(n * cols, 7 + log_n, noncanonical=True)
    want = oracle.build_merkle_tree(vals, 8 * n, 0, layers)
    d_res = zeros_dev(8 * n)
    glc.GLHasher.build_merkle_tree(to_dev(vals), d_res, 0, None, layers)
    assert (canon(from_dev(d_res)) == want).all()


def test_merkle_tree_rows_per_hash(glc, oracle):
    log_leaves, log_rows, cols = 10, 2, 5
    n = 1 << (log_leaves + log_rows)
    vals = rand_elems(n * cols, 5)
    want = oracle.build_merkle_tree(vals, 8 << log_leaves, log_rows, log_leaves + 1)
    d_res = zeros_dev(8 << log_leaves)
    glc.GLHasher.build_merkle_tree(to_dev(vals), d_res, log_rows, None, log_leaves + 1)
    assert (canon(from_dev(d_res)) == want).all()


def test_build_nodes_separate_buffers(glc, oracle):
    log_leaves = 11
    leaves = 1 << log_leaves
    digests = rand_elems(4 * leaves, 9)
    d_res = zeros_dev(4 * leaves)
    glc.GLHasher.build_merkle_tree_nodes(to_dev(digests), d_res, log_leaves)
    # reference recursion: layer 1 -> results[0..2L), layer 2 -> next quarter, ...
    layer, off, count = digests, 0, leaves
    got = canon(from_dev(d_res))
    for _ in range(log_leaves):
        nxt = oracle.nodes(np.ascontiguousarray(layer))
        assert (got[off:off + 2 * count] == nxt).all()
        layer, off, count = nxt, off + 2 * count, count // 2


def test_gather_rows(glc, oracle):
    src_log_rows, cols, n_idx, lr = 12, 16, 42, 1
    vals = rand_elems(cols << src_log_rows, 1)
    idx = np.random.default_rng(3).integers(0, 42, size=n_idx).astype(np.uint32)
    rows = n_idx << lr
    d_out = zeros_dev(rows * cols)
    import torch
    d_idx = torch.from_numpy(idx.view(np.int32)).cuda()
    glc.GLHasher.gather_rows(d_idx, lr, to_dev(vals), 1 << src_log_rows, cols, d_out, rows, cols)
    assert (from_dev(d_out) == oracle.gather_rows(idx, lr, vals, 1 << src_log_rows, cols)).all()


def test_gather_merkle_paths(glc, oracle):
    log_leaves, n_idx = 12, 42
    tree = rand_elems(4 << (log_leaves + 1), 2)
    idx = np.random.default_rng(4).integers(0, 1 << log_leaves, size=n_idx).astype(np.uint32)
    import torch
    d_idx = torch.from_numpy(idx.view(np.int32)).cuda()
    d_out = zeros_dev(4 * n_idx * log_leaves)
    glc.GLHasher.gather_merkle_paths(d_idx, to_dev(tree), d_out, log_leaves)
    assert (from_dev(d_out) == oracle.gather_merkle_paths(idx, tree, log_leaves)).all()


@pytest.mark.parametrize("log_rows", [0, 1, 5, 9, 10, 11, 16, 20])
def test_bit_reverse(glc, oracle, log_rows):
    n = 1 << log_rows
    cols = 3
    stride = n + 8
    x = rand_elems(cols * stride, log_rows)
    want = oracle.bit_reverse(x, log_rows, cols, src_stride=stride, dst_stride=stride)
    d_in, d_out = to_dev(x), zeros_dev(cols * stride)
    glc.ops_complex.bit_reverse(d_in, d_out, n, cols, stride, stride)
    got = from_dev(d_out)
    d_ip = to_dev(x)
    glc.ops_complex.bit_reverse_in_place(d_ip, n, cols, stride)
    got_ip = from_dev(d_ip)
    for c in range(cols):
        sl = slice(c * stride, c * stride + n)
        assert (got[sl] == want[c * stride:c * stride + n]).all()
        assert (got_ip[sl] == want[c * stride:c * stride + n]).all()


def test_contract_violations(glc):
    H = glc.GLHasher
    with pytest.raises(glc.GlcError):
        H.compute_leaf_hashes(zeros_dev(10), zeros_dev(6), 0, False, False)  # results_len % 4
    with pytest.raises(glc.GlcError):
        H.compute_leaf_hashes(zeros_dev(10), zeros_dev(8), 0, False, True)  # slab not a multiple of 8
    with pytest.raises(glc.GlcError):
        H.compute_node_hashes(zeros_dev(16), zeros_dev(4), None)
    with pytest.raises(glc.GlcError):
        H.build_merkle_tree(zeros_dev(16), zeros_dev(16), 0, None, 0)
    with pytest.raises(glc.GlcError):
        H.build_merkle_tree(zeros_dev(16), zeros_dev(16), 0, None, 3)  # 2^(layers-1) > leaves


def test_nodes_unaligned_input(glc, oracle):
    """A digest layer that starts 8 bytes past a 16-byte boundary takes the 8-byte load path."""
    count = 1 << 9
    vals = rand_elems(8 * count + 1, 5)
    d = to_dev(vals)
    d_res = zeros_dev(4 * count)
    glc.GLHasher.compute_node_hashes(d[1:], d_res)
    assert (canon(from_dev(d_res)) == oracle.nodes(np.ascontiguousarray(vals[1:]))).all()
    d_tree = zeros_dev(8 * count)
    glc.GLHasher.build_merkle_tree_nodes(d[1:], d_tree, 3)
    got = canon(from_dev(d_tree))
    l1 = oracle.nodes(np.ascontiguousarray(vals[1:]))
    l2 = oracle.nodes(l1)
    assert (got[:4 * count] == l1).all() and (got[4 * count:6 * count] == l2).all()
