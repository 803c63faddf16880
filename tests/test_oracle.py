"""CPU checks of the oracle itself: the C restatement against the definitions (pure Python,
O(n^2)), against a second restatement of the Poseidon2 permutation in Python, and against the
reference's layouts.  Golden vectors produced by the reference's own kernels are checked in
test_golden.py."""
import numpy as np
import pytest

from conftest import P, canon, rand_elems


def brev(x, bits):
    return int(format(x, "0%db" % bits)[::-1], 2) if bits else 0


def py_ntt(vals, log_n, bitrev_inputs, inverse, log_ext, coset):
    """Definitions of crates/boojum-cuda/src/ntt.rs:527-583 in Python integers."""
    n = 1 << log_n
    w = pow(7, (P - 1) >> log_n, P)
    s = 1
    if log_ext:
        s = 7 * pow(pow(7, (P - 1) >> (log_n + log_ext), P), coset, P) % P
    x = [int(vals[brev(j, log_n)] if bitrev_inputs else vals[j]) % P for j in range(n)]
    if not inverse:
        y = [sum(x[j] * pow(s * pow(w, i, P) % P, j, P) for j in range(n)) % P for i in range(n)]
    else:
        wi, si, ni = pow(w, P - 2, P), pow(s, P - 2, P), pow(n, P - 2, P)
        y = [sum(x[j] * pow(wi, i * j, P) for j in range(n)) * ni * pow(si, i, P) % P for i in range(n)]
    return [y[i if bitrev_inputs else brev(i, log_n)] for i in range(n)]


@pytest.mark.parametrize("log_n", [1, 2, 3, 4])
@pytest.mark.parametrize("bitrev_inputs", [False, True])
@pytest.mark.parametrize("inverse", [False, True])
@pytest.mark.parametrize("log_ext,coset", [(0, 0), (1, 0), (1, 1), (3, 3)])
def test_ntt_definitions(oracle, log_n, bitrev_inputs, inverse, log_ext, coset):
    n = 1 << log_n
    x = rand_elems(n, 1000 + log_n, noncanonical=True)
    got = oracle.batch_ntt(x, log_n, 1, n, n, bitrev_inputs, inverse, log_ext, coset)
    assert [int(v) for v in got] == py_ntt(x, log_n, bitrev_inputs, inverse, log_ext, coset)


@pytest.mark.parametrize("log_n", list(range(1, 9)))
def test_ntt_fast_vs_direct(oracle, log_n):
    n = 1 << log_n
    num, stride = 3, 2 * n
    for bitrev_inputs in (0, 1):
        for inverse in (0, 1):
            for log_ext, coset in ((0, 0), (2, 1), (3, 5)):
                x = rand_elems(num * stride, log_n * 100 + bitrev_inputs * 10 + inverse)
                a = oracle.batch_ntt(x, log_n, num, stride, stride, bitrev_inputs, inverse, log_ext, coset)
                b = oracle.batch_ntt(x, log_n, num, stride, stride, bitrev_inputs, inverse, log_ext, coset, naive=True)
                for k in range(num):
                    assert (a[k * stride:k * stride + n] == b[k * stride:k * stride + n]).all()


@pytest.mark.parametrize("log_n", [5, 12, 16])
def test_ntt_round_trips(oracle, log_n):
    n = 1 << log_n
    x = rand_elems(n, log_n)
    # forward n2b then inverse b2n is the identity
    y = oracle.batch_ntt(x, log_n, 1, n, n, 0, 0, 0, 0)
    z = oracle.batch_ntt(y, log_n, 1, n, n, 1, 1, 0, 0)
    assert (z == x).all()
    # coset LDE: forward on coset c then inverse on the same coset is the identity
    y = oracle.batch_ntt(x, log_n, 1, n, n, 0, 0, 2, 3)
    z = oracle.batch_ntt(y, log_n, 1, n, n, 1, 1, 2, 3)
    assert (z == x).all()
    # n2b output is the bit reversal of b2n output on the bit-reversed input
    y1 = oracle.batch_ntt(x, log_n, 1, n, n, 0, 0, 1, 1)
    y2 = oracle.batch_ntt(oracle.bit_reverse(x, log_n, 1), log_n, 1, n, n, 1, 0, 1, 1)
    assert (oracle.bit_reverse(y2, log_n, 1) == y1).all()


def test_ntt_contract(oracle):
    x = np.zeros(16, dtype=np.uint64)
    with pytest.raises(ValueError):
        oracle.batch_ntt(x, 0, 1, 16, 16, 0, 0, 0, 0)  # log_n >= 1
    with pytest.raises(ValueError):
        oracle.batch_ntt(x, 4, 1, 16, 16, 0, 0, 0, 1)  # coset without extension
    with pytest.raises(ValueError):
        oracle.batch_ntt(x, 4, 1, 8, 16, 0, 0, 0, 0)  # n > stride
    with pytest.raises(ValueError):
        oracle.batch_ntt(x, 4, 1, 16, 16, 0, 0, 1, 2)  # coset >= 2^log_ext


def test_bit_reverse(oracle):
    for log_n in (0, 1, 3, 10, 11):
        n = 1 << log_n
        x = rand_elems(2 * n + 3, log_n)
        y = oracle.bit_reverse(x, log_n, 2, src_stride=n + 1)
        for c in range(2):
            for i in range(n):
                assert y[c * n + i] == x[c * (n + 1) + brev(i, log_n)]


# ---- Poseidon2: second restatement in pure Python (poseidon2_gl_st.cu:9-23, *_st.cuh) ----

LOG_MU = [4, 14, 11, 8, 0, 5, 2, 9, 13, 6, 3, 12]
M4 = [[5, 7, 1, 3], [4, 6, 1, 1], [1, 3, 5, 7], [1, 1, 4, 6]]


def py_permutation(state, rc):
    s = [int(v) % P for v in state]

    def ext(s):
        t = [sum(M4[r][c] * s[4 * q + c] for c in range(4)) for q in range(3) for r in range(4)]
        acc = [t[j] + t[4 + j] + t[8 + j] for j in range(4)]
        return [(t[i] + acc[i % 4]) % P for i in range(12)]

    def internal(s):
        tot = sum(s)
        return [(tot + (s[i] << LOG_MU[i])) % P for i in range(12)]

    s = ext(s)
    for r in range(30):
        if r < 4 or r >= 26:
            s = [pow((s[i] + rc[12 * r + i]) % P, 7, P) for i in range(12)]
            s = ext(s)
        else:
            s[0] = pow((s[0] + rc[12 * r]) % P, 7, P)
            s = internal(s)
    return s


def test_m4_matches_addition_chain(oracle):
    # the matrix used above is the one the reference's addition chain computes (poseidon2_gl.cuh:11-25)
    for _ in range(4):
        x = [int(v) for v in rand_elems(4, _)]
        t0 = x[0] + x[1]; t1 = x[2] + x[3]; t2 = 2 * x[1] + t1; t3 = 2 * x[3] + t0
        t4 = 4 * t1 + t3; t5 = 4 * t0 + t2
        chain = [t3 + t5, t5, t2 + t4, t4]
        assert chain == [sum(M4[r][c] * x[c] for c in range(4)) for r in range(4)]


def test_permutation_two_restatements(oracle, round_constants):
    for seed in range(6):
        st = rand_elems(12, 50 + seed, noncanonical=seed % 2 == 1)
        assert [int(v) for v in oracle.permutation(st)] == py_permutation(st, round_constants)


def py_leaf(values, count, log_rows, i, rc, capacity=None, want_capacity=False):
    rows = 1 << log_rows
    cols = len(values) // (count * rows)
    seq = [int(values[(i << log_rows) + r + c * rows * count]) for c in range(cols) for r in range(rows)]
    s = [0] * 8 + (list(capacity) if capacity is not None else [0] * 4)
    for off in range(0, len(seq), 8):
        chunk = seq[off:off + 8]
        s[:8] = chunk + [0] * (8 - len(chunk))
        s = py_permutation(s, rc)
    return s[8:12] if want_capacity else s[:4]


@pytest.mark.parametrize("cols,log_rows,count", [(9, 1, 16), (8, 0, 32), (1, 0, 8), (3, 2, 4), (16, 0, 4)])
def test_leaves_layout(oracle, round_constants, cols, log_rows, count):
    vals = rand_elems(cols * count << log_rows, cols * 7 + log_rows)
    res = oracle.leaves(vals, 4 * count, log_rows)
    for i in range(count):
        d = py_leaf(vals, count, log_rows, i, round_constants)
        assert [int(res[j * count + i]) for j in range(4)] == d


def test_leaves_checkpointed_equals_whole(oracle):
    # compute_leaf_hashes in column slabs of 8 with load/store of the capacity (poseidon2.rs:645-659)
    count, log_rows, cols = 64, 1, 9
    rows = 1 << log_rows
    vals = rand_elems(cols * count * rows, 77)
    whole = oracle.leaves(vals, 4 * count, log_rows)
    res = np.zeros(4 * count, dtype=np.uint64)
    for c0 in range(0, cols, 8):
        c1 = min(cols, c0 + 8)
        slab = np.ascontiguousarray(vals[c0 * count * rows:c1 * count * rows])
        oracle.leaves(slab, 4 * count, log_rows, load_intermediate=c0 != 0, store_intermediate=c1 != cols, results=res)
    assert (res == whole).all()


def test_nodes_and_tree(oracle, round_constants):
    log_leaves = 6
    leaves = 1 << log_leaves
    vals = rand_elems(3 * leaves, 5)
    tree = oracle.build_merkle_tree(vals, 8 * leaves, 0, log_leaves + 1)
    layer = tree[:4 * leaves]
    assert (layer == oracle.leaves(vals, 4 * leaves, 0)).all()
    off, count = 4 * leaves, leaves
    while count > 1:
        nxt = tree[off:off + 2 * count]
        half = count // 2
        for i in range(half):
            s = [int(layer[k * count + 2 * i]) for k in range(4)] + [int(layer[k * count + 2 * i + 1]) for k in range(4)]
            d = py_permutation(s + [0] * 4, round_constants)[:4]
            assert [int(nxt[k * half + i]) for k in range(4)] == d
        assert (nxt == oracle.nodes(np.ascontiguousarray(layer))).all()
        layer, off, count = nxt, off + 2 * count, half
    assert (tree[off:] == 0).all()  # the unused tail of the results buffer


def test_tree_partial_layers(oracle):
    leaves = 32
    vals = rand_elems(2 * leaves, 9)
    full = oracle.build_merkle_tree(vals, 8 * leaves, 0, 6)
    part = oracle.build_merkle_tree(vals, 8 * leaves, 0, 3)  # cap of 8
    n = 4 * leaves + 2 * leaves + leaves
    assert (part[:n] == full[:n]).all() and (part[n:] == 0).all()


def test_gathers(oracle):
    src_log_rows, cols, n_idx, lr = 8, 5, 11, 1
    vals = rand_elems(cols << src_log_rows, 3)
    idx = np.random.default_rng(1).integers(0, (1 << src_log_rows) >> lr, size=n_idx).astype(np.uint32)
    out = oracle.gather_rows(idx, lr, vals, 1 << src_log_rows, cols)
    rows = n_idx << lr
    for i, ix in enumerate(idx):
        for j in range(1 << lr):
            for k in range(cols):
                assert out[k * rows + i * 2 + j] == vals[(k << src_log_rows) + (int(ix) << lr) + j]
    log_leaves, layers = 6, 6
    tree = rand_elems(4 << (log_leaves + 1), 4)
    idx = np.random.default_rng(2).integers(0, 1 << log_leaves, size=n_idx).astype(np.uint32)
    paths = oracle.gather_merkle_paths(idx, tree, layers)
    off, count = 0, 1 << log_leaves
    for layer in range(layers):
        for k in range(4):
            for i, ix in enumerate(idx):
                sib = (int(ix) >> layer) ^ 1
                assert paths[layer * n_idx * 4 + n_idx * k + i] == tree[off + k * count + sib]
        off += 4 * count
        count //= 2


def test_commit_matches_steps(oracle):
    """or_commit == iNTT, bit reverse, per-coset LDE (coset bitrev(c)) and per-coset subtrees."""
    log_n, cols, log_lde, log_cap = 6, 3, 1, 2
    n = 1 << log_n
    ev = rand_elems(cols * n, 21)
    mono, lde, trees, cap = oracle.commit(ev, log_n, cols, log_lde, log_cap)
    m2 = oracle.bit_reverse(oracle.batch_ntt(ev, log_n, cols, n, n, 0, 1, 0, 0), log_n, cols)
    assert (mono == m2).all()
    # monomials evaluate back to the evaluations
    assert (oracle.batch_ntt(mono, log_n, cols, n, n, 0, 0, 0, 0) == oracle.bit_reverse(ev, log_n, cols)).all()
    for c in range(1 << log_lde):
        l2 = oracle.batch_ntt(mono, log_n, cols, n, n, 0, 0, log_lde, brev(c, log_lde))
        assert (lde[c * cols * n:(c + 1) * cols * n] == l2).all()
        t2 = oracle.build_merkle_tree(l2, 8 * n, 0, log_n - (log_cap - log_lde) + 1)
        assert (trees[c * 8 * n:(c + 1) * 8 * n] == t2).all()
    # the cap equals the cap of ONE tree over the coset-major leaves
    all_leaves = np.concatenate([lde[c * cols * n:(c + 1) * cols * n].reshape(cols, n) for c in range(2)], axis=1)
    big = oracle.build_merkle_tree(np.ascontiguousarray(all_leaves.reshape(-1)), 8 * 2 * n, 0, log_n + 1 - log_cap + 2)
    cap_off = 8 * 2 * n - 8 * (1 << log_cap)
    assert (big[cap_off:cap_off + 4 * (1 << log_cap)] == cap).all()


def test_extension_layouts(oracle):
    # vectorized column k = base columns 2k (c0) and 2k+1 (c1), stride 7; tuples stride 5
    # (memory.cuh:545-612 accessors: c1 sits one stride after c0, a column step is two strides)
    v = np.arange(2 * 3 * 7, dtype=np.uint64)
    t = oracle.ef_vectorized_to_tuples(v, 7, 5, 3, 5)
    want = []
    for k in range(3):
        for r in range(5):
            want += [2 * k * 7 + r, (2 * k + 1) * 7 + r]
    assert t.tolist() == want
    back = oracle.ef_tuples_to_vectorized(t, 5, 5, 3, 7).reshape(6, 7)
    assert (back[:, :5] == v.reshape(6, 7)[:, :5]).all() and (back[:, 5:] == 0).all()


def test_select_and_trace_fill(oracle):
    """select: src[index], 0 for a placeholder (bit 31) or an index past the source; the trace fill
    is the variable selects, the witness selects and the zero-padded multiplicities, in that order
    (ops_complex.cu:158-164, trace.rs:108-193), restated here in numpy."""
    rng = np.random.default_rng(3)
    src = rng.integers(0, 2**64, size=300, dtype=np.uint64)
    ix = rng.integers(0, 350, size=4000, dtype=np.uint32)
    ix[::9] |= np.uint32(1 << 31)
    sel = lambda i: np.where(((i >> 31) == 0) & (i < src.size), src[np.minimum(i & 0x7FFFFFFF, src.size - 1)], 0)
    assert (oracle.select(ix, src) == sel(ix)).all()
    n, nv, nw = 64, 3, 2
    vi, wi = ix[:nv * n], ix[nv * n:(nv + nw) * n]
    mult = rng.integers(0, 2**32, size=40, dtype=np.uint32)
    got = oracle.trace_fill(vi, wi, src, mult, nv, nw, 1, n)
    want = np.concatenate([sel(vi), sel(wi), mult.astype(np.uint64), np.zeros(n - 40, np.uint64)])
    assert (got == want).all()
    assert (oracle.trace_fill(vi, None, src, None, nv, 0, 0, n) == sel(vi)).all()
