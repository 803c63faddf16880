"""NTT / LDE parity: libglc (sm_100a) against the oracle, bit-exact after canonicalisation,
over the reference test matrix (crates/boojum-cuda/src/ntt.rs:613-663): sizes 2^1..2^24, n2b and
b2n, forward and inverse, plain and coset LDE, in place and out of place, column strides with
an offset, 19 columns (two full 8-column groups plus a tail)."""
import numpy as np
import pytest

from conftest import canon, load_package, rand_elems
from gpu_util import from_dev, to_dev, zeros_dev

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def glc():
    g = load_package()
    ctx = g.Context.create(12, 12)
    yield g
    ctx.destroy()


def run_case(glc, oracle, log_n, num, inverse, log_ext, coset, seed):
    n = 1 << log_n
    off = n  # OFFSET_MULTIPLIER = 1
    stride = 2 * n
    x = rand_elems(num * stride, seed, noncanonical=True)
    xb = x.copy()
    for k in range(num):  # bit-reversed copy of each column for the b2n cases
        xb[k * stride + off:k * stride + off + n] = oracle.bit_reverse(x[k * stride + off:k * stride + off + n], log_n, 1)
    exp = np.zeros_like(x)
    for k in range(num):
        col = np.ascontiguousarray(x[k * stride + off:k * stride + off + n])
        exp[k * stride + off:k * stride + off + n] = oracle.batch_ntt(col, log_n, 1, n, n, 0, inverse, log_ext, coset)
    for bitrev_inputs in (False, True):
        src = xb if bitrev_inputs else x
        # in place
        d = to_dev(src)
        glc.ntt.batch_ntt_in_place(d, log_n, num, off, stride, bitrev_inputs, inverse, log_ext, coset)
        got_ip = from_dev(d)
        # out of place
        d_in = to_dev(src)
        d_out = zeros_dev(num * stride)
        glc.ntt.batch_ntt_out_of_place(d_in, d_out, log_n, num, off, off, stride, stride, bitrev_inputs, inverse,
                                       log_ext, coset)
        got_op = from_dev(d_out)
        assert (from_dev(d_in) == src).all(), "out-of-place call modified its input"
        for k in range(num):
            sl = slice(k * stride + off, k * stride + off + n)
            want = exp[sl] if not bitrev_inputs else oracle.bit_reverse(exp[sl], log_n, 1)
            assert (canon(got_ip[sl]) == want).all(), ("in place", log_n, bitrev_inputs, inverse, log_ext, coset, k)
            assert (canon(got_op[sl]) == want).all(), ("out of place", log_n, bitrev_inputs, inverse, log_ext, coset, k)
            # the region before the offset is untouched
            assert (got_op[k * stride:k * stride + off] == 0).all()


@pytest.mark.parametrize("log_n", list(range(1, 17)))
@pytest.mark.parametrize("inverse,log_ext,coset", [(False, 0, 0), (False, 3, 3), (True, 0, 0), (True, 3, 3)])
def test_ntt_small(glc, oracle, log_n, inverse, log_ext, coset):
    num = 19 if not (inverse or log_ext) else (1 if inverse and not log_ext else 3)
    run_case(glc, oracle, log_n, num, inverse, log_ext, coset, seed=log_n * 31 + inverse * 7 + log_ext)


@pytest.mark.parametrize("log_n", [17, 18, 19, 20, 21, 22, 23, 24])
@pytest.mark.parametrize("inverse,log_ext,coset", [(False, 0, 0), (False, 3, 3), (True, 0, 0), (True, 3, 3)])
def test_ntt_large(glc, oracle, log_n, inverse, log_ext, coset):
    run_case(glc, oracle, log_n, 2 if log_n < 23 else 1, inverse, log_ext, coset, seed=log_n * 131 + inverse)


@pytest.mark.parametrize("log_n", [5, 13, 18])
@pytest.mark.parametrize("bitrev_inputs,inverse,log_ext,coset", [(False, False, 1, 1), (False, True, 0, 0),
                                                                 (True, False, 2, 3), (False, False, 0, 0)])
def test_odd_stride_and_offset(glc, oracle, log_n, bitrev_inputs, inverse, log_ext, coset):
    # an odd element offset and an odd stride: the 16-byte load/store path does not apply, the
    # 8-byte one runs (and must agree)
    n = 1 << log_n
    num, off, stride = 3, 1, n + 3
    x = rand_elems(num * stride, log_n + 7 * coset, noncanonical=True)
    d_in, d_out = to_dev(x), zeros_dev(num * stride)
    glc.ntt.batch_ntt_out_of_place(d_in, d_out, log_n, num, off, off, stride, stride, bitrev_inputs, inverse,
                                   log_ext, coset)
    got = from_dev(d_out)
    for k in range(num):
        sl = slice(k * stride + off, k * stride + off + n)
        col = np.ascontiguousarray(x[sl])
        want = oracle.batch_ntt(col, log_n, 1, n, n, int(bitrev_inputs), int(inverse), log_ext, coset)
        assert (canon(got[sl]) == want).all(), (log_n, k)


def test_lde_cosets_every_index(glc, oracle):
    log_n, log_ext = 10, 2
    n = 1 << log_n
    x = rand_elems(5 * n, 3)
    for coset in range(1 << log_ext):
        d_in, d_out = to_dev(x), zeros_dev(5 * n)
        glc.ntt.batch_ntt_out_of_place(d_in, d_out, log_n, 5, 0, 0, n, n, False, False, log_ext, coset)
        assert (canon(from_dev(d_out)) == oracle.batch_ntt(x, log_n, 5, n, n, 0, 0, log_ext, coset)).all()


@pytest.mark.parametrize("log_n", [12, 20, 24])
def test_round_trip_full_size(glc, log_n):
    """Size-independent property at full size: iNTT(NTT(x)) == x for the coset LDE pair."""
    n = 1 << log_n
    cols = max(1, (1 << 24) >> log_n)
    x = rand_elems(cols * n, log_n)
    d = to_dev(x)
    glc.ntt.batch_ntt_in_place(d, log_n, cols, 0, n, False, False, 1, 1)
    glc.ntt.batch_ntt_in_place(d, log_n, cols, 0, n, True, True, 1, 1)
    assert (canon(from_dev(d)) == x).all()


def test_contract_violations(glc):
    d = zeros_dev(64)
    e = zeros_dev(64)
    with pytest.raises(glc.GlcError):
        glc.ntt.batch_ntt_in_place(d, 0, 1, 0, 64, False, False, 0, 0)
    with pytest.raises(glc.GlcError):
        glc.ntt.batch_ntt_in_place(d, 6, 2, 0, 64, False, False, 0, 0)  # len < num * stride
    with pytest.raises(glc.GlcError):
        glc.ntt.batch_ntt_in_place(d, 5, 1, 0, 32, False, False, 0, 1)  # coset without extension
    with pytest.raises(glc.GlcError):
        glc.ntt.batch_ntt_out_of_place(d, d, 5, 1, 0, 0, 32, 32, False, False, 0, 0)  # same matrix
    with pytest.raises(glc.GlcError):
        glc.ntt.batch_ntt_out_of_place(d, e, 5, 1, 16, 0, 32, 32, False, False, 0, 0)  # offset + n > stride
    with pytest.raises(glc.GlcError):
        glc.ntt.batch_ntt_in_place(d, 25, 1, 0, 1 << 25, False, False, 0, 0)
