"""GoldilocksExt2 layout conversions (extension_field.rs:60-90 semantics) against the oracle."""
import numpy as np
import pytest

from conftest import load_package, rand_elems
from gpu_util import from_dev, to_dev, zeros_dev

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def glc():
    return load_package()


@pytest.mark.parametrize("rows,cols,v_stride,t_stride", [(1, 1, 1, 1), (7, 3, 9, 8), (1024, 5, 1024, 1024),
                                                         (1000, 4, 1001, 1003), (1 << 16, 2, 1 << 16, 1 << 16),
                                                         (4097, 1, 4098, 4097)])
def test_vectorized_tuples_round_trip(glc, oracle, rows, cols, v_stride, t_stride):
    v = rand_elems(2 * cols * v_stride, seed=rows + cols)
    want_t = oracle.ef_vectorized_to_tuples(v, v_stride, rows, cols, t_stride)
    d_t = zeros_dev(2 * cols * t_stride)
    glc.extension_field.vectorized_to_tuples(to_dev(v), d_t, rows, cols, v_stride, t_stride)
    got_t = from_dev(d_t)
    assert (got_t == want_t).all()
    d_v = zeros_dev(2 * cols * v_stride)
    glc.extension_field.tuples_to_vectorized(d_t, d_v, rows, cols, t_stride, v_stride)
    assert (from_dev(d_v) == oracle.ef_tuples_to_vectorized(want_t, t_stride, rows, cols, v_stride)).all()
    # the rows of every column came back unchanged
    got_v = from_dev(d_v).reshape(2 * cols, v_stride)[:, :rows]
    assert (got_v == v.reshape(2 * cols, v_stride)[:, :rows]).all()


def test_contract_violations(glc):
    L = glc._lib.lib()
    buf = zeros_dev(64)
    assert L.glc_ef_vectorized_to_tuples(buf.data_ptr(), 4, buf.data_ptr() + 8, 8, 8, 1, None) == 1  # stride < rows
    assert b"stride" in L.glc_last_error_message()
    assert L.glc_ef_vectorized_to_tuples(buf.data_ptr(), 8, buf.data_ptr() + 8, 8, 8, 1, None) == 1  # misaligned
    assert b"aligned" in L.glc_last_error_message()
    assert L.glc_ef_tuples_to_vectorized(buf.data_ptr(), 8, buf.data_ptr(), 8, 0, 3, None) == 0  # empty
