"""The small, CPU-runnable configuration of the benchmark set, end to end through the
boojum-cuda-shaped API on the GPU: one Goldilocks column of 2^16 seeded ChaCha elements, forward
NTT then inverse NTT in natural order (bit-exact round trip); LDE by factor 2 on the coset of the
generator 7 with bit-reversed output; a Poseidon2 Merkle tree over the 2^17 LDE rows of 8 such
columns with cap 16.  Every stage is compared with the oracle."""
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


def test_small_configuration(glc, oracle):
    import torch
    log_n, cols, log_cap = 16, 8, 4
    n = 1 << log_n
    x = load_synthetic().random_field_elements("small-configuration", cols * n)
    # forward NTT (natural in, bit-reversed out) then inverse NTT (bit-reversed in, natural out)
    d_x, d_y = to_dev(x[:n]), zeros_dev(n)
    glc.ntt.batch_ntt_out_of_place(d_x, d_y, log_n, 1, 0, 0, n, n, False, False, 0, 0)
    fwd = canon(from_dev(d_y))
    assert (fwd == oracle.batch_ntt(x[:n], log_n, 1, n, n, False, False, 0, 0)).all()
    glc.ntt.batch_ntt_in_place(d_y, log_n, 1, 0, n, True, True, 0, 0)
    assert (canon(from_dev(d_y)) == x[:n]).all()
    # LDE x2 of the 8 columns on g = 7 cosets, bit-reversed: the commitment's LDE
    sz = glc.CommitJob.sizes(log_n, cols, 1, log_cap)
    dev = lambda k: torch.zeros(sz[k], dtype=torch.int64, device="cuda")
    job = glc.CommitJob(evals=to_dev(x), log_n=log_n, cols=cols, log_lde=1, log_cap=log_cap, lde=dev("lde"),
                        trees=dev("trees"), cap=dev("cap"))
    glc.commit.commit(job)
    _, want_lde, _, _ = oracle.commit(x, log_n, cols, 1, log_cap)
    lde = canon(from_dev(job.lde))
    assert (lde == want_lde).all()
    # the 2^17-row matrix over the whole LDE domain in bit-reversed order: coset 0 then coset 1
    # (bit-reversed position i < 2^16 is an even power, i.e. coset 0), column by column
    m = lde.reshape(2, cols, n).transpose(1, 0, 2).reshape(cols * 2 * n).copy()
    layers = (log_n + 1) - log_cap + 1
    want_tree = oracle.build_merkle_tree(m, 8 * 2 * n, 0, layers)
    d_tree = zeros_dev(8 * 2 * n)
    glc.GLHasher.build_merkle_tree(to_dev(m), d_tree, 0, None, layers)
    tree = canon(from_dev(d_tree))
    assert (tree == want_tree).all()
    # the cap: the 16 digests of the last layer ([4][16] at the end of the written layers)
    total = sum((4 * 2 * n) >> l for l in range(layers))
    assert (tree[total - 4 * 16:total] == want_tree[total - 4 * 16:total]).all()
