"""Rows of the operator evaluated densely (mlfma_dense_rows), the FP64 dense
reference for the error of a product: against the oracle's dense block, against
the product of an operator whose every interaction is near, and the MLFMA
error it measures on a sphere with a far field."""
import numpy as np
import pytest

from mlfma_b200 import MLFMA, MlfmaError, inputs
from mlfma_b200 import _lib
from oracle import mlfma_oracle as O

pytestmark = pytest.mark.gpu
PW = inputs.PlaneWave()


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def cvec(n, seed):
    r = np.random.default_rng(seed)
    return r.standard_normal(n) + 1j * r.standard_normal(n)


@pytest.mark.parametrize("self_terms", [0, 1])
def test_dense_rows_dipoles_match_oracle(cuda_device, self_terms):
    d = inputs.make_dipoles(2000, seed=41)
    op = MLFMA.dipoles(d, PW, max_node_srcs=16, self_terms=self_terms, ref_compat=1 - self_terms).setup()
    src = O.DipoleSources(d.pos, d.mom, PW)
    src.self_terms = bool(self_terms)
    rows = np.random.default_rng(3).choice(op.n, 48, replace=False)
    x = cvec(op.n, 4)
    ref = O.PHYS_C * PW.wavenum * (src.block(rows, np.arange(op.n), PW.wavenum) @ x)
    assert rel(op.dense_rows(rows, x), ref) <= 1e-12
    op.close()


@pytest.mark.parametrize("self_terms", [0, 1])
def test_dense_rows_rwg_match_oracle(cuda_device, self_terms):
    m = inputs.make_icosphere(2, radius=0.6)
    op = MLFMA.rwg(m, PW, max_node_srcs=16, self_terms=self_terms, ref_compat=1 - self_terms).setup()
    src = O.RWGSources(m.vertices, m.faces, m.rwgs, PW, quad_prec=2)
    src.self_terms = bool(self_terms)
    rows = np.random.default_rng(5).choice(op.n, 24, replace=False)
    x = cvec(op.n, 6)
    ref = O.PHYS_C * PW.wavenum * (src.block(rows, np.arange(op.n), PW.wavenum) @ x)
    assert rel(op.dense_rows(rows, x), ref) <= 1e-10
    op.close()


def test_dense_rows_equal_an_all_near_product(cuda_device):
    # one leaf holds every source: the MLFMA product is the dense product
    d = inputs.make_dipoles(300, seed=8, side=1.0)
    op = MLFMA.dipoles(d, PW, max_node_srcs=300, ref_compat=0, self_terms=1).setup()
    x = cvec(op.n, 9)
    rows = np.arange(op.n)
    assert rel(op.dense_rows(rows, x), op.matvec(x)) <= 1e-13
    op.close()


def test_mlfma_error_against_dense_rows(cuda_device):
    # a sphere with a far field: the 3-digit expansion is accurate to about 1e-3
    m = inputs.make_icosphere(4, radius=1.5)
    op = MLFMA.rwg(m, PW, max_node_srcs=24).setup()
    x = cvec(op.n, 10)
    rows = np.random.default_rng(11).choice(op.n, 64, replace=False)
    err = rel(op.matvec(x)[rows], op.dense_rows(rows, x))
    assert 1e-8 < err < 1e-2, err
    op.close()


def test_dense_rows_rejects_bad_rows(cuda_device):
    op = MLFMA.dipoles(inputs.make_dipoles(200, seed=1), PW, max_node_srcs=16).setup()
    with pytest.raises(MlfmaError) as e:
        op.dense_rows([0, op.n], cvec(op.n, 1))
    assert e.value.code == _lib.MLFMA_ERR_ARG
    assert op.dense_rows([], cvec(op.n, 1)).shape == (0,)
    op.close()
