"""Staged interpolation kernels of the one-vector product (mlfma_set_staged_interp):
M2M with the children shifted and summed first (k_m2m_sum) and L2L with the
parent staged in shared memory (k_l2l_st) against the per-child kernels, in
FP64 (rounding level), in complex float (1e-5) and through the transposed
product, on the benchmark sphere and on a 6-level sphere with the grids of the
largest benchmark (up to 58 x 116)."""
import numpy as np
import pytest

from mlfma_b200 import MLFMA, inputs

pytestmark = pytest.mark.gpu
PW = inputs.PlaneWave()


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def cvec(n, seed):
    r = np.random.default_rng(seed)
    return r.standard_normal(n) + 1j * r.standard_normal(n)


def sphere_dipoles(n, radius, seed):
    r = np.random.default_rng(seed)
    v = r.standard_normal((n, 3))
    pos = radius * v / np.linalg.norm(v, axis=1)[:, None]
    return inputs.Dipoles(pos=pos, mom=np.tile([1.0, 0.0, 0.0], (n, 1)))


CASES = {
    "rwg": lambda p: MLFMA.rwg(inputs.make_icosphere(5, radius=2.0), PW, max_node_srcs=54, ref_compat=0,
                               self_terms=1, precision=p),
    "sphere16": lambda p: MLFMA.dipoles(sphere_dipoles(40000, 7.99, 5), PW, max_node_srcs=2, max_level=6,
                                        root_leng=16.0, ref_compat=0, precision=p),
}


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("precision", [0, 1])
def test_staged_interp_matches_per_child_kernels(cuda_device, case, precision):
    op = CASES[case](precision).setup()
    tol = 1e-13 if precision == 0 else 1e-5
    x = cvec(op.n, 3)
    op.set_staged_interp(0)
    y0 = op.matvec(x)
    a0 = op.matvec_adjoint(x)
    for mode in (1, 2, 3, 5, 6, 7, 8, 9):
        op.set_staged_interp(mode)
        y = op.matvec(x)
        assert rel(y, y0) <= tol, (mode, rel(y, y0))
        assert rel(op.matvec(x), y) <= 1e-15  # graph replay
        assert rel(op.matvec_adjoint(x), a0) <= tol
    op.close()


def test_autotune_reports_staged_choice(cuda_device):
    op = CASES["rwg"](1).setup()
    x = cvec(op.n, 4)
    y0 = op.matvec(x)
    t = op.autotune(1, reps=2)
    assert "m2m_staged" in t and "l2l_staged" in t
    assert rel(op.matvec(x), y0) <= 1e-5
    op.close()
