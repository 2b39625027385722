"""Tensor-core interpolation and anterpolation (tcgen05, 3xTF32) of the
complex-float far field: its products must agree with the CUDA-core kernels'
to float rounding (1e-5 relative, the tolerance of the mixed-precision tests),
for one vector and for many right-hand sides, on small and on the largest
benchmark grids (58 x 116 directions), and a refined solve on it must meet the
FP64 residual."""
import numpy as np
import pytest

from mlfma_b200 import MLFMA, inputs

pytestmark = pytest.mark.gpu
PW = inputs.PlaneWave()
TOL = 1e-5


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def cvec(shape, seed):
    r = np.random.default_rng(seed)
    return r.standard_normal(shape) + 1j * r.standard_normal(shape)


def sphere_dipoles(n, radius, seed):
    r = np.random.default_rng(seed)
    v = r.standard_normal((n, 3))
    pos = radius * v / np.linalg.norm(v, axis=1)[:, None]
    mom = r.standard_normal((n, 3))
    mom /= np.linalg.norm(mom, axis=1)[:, None]
    return inputs.Dipoles(pos=pos, mom=mom)


CASES = {
    # 4-wavelength cube, 0.25-wavelength leaves (grids up to 21 x 42)
    "cube": lambda: (inputs.make_dipoles(6000, seed=3), dict(max_node_srcs=4, max_level=4, root_leng=4.0)),
    # the 2-wavelength RWG sphere of the benchmark (5 levels)
    "rwg": lambda: (inputs.make_icosphere(5, radius=2.0), dict(max_node_srcs=54)),
    # an 8-wavelength sphere in a 16-wavelength root box, 0.25-wavelength
    # leaves: the grids of the largest benchmark (up to 58 x 116)
    "sphere16": lambda: (sphere_dipoles(40000, 7.99, 5), dict(max_node_srcs=2, max_level=6, root_leng=16.0)),
}


def make(case, **kw):
    g, cfg = CASES[case]()
    mk = MLFMA.rwg if case == "rwg" else MLFMA.dipoles
    return mk(g, PW, ref_compat=0, **cfg, **kw).setup()


@pytest.mark.parametrize("case", ["cube", "rwg", "sphere16"])
def test_tc_one_vector_matches_cuda_cores(cuda_device, case):
    op = make(case, precision=1)
    x = cvec(op.n, 1)
    op.interp_path = 0
    y_cc = op.matvec(x)
    op.interp_path = 5  # M2M and L2L of the one-vector product
    assert op.interp_path == 5
    y_tc = op.matvec(x)
    y_tc2 = op.matvec(x)  # graph replay, same result
    assert rel(y_tc, y_cc) <= TOL
    assert rel(y_tc2, y_tc) <= 1e-12
    op.close()
    op64 = make(case, precision=0)
    assert rel(y_tc, op64.matvec(x)) <= TOL  # float rounding through the far field
    op64.close()


@pytest.mark.parametrize("case", ["cube", "sphere16"])
def test_tc_many_rhs_matches_cuda_cores(cuda_device, case):
    op = make(case, precision=1, max_rhs=8)
    X = cvec((5, op.n), 2)
    op.interp_path = 10  # M2M and L2L of the many-rhs product
    Y_tc = op.matvec_multi(X)
    op.interp_path = 0
    Y_cc = op.matvec_multi(X)
    for r in range(5):
        assert rel(Y_tc[r], Y_cc[r]) <= TOL
    # each column equals the one-vector product on the tensor cores too
    op.interp_path = 5
    assert rel(Y_tc[3], op.matvec(X[3])) <= TOL
    op.close()


def test_tc_refined_solve_meets_fp64_residual(cuda_device):
    m = inputs.make_icosphere(3, radius=1.0)
    op64 = MLFMA.rwg(m, PW, max_node_srcs=16, ref_compat=0, precision=0, self_terms=1).setup()
    opmx = MLFMA.rwg(m, PW, max_node_srcs=16, ref_compat=0, precision=1, self_terms=1).setup()
    opmx.interp_path = 5
    b = op64.rhs()
    tol = 1e-4
    x64, i64 = op64.solve(b, max_iter=400, tol=tol, restart=50, ref_givens=False)
    xmx, imx = opmx.solve(b, max_iter=400, tol=tol, restart=50, ref_givens=False, refine=True)
    assert i64.converged and imx.converged
    assert rel(op64.matvec(xmx), b) <= tol * 1.0001
    assert rel(xmx, x64) < 10 * tol
    op64.close()
    opmx.close()


def test_tc_state_rule_and_fp64_operator(cuda_device):
    # The reference's stale-local rule (ref_compat = 1): over a sequence of
    # products both kernel families keep the same state.
    d = inputs.make_dipoles(4000, seed=8)
    a = MLFMA.dipoles(d, PW, max_node_srcs=8, precision=1).setup()
    b = MLFMA.dipoles(d, PW, max_node_srcs=8, precision=1).setup()
    a.interp_path, b.interp_path = 0, 5
    for s in (3, 4, 5):
        x = cvec(a.n, s)
        assert rel(b.matvec(x), a.matvec(x)) <= TOL
    a.close()
    b.close()
    # an FP64 operator has no complex-float far field
    op = MLFMA.dipoles(d, PW, max_node_srcs=8, precision=0).setup()
    assert op.interp_path == 0
    with pytest.raises(Exception):
        op.interp_path = 5
    op.close()
