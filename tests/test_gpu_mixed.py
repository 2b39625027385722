"""Mixed precision (complex float far field, float accumulation; complex double
near field): its product must stay within float rounding of the FP64 product,
far below the MLFMA approximation error (3 digits here), and the solver must
still converge on it."""
import numpy as np
import pytest

from mlfma_b200 import MLFMA, inputs
from oracle import mlfma_oracle as O

pytestmark = pytest.mark.gpu
PW = inputs.PlaneWave()


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def cvec(n, seed):
    r = np.random.default_rng(seed)
    return r.standard_normal(n) + 1j * r.standard_normal(n)


@pytest.mark.parametrize("kind", ["dipole", "rwg"])
def test_mixed_close_to_fp64(cuda_device, kind):
    if kind == "dipole":
        g = inputs.make_dipoles(6000, seed=4)
        mk = lambda p: MLFMA.dipoles(g, PW, max_node_srcs=24, precision=p).setup()
    else:
        g = inputs.make_icosphere(5, radius=2.0)
        mk = lambda p: MLFMA.rwg(g, PW, max_node_srcs=54, precision=p).setup()
    a, b = mk(0), mk(1)
    x = cvec(a.n, 1)
    e = rel(b.matvec(x), a.matvec(x))
    assert e < 1e-5, e  # float rounding through five stages
    a.close()
    b.close()


def test_mixed_error_vs_dense_matches_fp64(cuda_device):
    d = inputs.make_dipoles(1500, seed=9)
    orc = O.Oracle(O.DipoleSources(d.pos, d.mom, PW), max_node_srcs=24)
    A = orc.dense()
    x = cvec(d.n, 2)
    yd = A @ x
    e64 = rel(MLFMA.dipoles(d, PW, max_node_srcs=24, precision=0).setup().matvec(x), yd)
    e32 = rel(MLFMA.dipoles(d, PW, max_node_srcs=24, precision=1).setup().matvec(x), yd)
    assert e64 < 1e-2 and abs(e32 - e64) < 1e-4 * max(1.0, e64 / 1e-3)


def test_mixed_gmres_tracks_fp64(cuda_device):
    # The reference's RWG operator has no self terms and converges slowly; the
    # check is that the mixed solve follows the FP64 solve iteration for
    # iteration (same residual, same iterate) rather than a target residual.
    m = inputs.make_icosphere(3, radius=1.0)
    ops = [MLFMA.rwg(m, PW, max_node_srcs=16, ref_compat=0, precision=p).setup() for p in (0, 1)]
    b = ops[0].rhs()
    (x64, i64), (x32, i32) = [op.solve(b, max_iter=60, tol=1e-3, restart=30, ref_givens=False) for op in ops]
    assert i32.iterations == i64.iterations
    assert abs(i32.true_residual - i64.true_residual) <= 1e-3 * i64.true_residual + 1e-6
    assert rel(x32, x64) < 1e-4


def test_refined_mixed_solve_meets_fp64_residual(cuda_device):
    # Iterative refinement: inner GMRES on the mixed operator, outer residual in
    # FP64.  The returned solution must meet the tolerance on the FP64 operator
    # (checked here with a separate FP64 operator) and agree with the FP64 solve.
    m = inputs.make_icosphere(3, radius=1.0)
    op64 = MLFMA.rwg(m, PW, max_node_srcs=16, ref_compat=0, precision=0, self_terms=1).setup()
    opmx = MLFMA.rwg(m, PW, max_node_srcs=16, ref_compat=0, precision=1, self_terms=1).setup()
    b = op64.rhs()
    tol = 1e-4
    x64, i64 = op64.solve(b, max_iter=400, tol=tol, restart=50, ref_givens=False)
    xmx, imx = opmx.solve(b, max_iter=400, tol=tol, restart=50, ref_givens=False, refine=True)
    assert i64.converged and imx.converged
    assert imx.refinements >= 1
    r = rel(op64.matvec(xmx), b)
    assert r <= tol * 1.0001, r
    assert abs(r - imx.true_residual) <= 1e-3 * r
    assert rel(xmx, x64) < 10 * tol
    op64.close()
    opmx.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_flexible_gmres_meets_fp64_residual(cuda_device, precision):
    # FGMRES: FP64 outer Krylov space over inner GMRES solves on the operator's
    # own far field (complex float on the mixed operator).  The answer must meet
    # the tolerance on the FP64 operator and agree with the FP64 GMRES solution.
    m = inputs.make_icosphere(3, radius=1.0)
    op64 = MLFMA.rwg(m, PW, max_node_srcs=16, ref_compat=0, precision=0, self_terms=1).setup()
    op = op64 if precision == 0 else MLFMA.rwg(m, PW, max_node_srcs=16, ref_compat=0, precision=1,
                                               self_terms=1).setup()
    b = op64.rhs()
    tol = 1e-6
    x64, i64 = op64.solve(b, max_iter=600, tol=tol, restart=50, ref_givens=False)
    xf, inf = op.solve(b, max_iter=600, tol=tol, restart=30, flexible=True, inner_iters=10)
    assert i64.converged and inf.converged
    assert inf.refinements >= 1 and inf.iterations >= inf.refinements
    r = rel(op64.matvec(xf), b)
    assert r <= tol * 1.0001, r
    assert abs(r - inf.true_residual) <= 1e-3 * r + 1e-12
    assert rel(xf, x64) < 100 * tol
    if op is not op64:
        op.close()
    op64.close()


def test_flexible_gmres_with_cheaper_inner_operator(cuda_device):
    # FGMRES whose inner iterations run on another operator of the same
    # sources and tree (here 1-digit angular sampling, 4-point interpolation,
    # complex-float far field): the outer FP64 residual still meets tol, and the
    # answer matches the FP64 GMRES solution.
    m = inputs.make_icosphere(3, radius=1.0)
    op64 = MLFMA.rwg(m, PW, max_node_srcs=16, ref_compat=0, precision=0, self_terms=1).setup()
    cheap = MLFMA.rwg(m, PW, max_node_srcs=16, ref_compat=0, precision=1, self_terms=1, digits=1,
                      interp_order=2).setup()
    b = op64.rhs()
    tol = 1e-6
    x64, _ = op64.solve(b, max_iter=600, tol=tol, restart=50, ref_givens=False)
    op64.set_inner_operator(cheap)
    xf, inf = op64.solve(b, max_iter=600, tol=tol, restart=30, flexible=True, inner_iters=10)
    assert inf.converged
    assert rel(op64.matvec(xf), b) <= tol * 1.0001
    assert rel(xf, x64) < 100 * tol
    # the inner operator serves flexible solves only; a plain solve ignores it
    x2, i2 = op64.solve(b, max_iter=600, tol=tol, restart=50, ref_givens=False)
    assert i2.converged and rel(x2, x64) < 1e-12
    # a different tree is refused; destroying the inner operator detaches it
    other = MLFMA.rwg(m, PW, max_node_srcs=8, ref_compat=0, precision=1, self_terms=1).setup()
    with pytest.raises(Exception):
        op64.set_inner_operator(other)
    other.close()
    cheap.close()
    xf2, inf2 = op64.solve(b, max_iter=600, tol=tol, restart=30, flexible=True, inner_iters=10)
    assert inf2.converged and rel(op64.matvec(xf2), b) <= tol * 1.0001
    op64.close()
