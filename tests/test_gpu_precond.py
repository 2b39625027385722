"""Leaf block-Jacobi right preconditioning of GMRES (opts.precond): every
leaf's diagonal block of A = C k Z + diag(loads) inverted on the GPU.

* One leaf holding every source: M = A, so preconditioned GMRES converges in
  one step (checks the inversion, loads included).
* The r = 1 wavelength RWG sphere with self terms: the same FP64 residual and
  solution, as GMRES and as the inner solves of mixed FGMRES.  On this EFIE
  the leaf blocks make a poor approximate inverse: GMRES(50) to 1e-6 takes
  about 4.6x more iterations with it than without (188 -> 871 here; a dense
  numpy restatement of the same operator, 137 -> 829), so the test asserts
  correctness, not a speed-up."""
import numpy as np
import pytest

from mlfma_b200 import MLFMA, inputs

pytestmark = pytest.mark.gpu
PW = inputs.PlaneWave()


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_one_leaf_preconditioner_is_the_inverse(cuda_device):
    d = inputs.make_dipoles(60, seed=5, side=0.5)
    op = MLFMA.dipoles(d, PW, max_node_srcs=64, self_terms=1, ref_compat=0).setup()
    z = np.random.default_rng(1).uniform(1, 5, op.n) + 1j * np.random.default_rng(2).uniform(-2, 2, op.n)
    op.set_loads(z)
    b = op.rhs()
    x, info = op.solve(b, max_iter=20, tol=1e-10, restart=20, ref_givens=False, precond=True)
    assert info.converged and info.iterations <= 2
    assert rel(op.matvec(x), b) <= 1e-10
    op.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_preconditioned_solves_meet_fp64_residual(cuda_device, precision):
    m = inputs.make_icosphere(3, radius=1.0)
    op64 = MLFMA.rwg(m, PW, max_node_srcs=16, ref_compat=0, precision=0, self_terms=1).setup()
    op = op64 if precision == 0 else MLFMA.rwg(m, PW, max_node_srcs=16, ref_compat=0, precision=1,
                                               self_terms=1).setup()
    b = op64.rhs()
    tol = 1e-6
    x0, i0 = op64.solve(b, max_iter=1000, tol=tol, restart=50, ref_givens=False)
    if precision == 0:
        xp, ip = op.solve(b, max_iter=1000, tol=tol, restart=50, ref_givens=False, precond=True)
    else:
        xp, ip = op.solve(b, max_iter=1000, tol=tol, restart=30, flexible=True, inner_iters=20, precond=True)
    assert i0.converged and ip.converged
    r = rel(op64.matvec(xp), b)
    assert r <= tol * 1.0001, r
    assert rel(xp, x0) < 100 * tol
    if op is not op64:
        op.close()
    op64.close()
