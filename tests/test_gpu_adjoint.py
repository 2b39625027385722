"""Adjoint product, adjoint solve and the far-field power gradient (no
counterpart in the reference; see the header of include/mlfma_b200.h).

Checks: the transposed MLFMA pipeline is the exact adjoint of the forward one
(<A^H y, x> = <y, A x> to rounding), the far-field adjoint likewise, the
gradient against a dense FP64 computation where MLFMA is exact (every
interaction in the near field), and against central finite differences on a
problem with a far field."""
import numpy as np
import pytest

from mlfma_b200 import MLFMA, inputs
from oracle import mlfma_oracle as O

PW = inputs.PlaneWave()


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def cvec(n, seed):
    r = np.random.default_rng(seed)
    return r.standard_normal(n) + 1j * r.standard_normal(n)


def loads(n, seed):
    r = np.random.default_rng(seed)
    return r.uniform(0, 50, n) + 1j * r.uniform(-20, 20, n)


def dense_objective(A, M, B, w):
    """J, dJ/dz (packed), dJ/dw (packed) for the dense system (A) I = B^T w."""
    b = B.T @ w
    I = np.linalg.solve(A, b)
    F = M @ I
    lam = np.linalg.solve(A.conj().T, M.conj().T @ F)
    # dJ = 2 Re(lam^H (db - dZ I)); packed gradients dJ/dRe + i dJ/dIm
    return float(np.vdot(F, F).real), -2 * lam * np.conj(I), 2 * (B.conj() @ lam), I


def test_dense_gradient_formula_matches_finite_differences():
    # The formulas the library uses, on a random dense system (CPU only).
    rng = np.random.default_rng(0)
    n, nd, ne = 12, 5, 2
    A0 = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)) + 6 * np.eye(n)
    M = rng.standard_normal((nd, n)) + 1j * rng.standard_normal((nd, n))
    B = rng.standard_normal((ne, n)) + 1j * rng.standard_normal((ne, n))
    w = np.array([1.0 + 0.5j, -0.3 + 0.2j])
    z = loads(n, 1) * 0.01
    J, gz, gw, _ = dense_objective(A0 + np.diag(z), M, B, w)
    h = 1e-6
    for k in (0, 5):
        for step, part in ((h, "re"), (1j * h, "im")):
            zp, zm = z.copy(), z.copy()
            zp[k] += step
            zm[k] -= step
            fd = (dense_objective(A0 + np.diag(zp), M, B, w)[0] - dense_objective(A0 + np.diag(zm), M, B, w)[0]) / (2 * h)
            an = gz[k].real if part == "re" else gz[k].imag
            assert abs(fd - an) <= 1e-6 * max(1.0, abs(an))
    for j in range(ne):
        for step, part in ((h, "re"), (1j * h, "im")):
            wp, wm = w.copy(), w.copy()
            wp[j] += step
            wm[j] -= step
            fd = (dense_objective(A0 + np.diag(z), M, B, wp)[0] - dense_objective(A0 + np.diag(z), M, B, wm)[0]) / (2 * h)
            an = gw[j].real if part == "re" else gw[j].imag
            assert abs(fd - an) <= 1e-6 * max(1.0, abs(an))


def make(kind, **kw):
    if kind == "dipole":
        return MLFMA.dipoles(inputs.make_dipoles(3000, seed=31), PW, max_node_srcs=16, ref_compat=0, **kw).setup()
    return MLFMA.rwg(inputs.make_icosphere(4, radius=1.5), PW, max_node_srcs=24, ref_compat=0, **kw).setup()


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["dipole", "rwg"])
@pytest.mark.parametrize("precision,tol", [(0, 1e-12), (1, 1e-5)])
def test_adjoint_identity(cuda_device, kind, precision, tol):
    op = make(kind, self_terms=1, precision=precision)
    x, y = cvec(op.n, 1), cvec(op.n, 2)
    Ax = op.matvec(x)
    AHy = op.matvec_adjoint(y)
    lhs, rhs = np.vdot(y, Ax), np.vdot(AHy, x)
    assert abs(lhs - rhs) <= tol * np.linalg.norm(y) * np.linalg.norm(Ax)
    # with loads: (A + Z)^H = A^H + conj(Z)
    z = loads(op.n, 3)
    op.set_loads(z)
    assert rel(op.matvec(x), Ax + z * x) <= 1e-13
    assert rel(op.matvec_adjoint(y), AHy + np.conj(z) * y) <= 1e-13
    op.close()


@pytest.mark.gpu
def test_adjoint_needs_state_free_operator(cuda_device):
    from mlfma_b200 import MlfmaError
    op = MLFMA.dipoles(inputs.make_dipoles(500, seed=2), PW, max_node_srcs=16).setup()  # ref_compat = 1
    with pytest.raises(MlfmaError):
        op.matvec_adjoint(cvec(op.n, 1))
    op.close()


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["dipole", "rwg"])
def test_farfield_adjoint_identity(cuda_device, kind):
    op = make(kind)
    kh = op.phi_cut(37, theta=1.1)
    I = cvec(op.n, 4)
    G = cvec(3 * kh.shape[0], 5).reshape(-1, 3)
    F = op.farfield(I, kh)
    g = op.farfield_adjoint(G, kh)
    assert abs(np.vdot(G.ravel(), F.ravel()) - np.vdot(g, I)) <= 1e-12 * np.linalg.norm(G) * np.linalg.norm(F)
    op.close()


@pytest.mark.gpu
def test_gmres_adjoint_residual(cuda_device):
    op = MLFMA.rwg(inputs.make_icosphere(3, radius=1.0), PW, max_node_srcs=16, ref_compat=0, self_terms=1).setup()
    op.set_loads(loads(op.n, 6))
    b = cvec(op.n, 7)
    x, info = op.solve_adjoint(b, max_iter=2000, tol=1e-8, restart=100)
    assert info.converged
    assert rel(op.matvec_adjoint(x), b) <= 1.0001e-8
    op.close()


def _dense_problem(kind, n_or_level):
    if kind == "dipole":
        d = inputs.make_dipoles(n_or_level, seed=8, side=1.0)
        src = O.DipoleSources(d.pos, d.mom, PW)
        op = MLFMA.dipoles(d, PW, max_node_srcs=n_or_level, ref_compat=0, self_terms=1).setup()
    else:
        m = inputs.make_icosphere(n_or_level, radius=0.3)
        src = O.RWGSources(m.vertices, m.faces, m.rwgs, PW, quad_prec=2)
        op = MLFMA.rwg(m, PW, max_node_srcs=m.rwgs.shape[0], ref_compat=0, self_terms=1).setup()
    src.self_terms = True
    return op, src


@pytest.mark.gpu
@pytest.mark.parametrize("kind,size", [("dipole", 160), ("rwg", 1)])
def test_vjp_matches_dense(cuda_device, kind, size):
    # One leaf holds every source: the operator is the dense matrix exactly,
    # so the gradient must match the dense FP64 computation.
    op, src = _dense_problem(kind, size)
    n, k = op.n, PW.wavenum
    A = O.PHYS_C * k * src.block(np.arange(n), np.arange(n), k)
    z = loads(n, 9)
    op.set_loads(z)
    A = A + np.diag(z)
    assert rel(op.matvec(cvec(n, 1)), A @ cvec(n, 1)) <= 1e-12
    kh = op.phi_cut(16, theta=0.9)
    M = np.stack([O.farfield(src, np.eye(n)[:, i], kh, k).ravel() for i in range(n)], axis=1)
    pws = inputs.fibonacci_planewaves(2, wavenum=k)
    B = np.stack([op.rhs_planewave(p) for p in pws])
    w = np.array([1.0 + 0.0j, 0.4 - 0.3j])
    # unrestarted GMRES on n unknowns reaches the exact solution within n steps
    J, gz, gw, I, infos = op.vjp_farfield_power(pws, w, kh, max_iter=n, tol=1e-12, restart=0)
    Jd, gzd, gwd, Id = dense_objective(A, M, B, w)
    assert abs(J - Jd) <= 1e-9 * Jd
    assert rel(I, Id) <= 1e-9
    assert rel(gz, gzd) <= 1e-8
    assert rel(gw, gwd) <= 1e-8
    op.close()


@pytest.mark.gpu
def test_vjp_matches_finite_differences(cuda_device):
    # A sphere with a far field: the gradient of the MLFMA objective against
    # central differences (step 1e-4 relative) on random coordinates.
    m = inputs.make_icosphere(3, radius=1.0)
    op = MLFMA.rwg(m, PW, max_node_srcs=16, ref_compat=0, self_terms=1).setup()
    z = loads(op.n, 10)
    rng = np.random.default_rng(11)
    kh = rng.standard_normal((16, 3))
    kh /= np.linalg.norm(kh, axis=1)[:, None]
    pws = [PW]
    w = np.array([1.0 + 0.0j])
    opts = dict(max_iter=3000, tol=1e-12, restart=100)
    op.set_loads(z)
    J, gz, gw, _, _ = op.vjp_farfield_power(pws, w, kh, **opts)

    def objective(zz, ww=w):
        op.set_loads(zz)
        return op.vjp_farfield_power(pws, ww, kh, **opts)[0]

    worst = 0.0
    for kidx in rng.choice(op.n, 6, replace=False):
        h = 1e-4 * abs(z[kidx])
        for step, part in ((h, 0), (1j * h, 1)):
            zp, zm = z.copy(), z.copy()
            zp[kidx] += step
            zm[kidx] -= step
            fd = (objective(zp) - objective(zm)) / (2 * h)
            an = gz[kidx].real if part == 0 else gz[kidx].imag
            worst = max(worst, abs(fd - an) / max(abs(an), 1e-3 * np.abs(gz).max()))
    # J = |w|^2 J(1) for one excitation: dJ/dRe w = 2 J, dJ/dIm w = 0 (scale by |gw|)
    for part, step in ((0, 1e-4), (1, 1e-4j)):
        fd = (objective(z, w + step) - objective(z, w - step)) / (2e-4)
        an = gw[0].real if part == 0 else gw[0].imag
        worst = max(worst, abs(fd - an) / abs(gw[0]))
    assert abs(gw[0] - 2 * J) <= 1e-10 * J
    assert worst <= 1e-5, worst
    op.close()
