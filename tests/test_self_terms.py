"""Self terms (no reference counterpart): closed-form triangle potentials and
the mixed-potential RWG entries that replace the reference's skipped
coincident-triangle terms when self_terms = 1.

CPU checks of the oracle's restatement: the closed forms against an
independent polar-coordinate quadrature, and the mixed-potential entries
against the reference's dyadic-Green quadrature on well-separated pairs, where
both forms are accurate and must agree."""
import numpy as np
import pytest

from mlfma_b200 import inputs
from oracle import mlfma_oracle as O


def polar_potentials(P, r, npts=400):
    """int_T 1/R and int_T (rho' - rho)/R by splitting T into the three signed
    triangles (rho, p, q) and integrating radially in closed form and along each
    edge by Gauss-Legendre."""
    n = np.cross(P[1] - P[0], P[2] - P[0])
    n /= np.linalg.norm(n)
    h = float(n @ (r - P[0]))
    rho = r - h * n
    ah = abs(h)
    s, w = np.polynomial.legendre.leggauss(npts)
    s, w = 0.5 * (s + 1.0), 0.5 * w
    I0, I1 = 0.0, np.zeros(3)
    for i in range(3):
        p, q = P[i], P[(i + 1) % 3]
        L = q - p
        pts = p[None, :] + s[:, None] * L[None, :] - rho[None, :]   # r'(s) - rho
        rm = np.linalg.norm(pts, axis=1)
        # signed dtheta = ((r' - rho) x L) . n / |r' - rho|^2 ds
        jac = np.cross(pts, L) @ n / rm ** 2
        Rm = np.sqrt(rm ** 2 + h * h)
        f0 = Rm - ah                                          # int_0^rm rho/R drho
        f1 = 0.5 * (rm * Rm - (h * h * np.log((rm + Rm) / ah) if ah > 0 else 0.0))  # int_0^rm rho^2/R
        I0 += np.sum(w * jac * f0)
        I1 += np.sum((w * jac * f1 / rm)[:, None] * pts, axis=0)
    return I0, I1


TRI = np.array([[0.0, 0.0, 0.0], [1.0, 0.1, 0.0], [0.3, 0.9, 0.2]])


@pytest.mark.parametrize("bary,h", [((0.3, 0.3, 0.4), 0.0), ((0.2, 0.5, 0.3), 0.05), ((0.6, 0.2, 0.2), -0.4),
                                    ((1.4, -0.2, -0.2), 0.0), ((-0.3, 0.6, 0.7), 0.2), ((0.1, 0.1, 0.8), 1e-3)])
def test_tri_potentials_match_polar_quadrature(bary, h):
    n = np.cross(TRI[1] - TRI[0], TRI[2] - TRI[0])
    n /= np.linalg.norm(n)
    r = np.asarray(bary) @ TRI + h * n
    I0, I1, rho = O.tri_potentials(TRI, r)
    J0, J1 = polar_potentials(TRI, r)
    assert abs(I0 - J0) <= 1e-10 * abs(J0)
    assert np.linalg.norm(I1 - J1) <= 1e-9 * max(np.linalg.norm(J1), 1e-3)
    assert np.allclose(rho + h * n, r)


def test_mpie_matches_dyadic_on_separated_pairs():
    m = inputs.make_icosphere(3, radius=1.0)
    S = O.RWGSources(m.vertices, m.faces, m.rwgs, inputs.PlaneWave(), quad_prec=2)
    k = 2 * np.pi
    rng = np.random.default_rng(0)
    rows = rng.choice(S.n, 40, replace=False)
    cols = rng.choice(S.n, 40, replace=False)
    Zd = S.block(rows, cols, k)
    d = np.linalg.norm(S.centers[rows][:, None] - S.centers[cols][None], axis=-1)
    ri, ci = np.nonzero(d > 0.5)            # > 5 edge lengths apart
    Zm = S.mpie(rows[ri], cols[ci], k)
    # entries between nearly orthogonal RWGs cancel to ~1e-17: scale by the
    # largest entry of the sample
    err = np.abs(Zm - Zd[ri, ci]) / np.abs(Zd[ri, ci]).max()
    assert err.max() < 1e-5, err.max()


def test_self_terms_symmetric_and_nonzero_diagonal():
    m = inputs.make_icosphere(2, radius=1.0)
    S = O.RWGSources(m.vertices, m.faces, m.rwgs, inputs.PlaneWave(), quad_prec=2)
    S.self_terms = True
    idx = np.arange(60)
    Z = S.block(idx, idx, 2 * np.pi)
    assert np.allclose(Z, Z.T, rtol=0, atol=1e-12 * np.abs(Z).max())
    assert np.all(np.abs(np.diag(Z)) > 0)
    # the diagonal dominates its row on a fine mesh (scalar-potential self term)
    assert np.all(np.abs(np.diag(Z)) >= np.abs(Z - np.diag(np.diag(Z))).max(axis=1))


# ---------------------------------------------------------------- GPU parity
def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def cvec(n, seed):
    r = np.random.default_rng(seed)
    return r.standard_normal(n) + 1j * r.standard_normal(n)


@pytest.mark.gpu
def test_self_terms_dipole_matvec_matches_oracle(cuda_device):
    from mlfma_b200 import MLFMA
    pw = inputs.PlaneWave()
    g = inputs.make_dipoles(1500, seed=21)
    src = O.DipoleSources(g.pos, g.mom, pw)
    src.self_terms = True
    op = MLFMA.dipoles(g, pw, max_node_srcs=24, self_terms=1).setup()
    x = cvec(op.n, 3)
    assert rel(op.matvec(x), O.Oracle(src, max_node_srcs=24).matvec(x)) <= 1e-10
    op.close()


@pytest.mark.gpu
def test_self_terms_rwg_near_field_matches_oracle(cuda_device):
    # The oracle's numpy RWG patterns round the closed-form plane-wave integral
    # differently (about 1e-9 relative on the product), so the check isolates
    # what the self terms change: (A_self - A_ref) x, in which the far field
    # cancels exactly on both sides.
    from mlfma_b200 import MLFMA
    pw = inputs.PlaneWave()
    g = inputs.make_icosphere(2, radius=0.8)
    x = cvec(g.rwgs.shape[0], 3)
    ys = []
    for st in (0, 1):
        op = MLFMA.rwg(g, pw, max_node_srcs=12, self_terms=st).setup()
        ys.append(op.matvec(x))
        op.close()
    yo = []
    for st in (False, True):
        src = O.RWGSources(g.vertices, g.faces, g.rwgs, pw, quad_prec=2)
        src.self_terms = st
        yo.append(O.Oracle(src, max_node_srcs=12).matvec(x))
    assert rel(ys[1] - ys[0], yo[1] - yo[0]) <= 1e-10


@pytest.mark.gpu
def test_self_terms_gmres_converges(cuda_device):
    # With the self terms the EFIE is well conditioned enough for GMRES(50) to
    # reach 1e-4 in tens of iterations (the reference's operator, without them,
    # needs thousands).
    from mlfma_b200 import MLFMA
    m = inputs.make_icosphere(3, radius=1.0)
    op = MLFMA.rwg(m, inputs.PlaneWave(), max_node_srcs=16, ref_compat=0, self_terms=1).setup()
    b = op.rhs()
    x, info = op.solve(b, max_iter=400, tol=1e-4, restart=50, ref_givens=False)
    assert info.converged and info.iterations < 200
    assert rel(op.matvec(x), b) <= 1.0001e-4
    op.close()
