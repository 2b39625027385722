"""Products and solves on many right-hand sides at once (mlfma_matvec_multi,
mlfma_gmres_multi) against the one-vector path, column by column.

The batched kernels sum in a different order (GEMM tiles, sibling-group M2L),
so FP64 columns agree to rounding (1e-12 relative); mixed columns to float
rounding (1e-5)."""
import numpy as np
import pytest

from mlfma_b200 import MLFMA, MlfmaError, inputs
from mlfma_b200 import _lib

pytestmark = pytest.mark.gpu
PW = inputs.PlaneWave()


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def cmat(nr, n, seed):
    r = np.random.default_rng(seed)
    return r.standard_normal((nr, n)) + 1j * r.standard_normal((nr, n))


def make(kind, **kw):
    if kind == "dipole":
        return MLFMA.dipoles(inputs.make_dipoles(3000, seed=31), PW, max_node_srcs=16, **kw).setup()
    return MLFMA.rwg(inputs.make_icosphere(4, radius=1.5), PW, max_node_srcs=24, **kw).setup()


@pytest.mark.parametrize("kind", ["dipole", "rwg"])
@pytest.mark.parametrize("nr", [1, 5, 33, 64])
def test_matvec_multi_matches_single(cuda_device, kind, nr):
    op = make(kind, ref_compat=0, max_rhs=64)
    X = cmat(nr, op.n, 7)
    Y = op.matvec_multi(X)
    for r in range(nr):
        assert rel(Y[r], op.matvec(X[r])) <= 1e-12
    # accumulate: Y += A X
    Y2 = op.matvec_multi(X, accumulate=True, out=Y.copy())
    assert rel(Y2, 2 * Y) <= 1e-14
    op.close()


def test_matvec_multi_reference_state_matches_single(cuda_device):
    # ref_compat = 1: boxes with an empty list 2 keep their local patterns from
    # the previous product; the batched path keeps its own copy of that state
    # and must follow the same sequence.
    single = make("rwg", max_rhs=1)
    multi = make("rwg", max_rhs=8)
    X = cmat(2, single.n, 9)
    for r in range(2):
        assert rel(multi.matvec_multi(X[r:r + 1])[0], single.matvec(X[r])) <= 1e-12
    single.close()
    multi.close()


@pytest.mark.parametrize("kind", ["dipole", "rwg"])
def test_matvec_multi_mixed(cuda_device, kind):
    op = make(kind, ref_compat=0, max_rhs=16, precision=1)
    X = cmat(16, op.n, 3)
    Y = op.matvec_multi(X)
    for r in (0, 7, 15):
        assert rel(Y[r], op.matvec(X[r])) <= 1e-5
    op.close()


def test_matvec_multi_rejects_too_many(cuda_device):
    op = make("dipole", max_rhs=4)
    with pytest.raises(MlfmaError) as e:
        op.matvec_multi(cmat(5, op.n, 1))
    assert e.value.code == _lib.MLFMA_ERR_ARG
    op.close()


def test_gmres_multi_matches_single(cuda_device):
    m = inputs.make_icosphere(3, radius=1.0)
    op = MLFMA.rwg(m, PW, max_node_srcs=16, ref_compat=0, self_terms=1, max_rhs=8).setup()
    B = np.stack([op.rhs_planewave(p) for p in inputs.fibonacci_planewaves(8)])
    tol = 1e-6
    X, infos = op.solve_multi(B, max_iter=400, tol=tol, restart=40)
    for r in range(8):
        assert infos[r].converged
        assert rel(op.matvec(X[r]), B[r]) <= tol * 1.0001
        x1, i1 = op.solve(B[r], max_iter=400, tol=tol, restart=40, ref_givens=False)
        assert i1.converged
        assert abs(infos[r].iterations - i1.iterations) <= 2
        assert rel(X[r], x1) <= 1e-4
    op.close()


def test_gmres_multi_refined_mixed(cuda_device):
    m = inputs.make_icosphere(3, radius=1.0)
    op64 = MLFMA.rwg(m, PW, max_node_srcs=16, ref_compat=0, self_terms=1).setup()
    opmx = MLFMA.rwg(m, PW, max_node_srcs=16, ref_compat=0, self_terms=1, max_rhs=6, precision=1).setup()
    B = np.stack([opmx.rhs_planewave(p) for p in inputs.fibonacci_planewaves(6)])
    tol = 1e-4
    X, infos = opmx.solve_multi(B, max_iter=400, tol=tol, restart=50, refine=True)
    for r in range(6):
        assert infos[r].converged and infos[r].refinements >= 1
        assert rel(op64.matvec(X[r]), B[r]) <= tol * 1.0001
    op64.close()
    opmx.close()


def test_rhs_planewave_matches_handle_rhs(cuda_device):
    op = make("rwg", max_rhs=1)
    assert np.array_equal(op.rhs_planewave(PW), op.rhs())
    op.close()


def test_autotune_keeps_results(cuda_device):
    # The tuner changes launch shapes only: the same call sequence on a tuned
    # and an untuned operator gives the same products to rounding, including
    # the reference's stale-local state (ref_compat = 1), which the tuner saves
    # and restores around its trial launches.
    tuned, plain = make("rwg", max_rhs=8), make("rwg", max_rhs=8)
    x = cmat(1, tuned.n, 21)[0]
    X = cmat(8, tuned.n, 22)
    seq = []
    for op, tune in ((tuned, True), (plain, False)):
        out = [op.matvec(x)]
        if tune:
            t1 = op.autotune(1, reps=3)
            assert t1["m2l_chunk"] in (32, 64, 96, 128) and t1["product_ms_after"] > 0
        out.append(op.matvec(x))
        out.append(op.matvec_multi(X))
        if tune:
            t8 = op.autotune(8, reps=3)
            assert t8["multi_l2l_pairs"] in (1, 2) and t8["multi_m2m_rows_fast"] in (0, 1)
        out.append(op.matvec_multi(X))
        out.append(op.matvec(x))
        seq.append(out)
    for a, b in zip(*seq):
        assert rel(a, b) <= 1e-12
    tuned.close()
    plain.close()


def test_multi_edge_cases(cuda_device):
    # every source in one leaf (no far field), and a zero right-hand side
    d = inputs.make_dipoles(40, seed=5, side=0.5)
    op = MLFMA.dipoles(d, PW, max_node_srcs=64, ref_compat=0, self_terms=1, max_rhs=4).setup()
    X = cmat(3, op.n, 8)
    Y = op.matvec_multi(X)
    for r in range(3):
        assert rel(Y[r], op.matvec(X[r])) <= 1e-13
    B = np.stack([op.rhs(), np.zeros(op.n, dtype=complex)])
    Xs, infos = op.solve_multi(B, max_iter=200, tol=1e-10, restart=0)
    assert infos[0].converged and infos[1].converged
    assert np.all(Xs[1] == 0)
    assert rel(op.matvec(Xs[0]), B[0]) <= 1.0001e-10
    op.close()


def test_operators_of_different_sizes_coexist(cuda_device):
    # Kernel launch limits are shared by every operator in the process: an
    # operator set up after one with larger leaves must not break the first
    # one's products (first launched here after the second set-up).
    from oracle import mlfma_oracle as O
    d = inputs.make_dipoles(3000, seed=51)
    big = MLFMA.dipoles(d, PW, max_node_srcs=64).setup()
    small = MLFMA.dipoles(inputs.make_dipoles(500, seed=52), PW, max_node_srcs=8).setup()
    x = cmat(1, big.n, 23)[0]
    y = big.matvec(x)
    ys = small.matvec(cmat(1, small.n, 24)[0])
    assert np.all(np.isfinite(ys))
    orc = O.Oracle(O.DipoleSources(d.pos, d.mom, PW), max_node_srcs=64)
    assert rel(y, orc.matvec(x)) <= 1e-10
    big.close()
    small.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_gmres_multi_flexible_matches_single(cuda_device, precision):
    """Batched FGMRES (mlfma_gmres_multi with flexible = 1): every column meets
    its tolerance on the FP64 residual and agrees with the one-vector FGMRES
    of the same right-hand side (same outer and inner steps up to rounding);
    columns stop on their own tolerance while the others go on."""
    m = inputs.make_icosphere(3, radius=1.0)
    op = MLFMA.rwg(m, PW, max_node_srcs=16, ref_compat=0, self_terms=1, max_rhs=8, precision=precision).setup()
    op64 = MLFMA.rwg(m, PW, max_node_srcs=16, ref_compat=0, self_terms=1).setup()
    B = np.stack([op.rhs_planewave(p) for p in inputs.fibonacci_planewaves(6)])
    B[3] *= 1e3  # a column of another scale: its own absolute target
    tol = 1e-7
    X, infos = op.solve_multi(B, max_iter=2000, tol=tol, restart=10, flexible=True, inner_iters=8)
    for r in range(6):
        assert infos[r].converged
        assert infos[r].refinements >= 1 and infos[r].iterations >= infos[r].refinements
        assert rel(op64.matvec(X[r]), B[r]) <= tol * 1.0001
        x1, i1 = op.solve(B[r], max_iter=2000, tol=tol, restart=10, flexible=True, inner_iters=8)
        assert i1.converged
        assert abs(infos[r].refinements - i1.refinements) <= 2
        assert rel(X[r], x1) <= 1e-5
    op.close()
    op64.close()


def test_gmres_multi_flexible_edge_cases(cuda_device):
    """A zero right-hand side gives x = 0 at once; one column; a budget that
    runs out reports the column as not converged with its true residual."""
    op = MLFMA.rwg(inputs.make_icosphere(3, radius=1.0), PW, max_node_srcs=16, ref_compat=0, self_terms=1,
                   max_rhs=4, precision=1).setup()
    B = cmat(3, op.n, 5)
    B[1] = 0.0
    X, infos = op.solve_multi(B, max_iter=600, tol=1e-8, restart=12, flexible=True, inner_iters=10)
    assert np.all(X[1] == 0) and infos[1].converged and infos[1].iterations == 0
    for r in (0, 2):
        assert infos[r].converged
        assert rel(op.matvec(X[r]), B[r]) <= 1e-4  # the mixed product; the FP64 residual met 1e-8
    X1, i1 = op.solve_multi(B[:1], max_iter=600, tol=1e-8, restart=12, flexible=True, inner_iters=10)
    assert i1[0].converged and rel(X1[0], X[0]) <= 1e-6
    Xs, ishort = op.solve_multi(B[:1], max_iter=5, tol=1e-12, restart=12, flexible=True, inner_iters=10)
    assert not ishort[0].converged and ishort[0].iterations <= 5 + 10
    assert ishort[0].true_residual < 1.0
    op.close()
