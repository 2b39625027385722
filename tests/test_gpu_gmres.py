"""GMRES on the device against the reference's Solver::solve."""
import os

import numpy as np
import pytest

from conftest import needs_ref
from mlfma_b200 import MLFMA, MlfmaError, inputs
from mlfma_b200 import _lib

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PW = inputs.PlaneWave()


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("name", ["dipole_n600", "rwg_ico2_r1"])
def test_reference_mode_matches_golden(cuda_device, name):
    import make_golden as mg
    case = mg.CASES[name]
    f = np.load(os.path.join(GOLD, name + ".npz"))
    g = mg.geometry(case)
    op = (MLFMA.dipoles if case["kind"] == "dipole" else MLFMA.rwg)(g, PW, max_node_srcs=case["max_node_srcs"])
    op.setup()
    # Same call sequence as the fixture: one matvec, then the solve.  Boxes whose
    # list 2 is empty keep their local patterns from call to call (the
    # reference's stale-local rule), so the solve depends on that history.
    op.matvec(f["x"])
    x, info = op.solve(max_iter=int(f["iters"]), tol=1e-12)
    assert info.iterations == int(f["iters"])
    assert rel(x, f["sol"]) <= 1e-8
    op.close()


@needs_ref
@pytest.mark.parametrize("kind", ["dipole", "rwg"])
def test_reference_mode_matches_reference(cuda_device, kind):
    from oracle import ref_lib
    g = inputs.make_dipoles(1200, seed=13) if kind == "dipole" else inputs.make_icosphere(3, radius=1.0)
    mns = 32 if kind == "dipole" else 16
    op = (MLFMA.dipoles if kind == "dipole" else MLFMA.rwg)(g, PW, max_node_srcs=mns).setup()
    P = ref_lib.RefProblem(kind, g, PW, max_node_srcs=mns)
    x, info = op.solve(max_iter=15, tol=1e-6)
    xr, itr = P.solve(max_iter=15, eps=1e-6)
    assert info.iterations == itr
    assert rel(x, xr) <= 1e-8
    op.close()


def test_restarted_gmres_true_residual(cuda_device):
    m = inputs.make_icosphere(3, radius=1.0)
    op = MLFMA.rwg(m, PW, max_node_srcs=16).setup()
    b = op.rhs()
    x, info = op.solve(b, max_iter=60, tol=1e-3, restart=20, ref_givens=False)
    r = rel(op.matvec(x), b)
    assert abs(r - info.true_residual) <= 1e-6 + 1e-6 * r
    assert info.true_residual < 1.0
    op.close()


def test_nonfinite_rhs_is_reported(cuda_device):
    op = MLFMA.dipoles(inputs.make_dipoles(300, seed=2), PW, max_node_srcs=32).setup()
    b = op.rhs()
    b[3] = np.nan
    with pytest.raises(MlfmaError) as e:
        op.solve(b, max_iter=5)
    assert e.value.code == _lib.MLFMA_ERR_NONFINITE
    op.close()
