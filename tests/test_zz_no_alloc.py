"""mlfma_gmres_noalloc: GMRES for callers that cannot allocate device memory
during a solve (a memory budget fixed at start-up, or an allocator policy that
forbids cudaMalloc after initialisation).  It runs on the library's fixed
device workspace; its answer must match mlfma_gmres, call after call.

Collected last (file name) so a failure here cannot hide other results."""
import ctypes

import numpy as np
import pytest

from mlfma_b200 import MLFMA, inputs
from mlfma_b200 import _lib
from mlfma_b200._lib import SolveInfo, SolverOpts

pytestmark = pytest.mark.gpu
TOL = 1e-10  # same tolerance as the other FP64 parity tests


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def solve_noalloc(op, b_dev, x_dev, **kw):
    o = SolverOpts(max_iter=kw["max_iter"], tol=kw["tol"], restart=kw["restart"], ref_givens=kw["ref_givens"],
                   refine=int(kw.get("refine", False)))
    info = SolveInfo()
    code = _lib.lib().mlfma_gmres_noalloc(op._h, ctypes.c_void_p(b_dev.data_ptr()), ctypes.c_void_p(x_dev.data_ptr()),
                                          ctypes.byref(o), ctypes.byref(info))
    return code, info


def test_gmres_noalloc_matches_gmres(cuda_device):
    import torch
    # ref_compat = 0: no state carried between products, so repeated solves of the
    # same system are comparable.
    op = MLFMA.rwg(inputs.make_icosphere(3, radius=1.0), inputs.PlaneWave(), max_node_srcs=16, ref_compat=0).setup()
    b = op.rhs()
    opts = dict(max_iter=40, tol=1e-8, restart=10, ref_givens=False)
    x_ref, info_ref = op.solve(b, **opts)
    b_dev = torch.from_numpy(b).cuda()
    for _ in range(2):  # two calls in a row share the workspace
        x_dev = torch.zeros_like(b_dev)
        code, info = solve_noalloc(op, b_dev, x_dev, **opts)
        assert code in (_lib.MLFMA_OK, _lib.MLFMA_ERR_NOT_CONVERGED)
        assert (code == _lib.MLFMA_OK) == info_ref.converged
        assert info.iterations == info_ref.iterations
        assert rel(x_dev.cpu().numpy(), x_ref) <= TOL
    op.close()


def test_gmres_noalloc_refined_mixed_matches_gmres(cuda_device):
    # A mixed-precision operator with refinement uses the two extra vectors of
    # the workspace (outer solution and right-hand side) and the FP64 far field
    # for its outer residuals.
    import torch
    op = MLFMA.rwg(inputs.make_icosphere(3, radius=1.0), inputs.PlaneWave(), max_node_srcs=16, ref_compat=0,
                   precision=1, self_terms=1).setup()
    b = op.rhs()
    opts = dict(max_iter=300, tol=1e-4, restart=30, ref_givens=False, refine=True)
    x_ref, info_ref = op.solve(b, **opts)
    assert info_ref.converged and info_ref.refinements >= 1
    b_dev = torch.from_numpy(b).cuda()
    for _ in range(2):
        x_dev = torch.zeros_like(b_dev)
        code, info = solve_noalloc(op, b_dev, x_dev, **opts)
        assert code == _lib.MLFMA_OK
        assert info.iterations == info_ref.iterations
        assert info.refinements == info_ref.refinements
        # mlfma_gmres orthogonalises in device-resident steps, this entry point
        # step by step on the fixed workspace: the same arithmetic up to the
        # order of the norm's partial sums, amplified by the complex-float far
        # field to float rounding
        assert abs(info.true_residual - info_ref.true_residual) <= 1e-3 * info_ref.true_residual
        assert rel(x_dev.cpu().numpy(), x_ref) <= 1e-5  # the mixed-precision tolerance
    op.close()


def test_gmres_noalloc_rejects_oversize(cuda_device):
    import torch
    op = MLFMA.dipoles(inputs.make_dipoles(2000, seed=3), inputs.PlaneWave(), max_node_srcs=64).setup()
    b_dev = torch.from_numpy(op.rhs()).cuda()
    x_dev = torch.zeros_like(b_dev)
    code, _ = solve_noalloc(op, b_dev, x_dev, max_iter=5000, tol=1e-6, restart=0, ref_givens=True)
    assert code == _lib.MLFMA_ERR_ARG
    assert "fixed workspace" in _lib.lib().mlfma_last_error().decode()
    op.close()
