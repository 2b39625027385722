"""The one-vector product's schedule (mlfma_set_schedule): translation lists
staged or not, near field early or after aggregation, one or two side streams
for the finer levels' translations, and the far-field chain's kernels as
programmatic dependent launches or plain launches.  Only the staging bit
changes an order of summation; the other bits reorder launches, never
arithmetic, so products under them are equal bit for bit.  Checked in FP64
against the reference (the parity contract, every schedule), on the
complex-float far field, through the transposed product and inside the GMRES
step graphs."""
import numpy as np
import pytest

from mlfma_b200 import MLFMA, inputs
from oracle import ref_lib

pytestmark = pytest.mark.gpu
PW = inputs.PlaneWave()


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def cvec(n, seed):
    r = np.random.default_rng(seed)
    return r.standard_normal(n) + 1j * r.standard_normal(n)


def test_schedules_match_reference(cuda_device):
    """Every schedule, FP64 reference rules: the same products as the
    reference library (1e-10), over a call sequence (the stale-local rule)."""
    mesh = inputs.make_icosphere(3, radius=1.0)
    ys = {}
    for sched in range(16):
        op = MLFMA.rwg(mesh, PW, max_node_srcs=24).setup()
        op.set_schedule(sched)
        xs = [cvec(op.n, s) for s in (1, 2)]
        ys[sched] = [op.matvec(x) for x in xs]
        op.close()
    for sched in range(16):
        for k in range(2):
            assert rel(ys[sched][k], ys[0][k]) <= 1e-13, (sched, k)
            assert np.array_equal(ys[sched][k], ys[sched & 1][k]), (sched, k)
    if ref_lib.available():
        P = ref_lib.RefProblem("rwg", mesh, PW, max_node_srcs=24)
        yr = [P.matvec(cvec(len(ys[0][0]), s)) for s in (1, 2)]
        for sched in range(16):
            for k in range(2):
                assert rel(ys[sched][k], yr[k]) <= 1e-10, (sched, k)


@pytest.mark.parametrize("precision", [0, 1])
def test_chain_launches_do_not_change_results(cuda_device, precision):
    """Bit 3 (programmatic dependent launches of the chain) on and off give
    identical products, adjoint products and GMRES solutions."""
    op = MLFMA.dipoles(inputs.make_dipoles(12000, seed=5), PW, max_node_srcs=24, ref_compat=0, self_terms=1,
                       precision=precision).setup()
    x = cvec(op.n, 3)
    b = op.rhs()
    out = {}
    for pdl in (0, 8):
        op.set_schedule(1 | pdl)
        y = op.matvec(x)
        a = op.matvec_adjoint(x)
        xs, info = op.solve(b, max_iter=60, tol=1e-12, restart=20)
        out[pdl] = (y, a, xs, info.iterations)
    assert np.array_equal(out[0][0], out[8][0])
    assert np.array_equal(out[0][1], out[8][1])
    assert out[0][3] == out[8][3]
    assert rel(out[8][2], out[0][2]) <= 1e-12
    op.close()


def test_schedule_rejects_bad_values(cuda_device):
    op = MLFMA.dipoles(inputs.make_dipoles(500, seed=1), PW, max_node_srcs=24).setup()
    with pytest.raises(Exception):
        op.set_schedule(16)
    with pytest.raises(Exception):
        op.set_schedule(-1)
    op.close()
