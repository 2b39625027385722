"""The near-field kernels of the one-vector product (mlfma_set_near_kernel):
one tile per thread block (row and column threads), one tile per warp from a
shared-memory ring, and one tile per warp read straight from global memory
(both with a warp reduce-scatter for the row sums).  Same tiles, partial slots and per-target
sums; products agree to FP64 rounding on RWG self tiles with their diagonal
(self terms), dipole self tiles without it, leaves larger than a tile (row
tiles), wide leaf-node blocks (list 3/4 partners) and products through the
transposed operator; the default product still matches the reference."""
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


def clustered(n, seed):
    r = np.random.default_rng(seed)
    pos = np.concatenate([r.uniform(-1.9, 1.9, (n // 2, 3)), 0.05 * r.standard_normal((n - n // 2, 3))])
    return inputs.Dipoles(pos=pos, mom=np.tile([0.0, 1.0, 0.0], (n, 1)))


CASES = {
    "rwg_self_terms": lambda: MLFMA.rwg(inputs.make_icosphere(4, radius=1.0), PW, max_node_srcs=54, self_terms=1,
                                        ref_compat=0),
    "dipoles": lambda: MLFMA.dipoles(inputs.make_dipoles(8000, seed=2), PW, max_node_srcs=24, ref_compat=0),
    "large_leaves": lambda: MLFMA.dipoles(clustered(12000, 3), PW, max_node_srcs=150, ref_compat=0, self_terms=1),
    "uneven": lambda: MLFMA.dipoles(clustered(20000, 4), PW, max_node_srcs=12, max_level=6, ref_compat=0),
}


@pytest.mark.parametrize("case", list(CASES))
def test_near_kernels_agree(cuda_device, case):
    op = CASES[case]().setup()
    x = cvec(op.n, 7)
    op.set_near_kernel(0)
    y0, a0 = op.matvec(x), op.matvec_adjoint(x)
    for kind in (1, 2):
        op.set_near_kernel(kind)
        y1, a1 = op.matvec(x), op.matvec_adjoint(x)
        assert rel(y1, y0) <= 1e-13, kind
        assert rel(a1, a0) <= 1e-13, kind
        assert np.array_equal(op.matvec(x), y1)  # deterministic: fixed summation order
    op.close()
