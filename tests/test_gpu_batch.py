"""Many independent operators of uneven size through one graph launch
(mlfma_batch_*): every operator's block of the batched product and of the
batched solve equals its own product and solve."""
import numpy as np
import pytest

from mlfma_b200 import MLFMA, Batch, inputs

pytestmark = pytest.mark.gpu
PW = inputs.PlaneWave()


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def make_ops(count=6, precision=1):
    rng = np.random.default_rng(12)
    ops = []
    for i in range(count):
        n = int(np.exp(rng.uniform(np.log(300), np.log(3000))))
        side = float(rng.uniform(1.0, 3.0))
        d = inputs.make_dipoles(n, seed=40 + i, side=side)
        ops.append(MLFMA.dipoles(d, PW, max_node_srcs=32, root_leng=side, ref_compat=0, self_terms=1,
                                 precision=precision).setup())
    return ops


def test_batch_matvec_matches_each_operator(cuda_device):
    ops = make_ops()
    batch = Batch(ops)
    rng = np.random.default_rng(3)
    xs = [rng.standard_normal(o.n) + 1j * rng.standard_normal(o.n) for o in ops]
    ys = batch.matvec(xs)
    for o, x, y in zip(ops, xs, ys):
        assert rel(y, o.matvec(x)) <= 1e-14
    ys2 = batch.matvec(np.concatenate(xs))  # packed input, second launch of the same graph
    for y, y2 in zip(ys, ys2):
        assert rel(y2, y) <= 1e-14
    batch.close()
    for o in ops:
        o.close()


def test_batch_gmres_matches_each_operator(cuda_device):
    ops = make_ops(count=4, precision=0)
    batch = Batch(ops)
    bs = [o.rhs() for o in ops]
    xs, infos = batch.solve(bs, max_iter=40, tol=1e-12, restart=20)
    for o, b, x, inf in zip(ops, bs, xs, infos):
        x1, i1 = o.solve(b, max_iter=40, tol=1e-12, restart=20, ref_givens=False)
        assert inf.iterations == i1.iterations
        assert rel(x, x1) <= 1e-12
    batch.close()
    for o in ops:
        o.close()
