"""The product on page-locked host buffers addressed by the device
(mlfma_matvec_mapped): the gather kernel reads x and the final kernel writes
y across the bus in caller order.  It equals the copy path (mlfma_matvec) and
the device path bit for bit, accumulates, applies impedance loads, follows the
reference to 1e-10 under its rules, and refuses pageable buffers."""
import numpy as np
import pytest
import torch

from mlfma_b200 import MLFMA, MlfmaError, inputs
from oracle import ref_lib

pytestmark = pytest.mark.gpu
PW = inputs.PlaneWave()


def cvec(n, seed):
    r = np.random.default_rng(seed)
    return r.standard_normal(n) + 1j * r.standard_normal(n)


def pinned(v):
    t = torch.empty(len(v), dtype=torch.complex128, pin_memory=True)
    t.numpy()[:] = v
    return t


@pytest.mark.parametrize("precision", [0, 1])
def test_mapped_matches_copy_path(cuda_device, precision):
    mesh = inputs.make_icosphere(4, radius=1.5)
    op = MLFMA.rwg(mesh, PW, max_node_srcs=24, ref_compat=0, self_terms=1, precision=precision).setup()
    x = cvec(op.n, 3)
    xp, yp = pinned(x), pinned(np.zeros(op.n))
    for _ in range(2):
        op.matvec_mapped(xp.data_ptr(), yp.data_ptr())
        assert np.array_equal(yp.numpy(), op.matvec(x))
    y0 = cvec(op.n, 4)
    yp.numpy()[:] = y0
    op.matvec_mapped(xp.data_ptr(), yp.data_ptr(), accumulate=True)
    assert np.array_equal(yp.numpy(), op.matvec(x, accumulate=True, out=y0.copy()))
    z = cvec(op.n, 5) * 10.0
    op.set_loads(z)
    op.matvec_mapped(xp.data_ptr(), yp.data_ptr())
    assert np.array_equal(yp.numpy(), op.matvec(x))
    op.close()


def test_mapped_matches_reference(cuda_device):
    d = inputs.make_dipoles(4000, seed=9)
    op = MLFMA.dipoles(d, PW, max_node_srcs=24).setup()
    xs = [cvec(op.n, s) for s in (1, 2)]
    yp = pinned(np.zeros(op.n))
    ys = []
    for x in xs:  # the reference's stale-local rule over a call sequence
        op.matvec_mapped(pinned(x).data_ptr(), yp.data_ptr())
        ys.append(yp.numpy().copy())
    if ref_lib.available():
        P = ref_lib.RefProblem("dipole", d, PW, max_node_srcs=24)
        for x, y in zip(xs, ys):
            yr = P.matvec(x)
            assert np.linalg.norm(y - yr) / np.linalg.norm(yr) <= 1e-10
    op.close()


def test_mapped_refuses_pageable(cuda_device):
    op = MLFMA.dipoles(inputs.make_dipoles(500, seed=1), PW, max_node_srcs=24).setup()
    x = cvec(op.n, 1)
    y = np.zeros(op.n, dtype=np.complex128)
    yp = pinned(np.zeros(op.n))
    with pytest.raises(MlfmaError):
        op.matvec_mapped(x.ctypes.data, yp.data_ptr())
    with pytest.raises(MlfmaError):
        op.matvec_mapped(pinned(x).data_ptr(), y.ctypes.data)
    op.close()
