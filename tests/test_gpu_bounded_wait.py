"""The failure path of the bounded mbarrier waits, exercised without a GPU
fault: a wait on a barrier that nothing arrives on runs out, the kernel
returns and reports it, and the context stays usable for a product checked
against the oracle."""
import ctypes

import numpy as np
import pytest

from mlfma_b200 import MLFMA, inputs
from mlfma_b200 import _lib
from oracle import mlfma_oracle as O

pytestmark = pytest.mark.gpu


def test_bounded_wait_runs_out_and_context_survives(cuda_device):
    flag = ctypes.c_int(-1)
    assert _lib.lib().mlfma_check_bounded_wait(0, ctypes.byref(flag)) == 0
    assert flag.value == 1
    pw = inputs.PlaneWave()
    d = inputs.make_dipoles(800, seed=12)
    op = MLFMA.dipoles(d, pw, max_node_srcs=16).setup()
    x = np.random.default_rng(1).standard_normal(op.n) + 0j
    y = op.matvec(x)
    ref = O.Oracle(O.DipoleSources(d.pos, d.mom, pw), max_node_srcs=16).matvec(x)
    assert np.linalg.norm(y - ref) / np.linalg.norm(ref) <= 1e-12
    op.close()
