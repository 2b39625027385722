"""M2L transfer functions built on the GPU (Tables::getAlpha, getInterpPsi,
buildTranslationTable, src/fmm/tables.cpp:90-220), which the operator uses,
against the host plan's tables (pinned to the reference's own tables in
tests/test_host_plan.py), on every level of a 4-wavelength cube and of the
16-wavelength root box of the largest benchmark (grids up to 58 x 116).  The
agreement is 1e-14 relative to the largest entry on the finer levels; on the
coarsest 16-wavelength level (L = 28 terms) the multipole sum cancels enough
to turn one-ulp differences of sin, cos and FMA contraction between the host
and the GPU into 5e-14, so the bound there is 1e-13."""
import numpy as np
import pytest

from mlfma_b200 import MLFMA, inputs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("root,n,mns,maxlev", [(4.0, 3000, 8, 0), (16.0, 20000, 2, 6)])
def test_gpu_tables_match_host(cuda_device, root, n, mns, maxlev):
    r = np.random.default_rng(1)
    if root == 4.0:
        d = inputs.make_dipoles(n, seed=2)
    else:
        v = r.standard_normal((n, 3))
        d = inputs.Dipoles(pos=7.99 * v / np.linalg.norm(v, axis=1)[:, None], mom=np.tile([1.0, 0, 0], (n, 1)))
    op = MLFMA.dipoles(d, inputs.PlaneWave(), max_node_srcs=mns, root_leng=root, max_level=maxlev).setup()
    st = op.stats()
    assert st["num_levels_far"] >= 3
    for level in range(2, st["max_level"] + 1):
        host, gpu = op.level_transl(level), op.level_transl_gpu(level)
        err = np.abs(gpu - host).max() / np.abs(host).max()
        assert err <= (1e-13 if op.level_info(level)["nth"] > 40 else 1e-14), (level, err)
    op.close()
