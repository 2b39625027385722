"""Octree and interaction lists built on the GPU (device_tree = 1): the same
boxes, node numbering, source order and lists 1, 2 and 4 as the host build
(which restates the Stem ctor's bucketing, src/fmm/stem.cpp:3-26, the
neighbour searches of src/fmm/nbor.cpp:10-644 and
Node::buildInteractionList, src/fmm/node.cpp:61-84), compared array by
array, and the same product bit for bit."""
import time

import numpy as np
import pytest

from mlfma_b200 import MLFMA, inputs

pytestmark = pytest.mark.gpu
PW = inputs.PlaneWave()


def cluster_dipoles(n, seed):
    # strongly non-uniform: Gaussian clusters of very different widths, so
    # leaves sit at many depths and coarse leaves touch deep ones
    r = np.random.default_rng(seed)
    centres = r.uniform(-1.5, 1.5, (6, 3))
    widths = np.array([0.5, 0.2, 0.05, 0.01, 0.002, 0.3])
    k = r.integers(0, 6, n)
    pos = np.clip(centres[k] + widths[k, None] * r.standard_normal((n, 3)), -1.99, 1.99)
    mom = r.standard_normal((n, 3))
    mom /= np.linalg.norm(mom, axis=1)[:, None]
    return inputs.Dipoles(pos=pos, mom=mom)


def grid_dipoles(m):
    # sources exactly on box faces: the strict test src > centre decides
    g = (np.arange(m) - (m - 1) / 2) * (3.0 / m)
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    pos = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    pos = np.concatenate([pos, np.zeros((5, 3)), np.full((3, 3), 0.75)])
    mom = np.tile([0.0, 0.0, 1.0], (pos.shape[0], 1))
    return inputs.Dipoles(pos=pos, mom=mom)


CASES = {
    "uniform": lambda: (inputs.make_dipoles(20000, seed=1), dict(max_node_srcs=8)),
    "cluster": lambda: (cluster_dipoles(30000, 2), dict(max_node_srcs=6, max_level=7)),
    "cluster_cap": lambda: (cluster_dipoles(30000, 3), dict(max_node_srcs=2, max_level=5)),
    # leaves down to ~1e-4 wavelengths: only a 2-point interpolation has
    # enough angular samples there
    "cluster_deep": lambda: (cluster_dipoles(20000, 4), dict(max_node_srcs=4, interp_order=1)),
    "grid": lambda: (grid_dipoles(16), dict(max_node_srcs=3, max_level=7)),
    "rwg": lambda: (inputs.make_icosphere(5, radius=2.0), dict(max_node_srcs=54)),
}


def make(case, device_tree, **kw):
    g, cfg = CASES[case]()
    mk = MLFMA.rwg if case == "rwg" else MLFMA.dipoles
    t = time.perf_counter()
    op = mk(g, PW, device_tree=device_tree, **cfg, **kw)
    return op, time.perf_counter() - t


@pytest.mark.parametrize("case", list(CASES))
def test_device_tree_matches_host(cuda_device, case):
    h, th = make(case, 0)
    d, td = make(case, 1)
    for which in range(6):
        a, b = h.tree_export(which), d.tree_export(which)
        assert a.shape == b.shape, which
        assert np.array_equal(a, b), which
    assert h.stats() == d.stats()
    h.setup()
    d.setup()
    x = np.random.default_rng(4).standard_normal(h.n) + 1j * np.random.default_rng(5).standard_normal(h.n)
    assert np.array_equal(h.matvec(x), d.matvec(x))
    print(f"{case}: n {h.n} nodes {h.stats()['num_nodes']} create host {th:.3f} s device {td:.3f} s")
    h.close()
    d.close()


def test_device_tree_deep_falls_back_to_host(cuda_device):
    # coincident sources with one source per box: the split goes on to the
    # host's depth cap (30 levels), past what the device keys hold (21); a
    # 2-point interpolation keeps boxes that small valid
    r = np.random.default_rng(6)
    pos = np.concatenate([r.uniform(-1, 1, (500, 3)), np.full((2, 3), 0.3)])
    mom = np.tile([1.0, 0.0, 0.0], (pos.shape[0], 1))
    dip = inputs.Dipoles(pos=pos, mom=mom)
    h = MLFMA.dipoles(dip, PW, max_node_srcs=1, interp_order=1, device_tree=0)
    d = MLFMA.dipoles(dip, PW, max_node_srcs=1, interp_order=1, device_tree=1)
    assert h.stats()["max_level"] == 30
    for which in range(6):
        assert np.array_equal(h.tree_export(which), d.tree_export(which))
    h.close()
    d.close()
