"""Far-field evaluator (Node::printFarSols, src/fmm/node.cpp:147-178, for any
direction list): the oracle is pinned to the reference library on the CPU, the
device evaluator is checked against both on the GPU."""
import numpy as np
import pytest

from conftest import needs_ref
from mlfma_b200 import MLFMA, inputs
from oracle import mlfma_oracle as O

PW = inputs.PlaneWave()
# RWG patterns go through the reference's closed-form triangle integral
# (RWG::getIntegratedPlaneWave, src/sources/rwg.cpp:46-86).  Its divided
# differences cancel when two of k.D0, k.D2, k.(D0-D2) nearly agree, so one ulp
# of exp/sincos grows to ~1e-7 in a few directions of a random set: numpy
# against the reference's own build already differs by 4e-8 (norm) here.
TOL = {"dipole": 1e-12, "rwg": 1e-6}


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _geom(kind):
    if kind == "dipole":
        g = inputs.make_dipoles(1500, seed=31)
        return g, O.DipoleSources(g.pos, g.mom, PW), 16
    g = inputs.make_icosphere(3, radius=1.1)
    return g, O.RWGSources(g.vertices, g.faces, g.rwgs, PW), 16


def _dirs(nd=97, seed=5):
    r = np.random.default_rng(seed).standard_normal((nd, 3))
    d = r / np.linalg.norm(r, axis=1)[:, None]
    # include the poles and a phi cut
    return np.concatenate([d, [[0, 0, 1.0], [0, 0, -1.0]], MLFMA.phi_cut(36)])


def _cur(n, seed=6):
    r = np.random.default_rng(seed)
    return r.standard_normal(n) + 1j * r.standard_normal(n)


@needs_ref
@pytest.mark.parametrize("kind", ["dipole", "rwg"])
def test_oracle_farfield_matches_reference(kind):
    from oracle import ref_lib
    g, S, mns = _geom(kind)
    P = ref_lib.RefProblem(kind, g, PW, max_node_srcs=mns)
    kh, cur = _dirs(), _cur(S.n)
    assert rel(O.farfield(S, cur, kh, PW.wavenum), P.farfield(cur, kh)) <= TOL[kind]


def test_oracle_farfield_is_transverse():
    g, S, _ = _geom("dipole")
    kh = _dirs()
    F = O.farfield(S, _cur(S.n), kh, PW.wavenum)
    assert np.max(np.abs(np.einsum("dc,dc->d", F, kh))) <= 1e-12 * np.max(np.abs(F))


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["dipole", "rwg"])
def test_device_farfield_matches_oracle(cuda_device, kind):
    g, S, mns = _geom(kind)
    op = (MLFMA.dipoles(g, PW, max_node_srcs=mns) if kind == "dipole"
          else MLFMA.rwg(g, PW, max_node_srcs=mns)).setup()
    kh, cur = _dirs(), _cur(S.n)
    F = op.farfield(cur, kh)
    assert rel(F, O.farfield(S, cur, kh, PW.wavenum)) <= TOL[kind]
    # linear in the currents
    c2 = _cur(S.n, seed=7)
    F2 = op.farfield(c2, kh)
    assert rel(op.farfield(cur + 2.0 * c2, kh), F + 2.0 * F2) <= 1e-12
    op.close()


@pytest.mark.gpu
@needs_ref
def test_device_farfield_of_solution_matches_reference(cuda_device):
    # the reference prints the far field of the GMRES solution on the root grid
    from oracle import ref_lib
    g, S, mns = _geom("dipole")
    P = ref_lib.RefProblem("dipole", g, PW, max_node_srcs=mns)
    x, _ = P.solve(max_iter=8)
    op = MLFMA.dipoles(g, PW, max_node_srcs=mns).setup()
    info = P.angles(0)  # the root's grid, on which printFarSols writes
    th, ph = np.meshgrid(info["thetas"], info["phis"], indexing="ij")
    kh = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], -1).reshape(-1, 3)
    assert rel(op.farfield(x, kh), P.farfield(x, kh)) <= TOL["dipole"]
    op.close()


@pytest.mark.gpu
def test_device_farfield_empty_and_errors(cuda_device):
    g, S, mns = _geom("dipole")
    op = MLFMA.dipoles(g, PW, max_node_srcs=mns)
    with pytest.raises(Exception):
        op.farfield(_cur(S.n), _dirs())  # before setup
    op.setup()
    assert op.farfield(_cur(S.n), np.zeros((0, 3))).shape == (0, 3)
    op.close()
