"""Pins the numpy oracle: against the golden fixtures (made by the reference
itself, tests/golden/make_golden.py) and the reference library, plus the
interpolation known answer of the reference's test/tInterp.cpp."""
import os

import numpy as np
import pytest

from conftest import needs_ref
from mlfma_b200 import inputs
from oracle import mlfma_oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PW = inputs.PlaneWave()

# Tolerances.  Dipole operators are well conditioned: rounding only.  The RWG
# patterns come from a closed form that cancels near alpha, beta, gamma = 0
# ((1 - e^{ia})/a^2, ...), so numpy's rounding differs from the reference's by
# up to ~1e-8 relative on these meshes; the product reproduces the reference's
# rounding exactly and is held to 1e-10 in its own tests.
TOL = {"dipole": 1e-12, "rwg": 1e-7}


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def sources(case, g):
    if case["kind"] == "dipole":
        return O.DipoleSources(g.pos, g.mom, PW)
    return O.RWGSources(g.vertices, g.faces, g.rwgs, PW)


@pytest.mark.parametrize("name", ["dipole_n600", "rwg_ico2_r1", "rwg_ico3_r1"])
def test_oracle_matches_golden(name):
    import make_golden as mg
    case = mg.CASES[name]
    f = np.load(os.path.join(GOLD, name + ".npz"))
    g = mg.geometry(case)
    orc = O.Oracle(sources(case, g), max_node_srcs=case["max_node_srcs"])
    assert rel(orc.rhs(), f["b"]) <= (0.0 if case["kind"] == "dipole" else 1e-10)
    y = orc.matvec(f["x"])
    assert rel(y, f["y"]) <= TOL[case["kind"]]
    if case["kind"] == "dipole":
        sol, it = O.gmres_reference(orc.matvec, orc.rhs(), max_iter=int(f["iters"]), eps=1e-12)
        assert it == int(f["iters"])
        assert rel(sol, f["sol"]) <= 1e-8


def test_oracle_tables_match_golden():
    t = np.load(os.path.join(GOLD, "tables_root4_k2pi.npz"))
    for lvl in (2, 3):
        lv = O.make_level(lvl, 2 * np.pi, 4.0, 3, 2.0, 3)
        np.testing.assert_array_equal(lv.thetas, t[f"thetas{lvl}"])
        assert np.abs(lv.weights - t[f"weights{lvl}"]).max() <= 1e-15
        T = lv.transl[t["offsets"]][:, :: int(t["dir_stride"])]
        assert np.abs(T - t[f"transl{lvl}"]).max() <= 1e-12 * np.abs(T).max()


def test_interpolation_known_answer():
    """test/tInterp.cpp:232-322: <f, I f> and <A f, f> both approximate
    int |f|^2 dOmega = 1 + 4 pi/3, and agree with each other exactly up to
    rounding because anterpolation is the transpose of interpolation."""
    lv2 = O.make_level(2, 2 * np.pi, 4.0, 3, 2.0, 3)
    lv3 = O.make_level(3, 2 * np.pi, 4.0, 3, 2.0, 3)
    vi, va = O.interp_kat(lv2, lv3, 3)
    exact = 1.0 + 4.0 * np.pi / 3.0
    assert abs(vi - va) <= 1e-12
    assert abs(vi.real - exact) / exact < 0.05
    assert abs(vi.imag) < 1e-12


def test_dense_agrees_with_mlfma_to_approximation_error():
    d = inputs.make_dipoles(700, seed=4)
    orc = O.Oracle(O.DipoleSources(d.pos, d.mom, PW), max_node_srcs=32)
    x = np.random.default_rng(1).standard_normal(700) + 0j
    assert rel(orc.matvec(x), orc.dense() @ x) < 1e-2  # 3-digit angular sampling


@needs_ref
@pytest.mark.parametrize("kind,size,mns", [("dipole", 1500, 16), ("rwg", 2, 6)])
def test_oracle_matches_reference_library(kind, size, mns):
    from oracle import ref_lib
    if kind == "dipole":
        g = inputs.make_dipoles(size, seed=21)
        S = O.DipoleSources(g.pos, g.mom, PW)
    else:
        g = inputs.make_icosphere(size, radius=1.3)
        S = O.RWGSources(g.vertices, g.faces, g.rwgs, PW)
    P = ref_lib.RefProblem(kind, g, PW, max_node_srcs=mns)
    orc = O.Oracle(S, max_node_srcs=mns)
    x = np.random.default_rng(2).standard_normal(S.n) + 1j * np.random.default_rng(3).standard_normal(S.n)
    assert rel(orc.matvec(x), P.matvec(x)) <= TOL[kind]
    # the stale-local rule keeps state across calls in both
    assert rel(orc.matvec(x), P.matvec(x)) <= TOL[kind]
    sol, it = O.gmres_reference(P.matvec, P.rhs(), max_iter=6)
    solr, itr = P.solve(max_iter=6)
    assert it == itr and rel(sol, solr) <= 1e-8
