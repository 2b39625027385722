"""Host setup (tree, lists, grids, tables, right-hand side, RWG patterns) against
the reference compiled from its sources and against the golden fixtures.
No GPU needed."""
import ctypes
import os

import numpy as np
import pytest

from conftest import needs_ref
from mlfma_b200 import MLFMA, inputs

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PW = inputs.PlaneWave()


def test_grids_and_tables_match_golden():
    t = np.load(os.path.join(GOLD, "tables_root4_k2pi.npz"))
    op = MLFMA.rwg(inputs.make_icosphere(3, radius=1.0), PW, max_node_srcs=16)
    for lvl in range(2, op.stats()["max_level"] + 1):
        info = op.level_info(lvl)
        np.testing.assert_array_equal(info["thetas"], t[f"thetas{lvl}"])   # bit-exact
        np.testing.assert_array_equal(info["weights"], t[f"weights{lvl}"])
        T = op.level_transl(lvl)[t["offsets"]][:, :: int(t["dir_stride"])]
        ref = t[f"transl{lvl}"]
        assert np.abs(T - ref).max() <= 1e-12 * np.abs(ref).max()
    op.close()


@pytest.mark.parametrize("name", ["dipole_n600", "dipole_n2000", "rwg_ico2_r1", "rwg_ico3_r1"])
def test_rhs_and_tree_match_golden(name):
    import make_golden as mg
    case = mg.CASES[name]
    g = mg.geometry(case)
    assert mg.geometry_digest(g) == str(np.load(os.path.join(GOLD, name + ".npz"))["digest"])
    f = np.load(os.path.join(GOLD, name + ".npz"))
    op = (MLFMA.dipoles if case["kind"] == "dipole" else MLFMA.rwg)(g, PW, max_node_srcs=case["max_node_srcs"])
    np.testing.assert_array_equal(op.rhs(), f["b"])  # bit-exact
    st = op.stats()
    assert [st["num_nodes"], st["num_leaves"], st["max_level"]] == f["info"].tolist()
    op.close()


def _pair(kind, seed_or_level, mns, **kw):
    from oracle import ref_lib
    if kind == "dipole":
        g = inputs.make_dipoles(seed_or_level, seed=5)
        op = MLFMA.dipoles(g, PW, max_node_srcs=mns, **kw)
    else:
        g = inputs.make_icosphere(seed_or_level, radius=1.2)
        op = MLFMA.rwg(g, PW, max_node_srcs=mns, **kw)
    return op, ref_lib.RefProblem(kind, g, PW, max_node_srcs=mns)


@needs_ref
@pytest.mark.parametrize("kind,size,mns", [("dipole", 2500, 16), ("dipole", 1200, 64), ("rwg", 3, 12)])
def test_plan_matches_reference(kind, size, mns):
    op, P = _pair(kind, size, mns)
    st, ri, rl = op.stats(), P.info(), P.list_stats()
    assert (st["num_nodes"], st["num_leaves"], st["max_level"]) == (ri["num_nodes"], ri["num_leaves"], ri["max_level"])
    assert st["list2"] == rl["list2"] and st["list4"] == rl["list4"]
    assert st["near_entries"] == rl["near_entries"] + rl["self_entries"] + rl["nonnear_entries"]
    np.testing.assert_array_equal(op.rhs(), P.rhs())
    for lvl in range(2, st["max_level"] + 1):
        a, r = op.level_info(lvl), P.angles(lvl)
        np.testing.assert_array_equal(a["thetas"], r["thetas"])
        np.testing.assert_array_equal(a["weights"], r["weights"])
        np.testing.assert_array_equal(a["phis"], r["phis"])
        T, Tr = op.level_transl(lvl), P.transl(lvl)
        assert np.abs(T - Tr).max() <= 1e-12 * np.abs(Tr).max()
    op.close()


@needs_ref
def test_rwg_patterns_bit_exact():
    """The closed-form RWG integral cancels badly near alpha, beta, gamma = 0;
    the host evaluation reproduces the reference's rounding exactly."""
    from oracle import ref_lib
    op, P = _pair("rwg", 3, 12)
    L = ref_lib.lib()
    L.ref_radpat.argtypes = [ctypes.c_int] * 3 + [ctypes.POINTER(ctypes.c_double)]
    info, perm = op.far_leaves()
    pat = op.rwg_patterns_host()
    by_set = {(lf["level"], tuple(sorted(lf["srcs"]))): (i, lf) for i, lf in enumerate(P.leaves())}
    out = np.zeros(4)
    off = 0
    checked = 0
    for level, box, src0, nsrc in info:
        lv = op.level_info(int(level))
        ndir = lv["nth"] * lv["nph"]
        srcs = perm[src0:src0 + nsrc]
        i, lf = by_set[(int(level), tuple(sorted(srcs)))]
        pos = {s: j for j, s in enumerate(lf["srcs"])}
        for s in range(nsrc):
            for d in range(0, ndir, 5):
                L.ref_radpat(i, pos[srcs[s]], d, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
                at = (off + s * ndir + d) * 2
                assert pat[at] == complex(out[0], out[1]) and pat[at + 1] == complex(out[2], out[3])
                checked += 1
        off += nsrc * ndir
    assert checked > 1000
    op.close()
