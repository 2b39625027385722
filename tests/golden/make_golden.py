"""Generate the golden fixtures in tests/golden/ by running the reference itself
(oracle/_ref, built from the reference sources by oracle/ref/Makefile) on small
seeded problems.

    make -C oracle/ref && python tests/golden/make_golden.py

Each fixture stores the problem parameters (the geometry is regenerated from
its seed by mlfma_b200.inputs, and a checksum of it is stored), a seeded x,
the reference's y = A x (first matvec after setup), its right-hand side
b = -V, its GMRES solution after a fixed number of iterations, and the
level-2 angular grid and transfer functions.
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from mlfma_b200 import inputs  # noqa: E402
from oracle import ref_lib  # noqa: E402

CASES = {
    "dipole_n600": dict(kind="dipole", n=600, side=4.0, seed=11, max_node_srcs=16, gmres_iters=12),
    "dipole_n2000": dict(kind="dipole", n=2000, side=4.0, seed=12, max_node_srcs=64, gmres_iters=8),
    "rwg_ico2_r1": dict(kind="rwg", level=2, radius=1.0, max_node_srcs=8, gmres_iters=12),
    "rwg_ico3_r1": dict(kind="rwg", level=3, radius=1.0, max_node_srcs=16, gmres_iters=8),
}


def geometry(case):
    if case["kind"] == "dipole":
        return inputs.make_dipoles(case["n"], side=case["side"], seed=case["seed"])
    return inputs.make_icosphere(case["level"], radius=case["radius"])


def geometry_digest(g) -> str:
    h = hashlib.sha256()
    for a in ((g.pos, g.mom) if hasattr(g, "pos") else (g.vertices, g.faces, g.rwgs)):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def seeded_x(n, seed):
    r = np.random.default_rng(seed)
    return r.standard_normal(n) + 1j * r.standard_normal(n)


TRANSL_OFFSETS = np.arange(0, 316, 15)  # stored subset of the 316 offsets
TRANSL_DIR_STRIDE = 3


def main():
    pw = inputs.PlaneWave()
    tables = {}
    for name, case in CASES.items():
        g = geometry(case)
        P = ref_lib.RefProblem(case["kind"], g, pw, max_node_srcs=case["max_node_srcs"])
        x = seeded_x(P.n, 99)
        y = P.matvec(x)
        b = P.rhs()
        sol, it = P.solve(max_iter=case["gmres_iters"], eps=1e-12)
        np.savez_compressed(
            os.path.join(HERE, name + ".npz"), x=x, y=y, b=b, sol=sol, iters=it,
            info=np.array([P.info()["num_nodes"], P.info()["num_leaves"], P.info()["max_level"]]),
            digest=geometry_digest(g))
        print(name, P.n, P.info(), it)
        # Tables depend only on (k, root box, digits, order, oversampling): all cases share them.
        for lvl in range(2, P.info()["max_level"] + 1):
            if lvl in tables:
                continue
            a = P.angles(lvl)
            T = P.transl(lvl)[TRANSL_OFFSETS][:, ::TRANSL_DIR_STRIDE]
            tables[lvl] = (a["thetas"], a["weights"], T)
    np.savez_compressed(os.path.join(HERE, "tables_root4_k2pi.npz"),
                        offsets=TRANSL_OFFSETS, dir_stride=TRANSL_DIR_STRIDE,
                        **{f"thetas{l}": v[0] for l, v in tables.items()},
                        **{f"weights{l}": v[1] for l, v in tables.items()},
                        **{f"transl{l}": v[2] for l, v in tables.items()})


if __name__ == "__main__":
    main()
