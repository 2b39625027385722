"""The benchmark workloads as named, seeded inputs, and a small driver that runs
a few products of one of them on the GPU (the command profilers are pointed
at):

    python -m mlfma_b200.workloads sphere_r2 --precision 1 --products 3
    python -m mlfma_b200.workloads sphere_r8 --precision 1 --staged 3 --products 2
    python -m mlfma_b200.workloads sphere_r2 --precision 1 --max-rhs 64 --interp-path 15
    python -m mlfma_b200.workloads sphere_r2 --products 1 --solve 40

sphere_r2: PEC sphere of radius 2 wavelengths, level-5 icosphere (20,480
triangles, 30,720 RWG unknowns), root box 4 wavelengths, boxes split above 54
RWGs, EFIE with self terms.  sphere_r8: radius 8 wavelengths, level-7
icosphere (491,520 RWGs), root box 16 wavelengths, the same rules.
"""
from __future__ import annotations

import argparse
import sys

import numpy as np

from . import MLFMA, default_config, inputs

WORKLOADS = {
    "sphere_r2": dict(level=5, radius=2.0, root_leng=4.0),
    "sphere_r8": dict(level=7, radius=8.0, root_leng=16.0),
}


def planewave() -> inputs.PlaneWave:
    """x-polarised unit plane wave incident along -z, wavelength 1."""
    return inputs.PlaneWave(amplitude=1.0, pol=(1.0, 0.0, 0.0), khat=(0.0, 0.0, -1.0), wavenum=2.0 * np.pi)


def make(name: str, precision: int = 0, max_rhs: int = 1, device: int = 0, **overrides) -> MLFMA:
    """The named workload's operator (not set up)."""
    w = WORKLOADS[name]
    mesh = inputs.make_icosphere(w["level"], radius=w["radius"])
    cfg = dict(quad_prec=2, digits=3, interp_order=3, over_interp=2.0, root_leng=w["root_leng"], max_node_srcs=54,
               device=device, precision=precision, self_terms=1, ref_compat=0, max_rhs=max_rhs)
    cfg.update(overrides)
    return MLFMA.rwg(mesh, planewave(), config=default_config(**cfg))


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("workload", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", type=int, default=0, help="0 FP64, 1 complex-float far field")
    ap.add_argument("--max-rhs", type=int, default=1, help="> 1: products on that many right-hand sides")
    ap.add_argument("--interp-path", type=int, default=None, help="mlfma_set_interp_path mode")
    ap.add_argument("--staged", type=int, default=None, help="mlfma_set_staged_interp mode")
    ap.add_argument("--autotune", action="store_true")
    ap.add_argument("--products", type=int, default=3)
    ap.add_argument("--solve", type=int, default=0,
                    help="> 0: then a GMRES(50) solve of the plane-wave right-hand side, that many iterations")
    ap.add_argument("--flexible", action="store_true",
                    help="the solve as FGMRES(30) with 50 inner iterations per outer step")
    a = ap.parse_args(argv)
    import torch

    op = make(a.workload, precision=a.precision, max_rhs=a.max_rhs).setup()
    if a.autotune:
        op.autotune(1, reps=3)
    if a.interp_path is not None:
        op.interp_path = a.interp_path
    if a.staged is not None:
        op.set_staged_interp(a.staged)
    if a.max_rhs > 1:
        X = torch.randn(a.max_rhs, op.n, dtype=torch.complex128, device="cuda")
        Y = torch.zeros_like(X)
        for _ in range(a.products):
            op.matvec_multi_device(a.max_rhs, X.data_ptr(), Y.data_ptr(), False, 0)
    else:
        x = torch.randn(op.n, dtype=torch.complex128, device="cuda")
        y = torch.zeros_like(x)
        for _ in range(a.products):
            op.matvec_device(x.data_ptr(), y.data_ptr(), False, 0)
    torch.cuda.synchronize()
    if a.solve > 0:
        b = op.rhs()
        if a.flexible:
            op.solve(b, max_iter=a.solve, tol=1e-14, restart=30, flexible=True, inner_iters=50)
        else:
            op.solve(b, max_iter=a.solve, tol=1e-14, restart=50, ref_givens=False)
    op.close()
    print("ok")
    return 0


if __name__ == "__main__":
    sys.exit(main())
