"""B200 MLFMA operator and GMRES solver (Python front end over the C ABI).

    from mlfma_b200 import MLFMA, inputs
    op = MLFMA.dipoles(inputs.make_dipoles(8192), inputs.PlaneWave())
    op.setup()                 # GPU: patterns + near field
    y = op.matvec(x)           # y = A x   (Solver::evalRvec)
    x, info = op.solve(op.rhs())   # GMRES  (Solver::solve)

Every numerical step runs in libmlfma_b200.so; this module only marshals
arrays.  The reference's setup steps map onto create (tree, lists, tables)
and setup (patterns and near field on the device).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import inputs
from ._lib import (Config, MlfmaError, NotConverged, PlaneWaveC, SolveInfo, SolverOpts, StageTimes, Stats,
                   Traffic, Tuning, check, lib)

__all__ = ["MLFMA", "Batch", "MlfmaError", "NotConverged", "inputs", "default_config"]

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def default_config(**overrides) -> Config:
    c = Config()
    check(lib().mlfma_config_default(ctypes.byref(c)))
    for k, v in overrides.items():
        if not hasattr(c, k):
            raise KeyError(k)
        setattr(c, k, v)
    return c


def _pw(p: inputs.PlaneWave) -> PlaneWaveC:
    c = PlaneWaveC()
    c.amplitude = p.amplitude
    for i in range(3):
        c.pol[i] = p.pol[i]
        c.khat[i] = p.khat[i]
    c.wavenum = p.wavenum
    return c


def read_planewave(path: str) -> inputs.PlaneWave:
    """The plane wave of the reference's text format (mlfma_read_planewave)."""
    c = PlaneWaveC()
    check(lib().mlfma_read_planewave(str(path).encode(), ctypes.byref(c)))
    return inputs.PlaneWave(amplitude=c.amplitude, pol=tuple(c.pol), khat=tuple(c.khat), wavenum=c.wavenum)


def write_solution(path: str, x) -> None:
    """Currents in the reference's solution format (mlfma_write_solution)."""
    a = np.ascontiguousarray(np.asarray(x, dtype=np.complex128).reshape(-1))
    check(lib().mlfma_write_solution(str(path).encode(), a.shape[0], a.view(np.float64).ctypes.data_as(_dp)))


def _cvec(x, n):
    a = np.ascontiguousarray(np.asarray(x, dtype=np.complex128).reshape(-1))
    if a.shape[0] != n:
        raise ValueError(f"expected {n} entries, got {a.shape[0]}")
    return a


@dataclass
class SolveResult:
    iterations: int
    residual: float
    true_residual: float
    seconds: float
    converged: bool
    refinements: int = 0


class MLFMA:
    """One operator instance (one handle)."""

    def __init__(self, handle: ctypes.c_void_p, n: int, kind: str):
        self._h = handle
        self.n = n
        self.kind = kind
        self._ready = False

    # ---------------------------------------------------------------- create
    @classmethod
    def dipoles(cls, d: inputs.Dipoles, pw: inputs.PlaneWave, config: Config | None = None, **kw) -> "MLFMA":
        cfg = config or default_config(**kw)
        pos = np.ascontiguousarray(d.pos, dtype=np.float64)
        mom = np.ascontiguousarray(d.mom, dtype=np.float64)
        h = ctypes.c_void_p()
        p = _pw(pw)
        check(lib().mlfma_create_dipoles(ctypes.byref(cfg), ctypes.byref(p), d.n, pos.ctypes.data_as(_dp),
                                         mom.ctypes.data_as(_dp), ctypes.byref(h)))
        return cls(h, d.n, "dipole")

    @classmethod
    def rwg(cls, m: inputs.RWGMesh, pw: inputs.PlaneWave, config: Config | None = None, **kw) -> "MLFMA":
        cfg = config or default_config(**kw)
        V = np.ascontiguousarray(m.vertices, dtype=np.float64)
        F = np.ascontiguousarray(m.faces, dtype=np.int32)
        E = np.ascontiguousarray(m.rwgs, dtype=np.int32)
        h = ctypes.c_void_p()
        p = _pw(pw)
        check(lib().mlfma_create_rwg(ctypes.byref(cfg), ctypes.byref(p), V.shape[0], V.ctypes.data_as(_dp),
                                     F.shape[0], F.ctypes.data_as(_ip), E.shape[0], E.ctypes.data_as(_ip),
                                     ctypes.byref(h)))
        return cls(h, m.n, "rwg")

    @classmethod
    def dipoles_from_file(cls, path: str, pw: inputs.PlaneWave, config: Config | None = None, **kw) -> "MLFMA":
        """Dipoles from the reference's text format (mlfma_create_dipoles_from_file)."""
        cfg = config or default_config(**kw)
        h = ctypes.c_void_p()
        p = _pw(pw)
        check(lib().mlfma_create_dipoles_from_file(ctypes.byref(cfg), ctypes.byref(p), str(path).encode(),
                                                   ctypes.byref(h)))
        n = ctypes.c_int()
        check(lib().mlfma_num_unknowns(h, ctypes.byref(n)))
        return cls(h, n.value, "dipole")

    @classmethod
    def rwg_from_files(cls, vertices: str, faces: str, rwgs: str, pw: inputs.PlaneWave,
                       config: Config | None = None, **kw) -> "MLFMA":
        """RWG mesh from the reference's text files (mlfma_create_rwg_from_files)."""
        cfg = config or default_config(**kw)
        h = ctypes.c_void_p()
        p = _pw(pw)
        check(lib().mlfma_create_rwg_from_files(ctypes.byref(cfg), ctypes.byref(p), str(vertices).encode(),
                                                str(faces).encode(), str(rwgs).encode(), ctypes.byref(h)))
        n = ctypes.c_int()
        check(lib().mlfma_num_unknowns(h, ctypes.byref(n)))
        return cls(h, n.value, "rwg")

    def setup(self) -> "MLFMA":
        check(lib().mlfma_setup(self._h))
        self._ready = True
        return self

    def close(self) -> None:
        if self._h:
            lib().mlfma_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---------------------------------------------------------------- host queries
    def stats(self) -> dict:
        s = Stats()
        check(lib().mlfma_get_stats(self._h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in Stats._fields_}

    def rhs(self) -> np.ndarray:
        b = np.zeros(self.n, dtype=np.complex128)
        check(lib().mlfma_rhs(self._h, b.view(np.float64).ctypes.data_as(_dp)))
        return b

    def level_info(self, level: int) -> dict:
        sz = np.zeros(3, dtype=np.int32)
        check(lib().mlfma_level_info(self._h, level, sz.ctypes.data_as(_ip), None, None, None))
        nth, nph, L = (int(v) for v in sz)
        th, w, ph = np.zeros(nth), np.zeros(nth), np.zeros(nph)
        check(lib().mlfma_level_info(self._h, level, sz.ctypes.data_as(_ip), th.ctypes.data_as(_dp),
                                     w.ctypes.data_as(_dp), ph.ctypes.data_as(_dp)))
        return dict(thetas=th, weights=w, phis=ph, L=L, nth=nth, nph=nph)

    def level_boxes(self, level: int) -> np.ndarray:
        nb = ctypes.c_int()
        check(lib().mlfma_level_boxes(self._h, level, ctypes.byref(nb), None))
        c = np.zeros((max(nb.value, 1), 3), dtype=np.int32)
        check(lib().mlfma_level_boxes(self._h, level, ctypes.byref(nb), c.ctypes.data_as(_ip)))
        return c[: nb.value]

    def level_transl(self, level: int) -> np.ndarray:
        info = self.level_info(level)
        ndir = info["nth"] * info["nph"]
        out = np.zeros(316 * ndir, dtype=np.complex128)
        check(lib().mlfma_level_transl(self._h, level, out.view(np.float64).ctypes.data_as(_dp)))
        return out.reshape(316, ndir)

    def level_transl_gpu(self, level: int) -> np.ndarray:
        """The level's transfer functions as built on the GPU (after setup)."""
        info = self.level_info(level)
        ndir = info["nth"] * info["nph"]
        out = np.zeros(316 * ndir, dtype=np.complex128)
        check(lib().mlfma_level_transl_gpu(self._h, level, out.view(np.float64).ctypes.data_as(_dp)))
        return out.reshape(316, ndir)

    def far_leaves(self):
        """(info[:, (level, box, src0, nsrc)], perm) with perm[tree slot] = caller index."""
        cnt = ctypes.c_int()
        check(lib().mlfma_far_leaves(self._h, ctypes.byref(cnt), None, None))
        info = np.zeros((max(cnt.value, 1), 4), dtype=np.int32)
        perm = np.zeros(self.n, dtype=np.int32)
        check(lib().mlfma_far_leaves(self._h, ctypes.byref(cnt), info.ctypes.data_as(_ip),
                                     perm.ctypes.data_as(_ip)))
        return info[: cnt.value], perm

    def tree_export(self, which: int) -> np.ndarray:
        """The octree (0: 14 ints per node), source order (1) or a list (2
        neighbours, 3 list 1, 4 list 2, 5 list 4: per node its length, then
        node ids) as one int32 array (mlfma_tree_export)."""
        cnt = ctypes.c_longlong()
        check(lib().mlfma_tree_export(self._h, which, None, 0, ctypes.byref(cnt)))
        out = np.zeros(max(cnt.value, 1), dtype=np.int32)
        check(lib().mlfma_tree_export(self._h, which, out.ctypes.data_as(_ip), out.size, ctypes.byref(cnt)))
        return out[: cnt.value]

    def rwg_patterns_host(self) -> np.ndarray:
        n = self.stats()["pattern_elems"]
        out = np.zeros(2 * n, dtype=np.complex128)
        check(lib().mlfma_rwg_patterns_host(self._h, out.view(np.float64).ctypes.data_as(_dp), out.size * 2))
        return out

    # ---------------------------------------------------------------- device
    def matvec(self, x, accumulate: bool = False, out: np.ndarray | None = None) -> np.ndarray:
        xv = _cvec(x, self.n)
        y = out if out is not None else np.zeros(self.n, dtype=np.complex128)
        if y.dtype != np.complex128 or not y.flags.c_contiguous or y.shape[0] != self.n:
            raise ValueError("out must be a contiguous complex128 vector of length n")
        check(lib().mlfma_matvec(self._h, xv.view(np.float64).ctypes.data_as(_dp),
                                 y.view(np.float64).ctypes.data_as(_dp), int(accumulate)))
        return y

    def matvec_device(self, x_ptr: int, y_ptr: int, accumulate: bool = False, stream: int = 0) -> None:
        check(lib().mlfma_matvec_device(self._h, ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr),
                                        int(accumulate), ctypes.c_void_p(stream)))

    def matvec_mapped(self, x_ptr: int, y_ptr: int, accumulate: bool = False) -> None:
        """y = A x on page-locked, device-mapped host buffers given by address
        (e.g. torch pin_memory tensors): no separate copies (mlfma_matvec_mapped)."""
        check(lib().mlfma_matvec_mapped(self._h, ctypes.cast(x_ptr, _dp), ctypes.cast(y_ptr, _dp), int(accumulate)))

    def solve(self, b=None, max_iter: int = 500, tol: float = 1e-6, restart: int = 0,
              ref_givens: bool = True, raise_on_fail: bool = False, refine: bool = False, inner_tol: float = 0.0,
              flexible: bool = False, inner_iters: int = 0, precond: bool = False):
        """GMRES (Solver::solve).  On a mixed operator, refine=True runs
        iterative refinement: inner GMRES on the mixed operator, outer FP64
        residual; tol then holds for the FP64 residual.  flexible=True runs
        FGMRES(restart): FP64 outer Krylov space, each outer step preconditioned
        by inner_iters GMRES iterations on the operator's own far field.
        precond=True: leaf block-Jacobi right preconditioning (of the inner
        solves when flexible)."""
        bv = self.rhs() if b is None else _cvec(b, self.n)
        x = np.zeros(self.n, dtype=np.complex128)
        o = SolverOpts(max_iter=max_iter, tol=tol, restart=restart, ref_givens=int(ref_givens),
                       refine=int(refine), inner_tol=inner_tol, flexible=int(flexible), inner_iters=inner_iters,
                       precond=int(precond))
        info = SolveInfo()
        code = lib().mlfma_gmres(self._h, bv.view(np.float64).ctypes.data_as(_dp),
                                 x.view(np.float64).ctypes.data_as(_dp), ctypes.byref(o), ctypes.byref(info))
        converged = code == 0
        if code not in (0, 4) or (raise_on_fail and code != 0):
            check(code)
        return x, SolveResult(info.iterations, info.residual, info.true_residual, info.seconds, converged,
                              info.refinements)

    def set_staged_interp(self, mode: int) -> None:
        """bit 0: M2M children summed first in shared memory; bit 1: L2L with the parent
        staged in shared memory; bit 2: their phi passes column-stationary
        (mlfma_set_staged_interp)."""
        check(lib().mlfma_set_staged_interp(self._h, int(mode)))

    def set_schedule(self, schedule: int) -> None:
        """One-vector product schedule bits, as autotune() reports them (mlfma_set_schedule)."""
        check(lib().mlfma_set_schedule(self._h, int(schedule)))

    def set_near_kernel(self, kind: int) -> None:
        """0: one near-field tile per thread block; 1: one per warp (mlfma_set_near_kernel)."""
        check(lib().mlfma_set_near_kernel(self._h, int(kind)))

    def set_inner_operator(self, inner: "MLFMA | None") -> None:
        """Operator of the inner iterations of flexible solves (mlfma_set_inner_operator):
        same sources and tree, e.g. fewer digits or mixed precision.  None detaches it."""
        check(lib().mlfma_set_inner_operator(self._h, inner._h if inner is not None else None))
        self._inner = inner  # keeps it alive while registered

    # ---------------------------------------------------------------- many right-hand sides
    def rhs_planewave(self, pw: inputs.PlaneWave) -> np.ndarray:
        """-V for another incident plane wave (same wavenumber)."""
        b = np.zeros(self.n, dtype=np.complex128)
        p = _pw(pw)
        check(lib().mlfma_rhs_planewave(self._h, ctypes.byref(p), b.view(np.float64).ctypes.data_as(_dp)))
        return b

    def _cmat(self, X):
        a = np.ascontiguousarray(np.asarray(X, dtype=np.complex128))
        if a.ndim != 2 or a.shape[1] != self.n:
            raise ValueError(f"expected (nrhs, {self.n}) array")
        return a

    def matvec_multi(self, X, accumulate: bool = False, out: np.ndarray | None = None) -> np.ndarray:
        """Y = A X for the rows of X (nrhs x n), one batched product."""
        xv = self._cmat(X)
        y = out if out is not None else np.zeros_like(xv)
        check(lib().mlfma_matvec_multi(self._h, xv.shape[0], xv.view(np.float64).ctypes.data_as(_dp),
                                       y.view(np.float64).ctypes.data_as(_dp), int(accumulate)))
        return y

    def matvec_multi_device(self, nrhs: int, x_ptr: int, y_ptr: int, accumulate: bool = False,
                            stream: int = 0) -> None:
        check(lib().mlfma_matvec_multi_device(self._h, nrhs, ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr),
                                              int(accumulate), ctypes.c_void_p(stream)))

    def solve_multi(self, B, max_iter: int = 500, tol: float = 1e-6, restart: int = 0, refine: bool = False,
                    inner_tol: float = 0.0, raise_on_fail: bool = False, flexible: bool = False,
                    inner_iters: int = 0):
        """GMRES on the rows of B (nrhs x n) at once; returns (X, [SolveResult]).
        flexible: FGMRES(restart) per row, inner solves of inner_iters iterations run together."""
        bv = self._cmat(B)
        nr = bv.shape[0]
        x = np.zeros_like(bv)
        o = SolverOpts(max_iter=max_iter, tol=tol, restart=restart, ref_givens=0, refine=int(refine),
                       inner_tol=inner_tol, flexible=int(flexible), inner_iters=inner_iters)
        infos = (SolveInfo * nr)()
        code = lib().mlfma_gmres_multi(self._h, nr, bv.view(np.float64).ctypes.data_as(_dp),
                                       x.view(np.float64).ctypes.data_as(_dp), ctypes.byref(o), infos)
        if code not in (0, 4) or (raise_on_fail and code != 0):
            check(code)
        tol_ok = [i.true_residual <= tol * (1 + 1e-12) for i in infos]
        return x, [SolveResult(i.iterations, i.residual, i.true_residual, i.seconds, ok, i.refinements)
                   for i, ok in zip(infos, tol_ok)]

    def stage_times_multi(self, nrhs: int) -> dict:
        t = StageTimes()
        check(lib().mlfma_time_stages_multi(self._h, nrhs, ctypes.byref(t)))
        return {k: float(getattr(t, k)) for k, _ in StageTimes._fields_}

    # ---------------------------------------------------------------- adjoint and gradients
    def set_loads(self, z=None) -> None:
        """Diagonal loads z (n complex, caller order) added to the operator; None removes them."""
        if z is None:
            check(lib().mlfma_set_loads(self._h, None))
            return
        zv = _cvec(z, self.n)
        check(lib().mlfma_set_loads(self._h, zv.view(np.float64).ctypes.data_as(_dp)))

    def matvec_adjoint(self, x, accumulate: bool = False, out: np.ndarray | None = None) -> np.ndarray:
        """y = A^H x (loads included)."""
        xv = _cvec(x, self.n)
        y = out if out is not None else np.zeros(self.n, dtype=np.complex128)
        check(lib().mlfma_matvec_adjoint(self._h, xv.view(np.float64).ctypes.data_as(_dp),
                                         y.view(np.float64).ctypes.data_as(_dp), int(accumulate)))
        return y

    def solve_adjoint(self, b, max_iter: int = 500, tol: float = 1e-6, restart: int = 0, raise_on_fail: bool = False):
        """GMRES on A^H x = b."""
        bv = _cvec(b, self.n)
        x = np.zeros(self.n, dtype=np.complex128)
        o = SolverOpts(max_iter=max_iter, tol=tol, restart=restart, ref_givens=0)
        info = SolveInfo()
        code = lib().mlfma_gmres_adjoint(self._h, bv.view(np.float64).ctypes.data_as(_dp),
                                         x.view(np.float64).ctypes.data_as(_dp), ctypes.byref(o), ctypes.byref(info))
        if code not in (0, 4) or (raise_on_fail and code != 0):
            check(code)
        return x, SolveResult(info.iterations, info.residual, info.true_residual, info.seconds, code == 0,
                              info.refinements)

    def farfield_adjoint(self, F, khat) -> np.ndarray:
        """g = M^H F, the adjoint of farfield (F: ndir x 3 complex)."""
        kh = np.ascontiguousarray(np.asarray(khat, dtype=np.float64).reshape(-1, 3))
        Fv = np.ascontiguousarray(np.asarray(F, dtype=np.complex128).reshape(kh.shape[0], 3))
        g = np.zeros(self.n, dtype=np.complex128)
        check(lib().mlfma_farfield_adjoint(self._h, kh.shape[0], kh.ctypes.data_as(_dp),
                                           Fv.view(np.float64).ctypes.data_as(_dp),
                                           g.view(np.float64).ctypes.data_as(_dp)))
        return g

    def vjp_farfield_power(self, pws, weights, khat, max_iter: int = 500, tol: float = 1e-10, restart: int = 0):
        """J = sum |F(khat)|^2 for currents solving (A + diag(loads)) I = sum_j w_j b_j, and
        its gradient: returns (J, grad_loads, grad_w, I, (forward info, adjoint info)),
        gradients packed as dJ/dRe + i dJ/dIm."""
        pws = list(pws)
        w = np.ascontiguousarray(np.asarray(weights, dtype=np.complex128).reshape(len(pws)))
        kh = np.ascontiguousarray(np.asarray(khat, dtype=np.float64).reshape(-1, 3))
        parr = (PlaneWaveC * len(pws))(*[_pw(p) for p in pws])
        o = SolverOpts(max_iter=max_iter, tol=tol, restart=restart, ref_givens=0)
        J = ctypes.c_double()
        gz = np.zeros(self.n, dtype=np.complex128)
        gw = np.zeros(len(pws), dtype=np.complex128)
        cur = np.zeros(self.n, dtype=np.complex128)
        infos = (SolveInfo * 2)()
        check(lib().mlfma_vjp_farfield_power(self._h, len(pws), parr, w.view(np.float64).ctypes.data_as(_dp),
                                             kh.shape[0], kh.ctypes.data_as(_dp), ctypes.byref(o), ctypes.byref(J),
                                             gz.view(np.float64).ctypes.data_as(_dp),
                                             gw.view(np.float64).ctypes.data_as(_dp),
                                             cur.view(np.float64).ctypes.data_as(_dp), infos))
        return J.value, gz, gw, cur, tuple(infos)

    def farfield(self, currents, khat) -> np.ndarray:
        """Far field (ndir x 3 complex) of `currents` along unit directions `khat` (ndir x 3)."""
        cur = _cvec(currents, self.n)
        kh = np.ascontiguousarray(np.asarray(khat, dtype=np.float64).reshape(-1, 3))
        out = np.zeros((kh.shape[0], 3), dtype=np.complex128)
        check(lib().mlfma_farfield(self._h, cur.view(np.float64).ctypes.data_as(_dp), kh.shape[0],
                                   kh.ctypes.data_as(_dp), out.view(np.float64).ctypes.data_as(_dp)))
        return out

    def dense_rows(self, rows, x) -> np.ndarray:
        """(A x)[rows] with every interaction evaluated directly in FP64
        (mlfma_dense_rows): the dense reference for sampled rows."""
        r = np.ascontiguousarray(np.asarray(rows, dtype=np.int32).ravel())
        xv = _cvec(x, self.n)
        out = np.zeros(r.shape[0], dtype=np.complex128)
        check(lib().mlfma_dense_rows(self._h, r.shape[0], r.ctypes.data_as(_ip), xv.view(np.float64).ctypes.data_as(_dp),
                                     out.view(np.float64).ctypes.data_as(_dp)))
        return out

    def dense_block_device(self, rows, out_ptr: int, ld: int | None = None) -> None:
        """Rows of the operator's matrix (every interaction direct, FP64) into
        device memory at out_ptr: entry (i, j) at out_ptr + 16 (i ld + j)."""
        r = np.ascontiguousarray(np.asarray(rows, dtype=np.int32).reshape(-1))
        check(lib().mlfma_dense_block_device(self._h, r.shape[0], r.ctypes.data_as(_ip), ctypes.c_void_p(out_ptr),
                                             int(ld if ld is not None else self.n)))

    @staticmethod
    def phi_cut(n: int = 360, theta: float = np.pi / 2) -> np.ndarray:
        """Unit directions of a phi cut at fixed theta (n equally spaced phi)."""
        ph = 2.0 * np.pi * np.arange(n) / n
        return np.stack([np.sin(theta) * np.cos(ph), np.sin(theta) * np.sin(ph), np.full(n, np.cos(theta))], -1)

    def autotune(self, nrhs: int = 1, reps: int = 5) -> dict:
        """Choose launch shapes by timing them on this operator (mlfma_autotune)."""
        t = Tuning()
        check(lib().mlfma_autotune(self._h, nrhs, reps, ctypes.byref(t)))
        return {"m2l_chunk": t.m2l_chunk, "m2m_rows": list(t.m2m_rows), "multi_m2m_rows_fast": t.multi_m2m_rows_fast,
                "multi_l2l_pairs": t.multi_l2l_pairs, "product_ms_before": t.product_ms_before,
                "product_ms_after": t.product_ms_after, "near_blocks_per_sm": t.near_blocks_per_sm,
                "interp_path": t.interp_path, "schedule": t.schedule, "m2m_staged": t.m2m_staged,
                "l2l_staged": t.l2l_staged, "near_kernel": t.near_kernel}

    @property
    def interp_path(self) -> int:
        """Interpolation/anterpolation kernels of the complex-float far field
        (mlfma_set_interp_path) on the tensor cores: bit 0 M2M one vector,
        bit 1 M2M many right-hand sides, bit 2 L2L one vector, bit 3 L2L many;
        0 = CUDA cores."""
        m = ctypes.c_int()
        check(lib().mlfma_get_interp_path(self._h, ctypes.byref(m)))
        return m.value

    @interp_path.setter
    def interp_path(self, mode: int) -> None:
        check(lib().mlfma_set_interp_path(self._h, int(mode)))

    def stream(self) -> int:
        s = ctypes.c_void_p()
        check(lib().mlfma_get_stream(self._h, ctypes.byref(s)))
        return s.value or 0

    def stage_times(self) -> dict:
        t = StageTimes()
        check(lib().mlfma_time_stages(self._h, ctypes.byref(t)))
        return {k: float(getattr(t, k)) for k, _ in StageTimes._fields_}

    def level_times(self) -> dict:
        """Per far level: {"m2m": ms into it, "m2l": ms at it, "l2l": ms out of it} (mlfma_time_levels)."""
        nl = ctypes.c_int()
        check(lib().mlfma_time_levels(self._h, 0, None, ctypes.byref(nl)))
        buf = (ctypes.c_float * (3 * nl.value))()
        check(lib().mlfma_time_levels(self._h, 3 * nl.value, buf, ctypes.byref(nl)))
        return {l: {"m2m": buf[3 * l], "m2l": buf[3 * l + 1], "l2l": buf[3 * l + 2]}
                for l in range(nl.value) if any(buf[3 * l + k] for k in range(3))}

    def traffic(self) -> dict:
        t = Traffic()
        check(lib().mlfma_get_traffic(self._h, ctypes.byref(t)))
        return {k: float(getattr(t, k)) for k, _ in Traffic._fields_}

    def level_patterns(self, level: int, which: int = 0) -> np.ndarray:
        info = self.level_info(level)
        nb = self.level_boxes(level).shape[0]
        ndir = info["nth"] * info["nph"]
        out = np.zeros(nb * ndir * 2, dtype=np.complex128)
        check(lib().mlfma_level_patterns(self._h, level, which, out.view(np.float64).ctypes.data_as(_dp),
                                         out.size))
        return out.reshape(nb, ndir, 2)


class Batch:
    """Many set-up operators applied together (mlfma_batch_*): one graph launch
    runs every product; solve() runs every GMRES at once.  Vectors are lists
    (one array per operator) or one packed array."""

    def __init__(self, ops):
        self.ops = list(ops)
        arr = (ctypes.c_void_p * len(self.ops))(*[o._h.value for o in self.ops])
        h = ctypes.c_void_p()
        check(lib().mlfma_batch_create(len(self.ops), arr, ctypes.byref(h)))
        self._h = h
        self.sizes = [o.n for o in self.ops]
        self.total = sum(self.sizes)

    def _pack(self, xs):
        if isinstance(xs, np.ndarray) and xs.ndim == 1 and xs.shape[0] == self.total:
            return np.ascontiguousarray(xs, dtype=np.complex128)
        return np.ascontiguousarray(np.concatenate([np.asarray(x, dtype=np.complex128) for x in xs]))

    def _split(self, v):
        return np.split(v, np.cumsum(self.sizes)[:-1])

    def matvec(self, xs):
        x = self._pack(xs)
        y = np.zeros_like(x)
        check(lib().mlfma_batch_matvec(self._h, x.view(np.float64).ctypes.data_as(_dp),
                                       y.view(np.float64).ctypes.data_as(_dp)))
        return self._split(y)

    def matvec_device(self, x_ptr: int, y_ptr: int, stream: int = 0) -> None:
        check(lib().mlfma_batch_matvec_device(self._h, ctypes.c_void_p(x_ptr), ctypes.c_void_p(y_ptr),
                                              ctypes.c_void_p(stream)))

    def solve(self, bs, max_iter: int = 500, tol: float = 1e-6, restart: int = 0, refine: bool = False):
        b = self._pack(bs)
        x = np.zeros_like(b)
        o = SolverOpts(max_iter=max_iter, tol=tol, restart=restart, ref_givens=0, refine=int(refine))
        infos = (SolveInfo * len(self.ops))()
        code = lib().mlfma_batch_gmres(self._h, b.view(np.float64).ctypes.data_as(_dp),
                                       x.view(np.float64).ctypes.data_as(_dp), ctypes.byref(o), infos)
        if code not in (0, 4):
            check(code)
        return self._split(x), [SolveResult(i.iterations, i.residual, i.true_residual, i.seconds,
                                            i.true_residual <= tol * (1 + 1e-12), i.refinements) for i in infos]

    def close(self):
        if self._h:
            lib().mlfma_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
