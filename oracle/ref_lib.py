"""ctypes binding of oracle/_ref/libmlfma_ref.so, the reference MLFMA compiled
from its own sources (oracle/ref/Makefile).

TEST INFRASTRUCTURE ONLY: used by tests/, the golden-fixture script and the
CPU-baseline leg of bench.py.  The reference keeps its state in class statics,
so one problem exists per process at a time.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libmlfma_ref.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_lp = ctypes.POINTER(ctypes.c_longlong)
_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"reference oracle library missing: {LIB_PATH} (make -C oracle/ref)")
        L = ctypes.CDLL(LIB_PATH)
        L.ref_create_dipoles.argtypes = [_dp, _dp, ctypes.c_int, _dp, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_int]
        L.ref_create_rwg.argtypes = [_dp, ctypes.c_int, _ip, ctypes.c_int, _ip, ctypes.c_int, _dp,
                                     ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                     ctypes.c_double, ctypes.c_int]
        L.ref_info.argtypes = [_ip]
        L.ref_rhs.argtypes = [_dp]
        L.ref_matvec.argtypes = [_dp, _dp]
        L.ref_solve.argtypes = [ctypes.c_int, ctypes.c_double, _dp, _ip]
        L.ref_angles.argtypes = [ctypes.c_int, _ip, _dp, _dp, _dp]
        L.ref_interp.argtypes = [ctypes.c_int, _dp, _ip, _dp, _ip]
        L.ref_transl.argtypes = [ctypes.c_int, _dp]
        L.ref_leaf.argtypes = [ctypes.c_int, _ip, _dp, _ip, _ip]
        L.ref_list_stats.argtypes = [_lp]
        L.ref_entry.argtypes = [ctypes.c_int, ctypes.c_int, _dp]
        L.ref_create_dipoles_file.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                              ctypes.c_double, ctypes.c_double, ctypes.c_int]
        L.ref_create_rwg_files.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                           ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                           ctypes.c_double, ctypes.c_int]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_ip)


class RefProblem:
    """One reference problem: setup happens in the constructor, like the
    reference's main() (src/mlfma.cpp:16-64)."""

    def __init__(self, kind, geom, pw, digits=3, interp_order=3, over_interp=2.0,
                 root_leng=4.0, max_node_srcs=64, quad_prec=2):
        L = lib()
        pwa = np.ascontiguousarray(pw.as_array())
        if kind == "dipole":
            pos = np.ascontiguousarray(geom.pos, dtype=np.float64)
            mom = np.ascontiguousarray(geom.mom, dtype=np.float64)
            rc = L.ref_create_dipoles(_d(pos), _d(mom), geom.n, _d(pwa), digits, interp_order,
                                      over_interp, root_leng, max_node_srcs)
        elif kind == "rwg":
            V = np.ascontiguousarray(geom.vertices, dtype=np.float64)
            F = np.ascontiguousarray(geom.faces, dtype=np.int32)
            E = np.ascontiguousarray(geom.rwgs, dtype=np.int32)
            rc = L.ref_create_rwg(_d(V), V.shape[0], _i(F), F.shape[0], _i(E), E.shape[0], _d(pwa),
                                  quad_prec, digits, interp_order, over_interp, root_leng,
                                  max_node_srcs)
        else:
            raise ValueError(kind)
        if rc != 0:
            raise RuntimeError("reference setup failed")
        self.n = L.ref_num_srcs()
        self.order = interp_order

    @classmethod
    def from_files(cls, kind, paths, pw_path, digits=3, interp_order=3, over_interp=2.0, root_leng=4.0,
                   max_node_srcs=64, quad_prec=2):
        """The reference's own importers on its text files (src/fileio.h):
        paths = dipole file, or (vertices, faces, rwgs).  Raises when an
        importer throws."""
        L = lib()
        self = cls.__new__(cls)
        enc = lambda p: str(p).encode()  # noqa: E731
        if kind == "dipole":
            rc = L.ref_create_dipoles_file(enc(paths), enc(pw_path), digits, interp_order, over_interp, root_leng,
                                           max_node_srcs)
        else:
            v, f, r = paths
            rc = L.ref_create_rwg_files(enc(v), enc(f), enc(r), enc(pw_path), quad_prec, digits, interp_order,
                                        over_interp, root_leng, max_node_srcs)
        if rc != 0:
            raise RuntimeError("reference importer failed")
        self.n = L.ref_num_srcs()
        self.order = interp_order
        return self

    def info(self):
        out = np.zeros(3, dtype=np.int32)
        lib().ref_info(_i(out))
        return dict(num_nodes=int(out[0]), num_leaves=int(out[1]), max_level=int(out[2]))

    def rhs(self):
        b = np.zeros(2 * self.n)
        lib().ref_rhs(_d(b))
        return b.view(np.complex128)

    def matvec(self, x):
        xi = np.ascontiguousarray(np.asarray(x, dtype=np.complex128)).view(np.float64)
        y = np.zeros(2 * self.n)
        if lib().ref_matvec(_d(xi), _d(y)) != 0:
            raise RuntimeError("reference matvec failed")
        return y.view(np.complex128)

    def solve(self, max_iter=500, eps=1e-6):
        cur = np.zeros(2 * self.n)
        it = np.zeros(1, dtype=np.int32)
        if lib().ref_solve(max_iter, eps, _d(cur), _i(it)) != 0:
            raise RuntimeError("reference solve failed")
        return cur.view(np.complex128), int(it[0])

    def angles(self, level):
        sz = np.zeros(3, dtype=np.int32)
        if lib().ref_angles(level, _i(sz), None, None, None) != 0:
            raise IndexError(level)
        nth, nph, L = (int(v) for v in sz)
        th, w, ph = np.zeros(nth), np.zeros(nth), np.zeros(nph)
        lib().ref_angles(level, _i(sz), _d(th), _d(w), _d(ph))
        return dict(thetas=th, weights=w, phis=ph, L=L)

    def interp(self, level):
        a0, a1 = self.angles(level), self.angles(level + 1)
        o2 = 2 * self.order
        nth, nph = len(a0["thetas"]), len(a0["phis"])
        tc, tn = np.zeros(nth * o2), np.zeros(nth, dtype=np.int32)
        pc, pn = np.zeros(nph * o2), np.zeros(nph, dtype=np.int32)
        if lib().ref_interp(level, _d(tc), _i(tn), _d(pc), _i(pn)) != 0:
            raise IndexError(level)
        return dict(theta_coef=tc.reshape(nth, o2), theta_near=tn,
                    phi_coef=pc.reshape(nph, o2), phi_near=pn)

    def transl(self, level):
        a = self.angles(level)
        ndir = len(a["thetas"]) * len(a["phis"])
        out = np.zeros(2 * 316 * ndir)
        if lib().ref_transl(level, _d(out)) != 0:
            raise IndexError(level)
        return out.view(np.complex128).reshape(316, ndir)

    def leaves(self):
        res = []
        for i in range(lib().ref_num_leaves()):
            lvl = np.zeros(1, dtype=np.int32)
            c = np.zeros(3)
            ns = np.zeros(1, dtype=np.int32)
            lib().ref_leaf(i, _i(lvl), _d(c), _i(ns), None)
            idx = np.zeros(max(int(ns[0]), 1), dtype=np.int32)
            lib().ref_leaf(i, _i(lvl), _d(c), _i(ns), _i(idx))
            res.append(dict(level=int(lvl[0]), center=c, srcs=idx[: int(ns[0])].copy()))
        return res

    def list_stats(self):
        out = np.zeros(6, dtype=np.int64)
        lib().ref_list_stats(out.ctypes.data_as(_lp))
        keys = ["list2", "list4", "near_pairs", "self_entries", "near_entries", "nonnear_entries"]
        return dict(zip(keys, (int(v) for v in out)))

    def farfield(self, currents, khat):
        """Far field (ndir x 3 complex) of `currents` along unit directions khat."""
        L = lib()
        L.ref_farfield.argtypes = [_dp, ctypes.c_int, _dp, _dp]
        cur = np.ascontiguousarray(np.asarray(currents, dtype=np.complex128)).view(np.float64)
        kh = np.ascontiguousarray(np.asarray(khat, dtype=np.float64).reshape(-1, 3))
        out = np.zeros(kh.shape[0] * 6)
        if L.ref_farfield(_d(cur), kh.shape[0], _d(kh), _d(out)) != 0:
            raise RuntimeError("reference far field failed")
        return out.view(np.complex128).reshape(-1, 3)

    def entry(self, m, n):
        out = np.zeros(2)
        lib().ref_entry(m, n, _d(out))
        return complex(out[0], out[1])
