"""ctypes binding of libmlfma_b200.so (declarations in include/mlfma_b200.h).

The library is loaded from the package directory.  A missing library raises
immediately: there is no fallback implementation.
"""
from __future__ import annotations

import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmlfma_b200.so")

MLFMA_OK = 0
MLFMA_ERR_ARG = 1
MLFMA_ERR_CUDA = 2
MLFMA_ERR_STATE = 3
MLFMA_ERR_NOT_CONVERGED = 4
MLFMA_ERR_NONFINITE = 5
MLFMA_ERR_INTERNAL = 6

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


class Config(ctypes.Structure):
    _fields_ = [("quad_prec", ctypes.c_int), ("digits", ctypes.c_int), ("interp_order", ctypes.c_int),
                ("over_interp", ctypes.c_double), ("root_leng", ctypes.c_double),
                ("max_node_srcs", ctypes.c_int), ("max_level", ctypes.c_int),
                ("ref_compat", ctypes.c_int), ("device", ctypes.c_int), ("precision", ctypes.c_int),
                ("self_terms", ctypes.c_int), ("max_rhs", ctypes.c_int), ("device_tree", ctypes.c_int)]


class PlaneWaveC(ctypes.Structure):
    _fields_ = [("amplitude", ctypes.c_double), ("pol", ctypes.c_double * 3),
                ("khat", ctypes.c_double * 3), ("wavenum", ctypes.c_double)]


class Stats(ctypes.Structure):
    _fields_ = [("num_nodes", ctypes.c_int), ("num_leaves", ctypes.c_int), ("max_level", ctypes.c_int),
                ("num_levels_far", ctypes.c_int), ("list2", ctypes.c_longlong),
                ("list4", ctypes.c_longlong), ("near_pairs", ctypes.c_longlong),
                ("near_entries", ctypes.c_longlong), ("pattern_elems", ctypes.c_longlong),
                ("device_bytes", ctypes.c_longlong), ("launches_per_matvec", ctypes.c_int)]


class StageTimes(ctypes.Structure):
    _fields_ = [(k, ctypes.c_float) for k in
                ("gather", "s2m", "m2m", "m2l", "l2l", "l2t", "near_field", "finish", "total")]


class Traffic(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("s2m", "m2m", "m2l", "l2l", "l2t", "near_field", "total")]


class SolverOpts(ctypes.Structure):
    _fields_ = [("max_iter", ctypes.c_int), ("tol", ctypes.c_double), ("restart", ctypes.c_int),
                ("ref_givens", ctypes.c_int), ("refine", ctypes.c_int), ("inner_tol", ctypes.c_double),
                ("flexible", ctypes.c_int), ("inner_iters", ctypes.c_int), ("precond", ctypes.c_int)]


class SolveInfo(ctypes.Structure):
    _fields_ = [("iterations", ctypes.c_int), ("residual", ctypes.c_double),
                ("true_residual", ctypes.c_double), ("seconds", ctypes.c_double),
                ("refinements", ctypes.c_int)]


class Tuning(ctypes.Structure):
    _fields_ = [("m2l_chunk", ctypes.c_int), ("m2m_rows", ctypes.c_int * 20), ("multi_m2m_rows_fast", ctypes.c_int),
                ("multi_l2l_pairs", ctypes.c_int), ("product_ms_before", ctypes.c_float),
                ("product_ms_after", ctypes.c_float), ("near_blocks_per_sm", ctypes.c_int),
                ("interp_path", ctypes.c_int), ("schedule", ctypes.c_int), ("m2m_staged", ctypes.c_int),
                ("l2l_staged", ctypes.c_int), ("near_kernel", ctypes.c_int)]


# name -> (restype, argtypes); every symbol the header declares.
SIGNATURES = {
    "mlfma_config_default": (ctypes.c_int, [ctypes.POINTER(Config)]),
    "mlfma_create_dipoles": (ctypes.c_int, [ctypes.POINTER(Config), ctypes.POINTER(PlaneWaveC), ctypes.c_int,
                                            _dp, _dp, ctypes.POINTER(ctypes.c_void_p)]),
    "mlfma_create_rwg": (ctypes.c_int, [ctypes.POINTER(Config), ctypes.POINTER(PlaneWaveC), ctypes.c_int, _dp,
                                        ctypes.c_int, _ip, ctypes.c_int, _ip, ctypes.POINTER(ctypes.c_void_p)]),
    "mlfma_setup": (ctypes.c_int, [ctypes.c_void_p]),
    "mlfma_num_unknowns": (ctypes.c_int, [ctypes.c_void_p, _ip]),
    "mlfma_get_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Stats)]),
    "mlfma_rhs": (ctypes.c_int, [ctypes.c_void_p, _dp]),
    "mlfma_matvec": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp, ctypes.c_int]),
    "mlfma_matvec_mapped": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp, ctypes.c_int]),
    "mlfma_matvec_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                           ctypes.c_void_p]),
    "mlfma_gmres": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp, ctypes.POINTER(SolverOpts),
                                   ctypes.POINTER(SolveInfo)]),
    "mlfma_farfield": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_int, _dp, _dp]),
    "mlfma_dense_rows": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _ip, _dp, _dp]),
    "mlfma_check_bounded_wait": (ctypes.c_int, [ctypes.c_int, _ip]),
    "mlfma_gmres_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                           ctypes.POINTER(SolverOpts), ctypes.POINTER(SolveInfo)]),
    "mlfma_rhs_planewave": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(PlaneWaveC), _dp]),
    "mlfma_matvec_multi": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _dp, _dp, ctypes.c_int]),
    "mlfma_matvec_multi_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.c_int, ctypes.c_void_p]),
    "mlfma_gmres_multi": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _dp, _dp, ctypes.POINTER(SolverOpts),
                                         ctypes.POINTER(SolveInfo)]),
    "mlfma_time_stages_multi": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(StageTimes)]),
    "mlfma_set_loads": (ctypes.c_int, [ctypes.c_void_p, _dp]),
    "mlfma_matvec_adjoint": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp, ctypes.c_int]),
    "mlfma_gmres_adjoint": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp, ctypes.POINTER(SolverOpts),
                                           ctypes.POINTER(SolveInfo)]),
    "mlfma_farfield_adjoint": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _dp, _dp, _dp]),
    "mlfma_vjp_farfield_power": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(PlaneWaveC), _dp,
                                                ctypes.c_int, _dp, ctypes.POINTER(SolverOpts), _dp, _dp, _dp, _dp,
                                                ctypes.POINTER(SolveInfo)]),
    "mlfma_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(Tuning)]),
    "mlfma_set_interp_path": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "mlfma_read_planewave": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(PlaneWaveC)]),
    "mlfma_create_dipoles_from_file": (ctypes.c_int, [ctypes.POINTER(Config), ctypes.POINTER(PlaneWaveC),
                                                      ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p)]),
    "mlfma_create_rwg_from_files": (ctypes.c_int, [ctypes.POINTER(Config), ctypes.POINTER(PlaneWaveC),
                                                   ctypes.c_char_p, ctypes.c_char_p, ctypes.c_char_p,
                                                   ctypes.POINTER(ctypes.c_void_p)]),
    "mlfma_write_solution": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, _dp]),
    "mlfma_dense_block_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _ip, ctypes.c_void_p,
                                                ctypes.c_longlong]),
    "mlfma_get_interp_path": (ctypes.c_int, [ctypes.c_void_p, _ip]),
    "mlfma_batch_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                          ctypes.POINTER(ctypes.c_void_p)]),
    "mlfma_batch_size": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)]),
    "mlfma_batch_matvec": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp]),
    "mlfma_batch_matvec_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "mlfma_batch_gmres": (ctypes.c_int, [ctypes.c_void_p, _dp, _dp, ctypes.POINTER(SolverOpts),
                                         ctypes.POINTER(SolveInfo)]),
    "mlfma_batch_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "mlfma_get_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    "mlfma_time_stages": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(StageTimes)]),
    "mlfma_time_levels": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_float), _ip]),
    "mlfma_get_traffic": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Traffic)]),
    "mlfma_level_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _ip, _dp, _dp, _dp]),
    "mlfma_level_boxes": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _ip, _ip]),
    "mlfma_level_patterns": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, ctypes.c_longlong]),
    "mlfma_level_transl": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _dp]),
    "mlfma_level_transl_gpu": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _dp]),
    "mlfma_set_staged_interp": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "mlfma_set_near_kernel": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "mlfma_set_schedule": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "mlfma_set_inner_operator": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "mlfma_far_leaves": (ctypes.c_int, [ctypes.c_void_p, _ip, _ip, _ip]),
    "mlfma_tree_export": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _ip, ctypes.c_longlong,
                                         ctypes.POINTER(ctypes.c_longlong)]),
    "mlfma_rwg_patterns_host": (ctypes.c_int, [ctypes.c_void_p, _dp, ctypes.c_longlong]),
    "mlfma_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "mlfma_last_error": (ctypes.c_char_p, []),
}

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"mlfma_b200 native library not built: {LIB_PATH} "
                               "(run `python -m mlfma_b200.build`)")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


class MlfmaError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class NotConverged(MlfmaError):
    pass


def check(code: int) -> None:
    if code == MLFMA_OK:
        return
    msg = lib().mlfma_last_error().decode(errors="replace")
    if code == MLFMA_ERR_NOT_CONVERGED:
        raise NotConverged(code, msg)
    raise MlfmaError(code, msg)
