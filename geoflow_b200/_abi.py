"""ctypes binding of the libgfgpu C ABI (include/gfgpu.h).

The shared library is built in-tree (geoflow_b200/libgfgpu.so).  Loading
fails loudly when it is missing: there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_LIB_PATH = Path(__file__).resolve().parent / "libgfgpu.so"

c_int, c_double, c_void_p, c_int64 = C.c_int, C.c_double, C.c_void_p, C.c_int64
P_int, P_double, P_int32 = C.POINTER(C.c_int), C.POINTER(C.c_double), C.POINTER(C.c_int32)
P_void = C.POINTER(C.c_void_p)

# status codes
GF_OK = 0
GF_CG_NOCONVERGE, GF_CG_SOLVE, GF_CG_PRECOND, GF_CG_BADITERNUM = 1, 2, 3, 4
GF_ERR_ARG, GF_ERR_CUDA, GF_ERR_UNSUPPORTED, GF_ERR_NOMEM = -1, -2, -3, -4
GF_ERR_NONFINITE, GF_ERR_WATCHDOG, GF_ERR_IO = -5, -6, -7
# enums
GF_F64, GF_F32 = 0, 1
GF_DSS_SUM, GF_DSS_SMOOTH, GF_DSS_MAX, GF_DSS_MIN = 0, 1, 2, 3
GF_NORM_INF, GF_NORM_EUC, GF_NORM_L2, GF_NORM_L1 = 0, 1, 2, 3
GF_PRECOND_NONE, GF_PRECOND_JACOBI, GF_PRECOND_CHEBYSHEV, GF_PRECOND_PMG, GF_PRECOND_PMG64 = (
    0, 1, 2, 3, 4)
GF_CG_FP64, GF_CG_MIXED = 0, 1
GF_PMG_PREPARE, GF_PMG_APPLY64, GF_PMG_APPLY, GF_PMG_STEP, GF_PMG_RESID = 0, 1, 2, 3, 4
GF_PMG_RESTRICT, GF_PMG_PROLONG = 5, 6
GF_GEOM_AFFINE, GF_GEOM_REGULAR, GF_GEOM_DEFORMED, GF_GEOM_EMBEDDED = 0, 1, 2, 3
GF_EQN_ADVECT, GF_EQN_BURGERS, GF_EQN_HEAT = 0, 1, 2
GF_FILTER_BOYD, GF_FILTER_PROJECTION = 0, 1
GF_FP32_APPLY_FMA, GF_FP32_APPLY_TF32 = 0, 1
GF_ICOS_BISECTION, GF_ICOS_LAGRANGIAN = 0, 1
GF_RK1, GF_RK2, GF_RK3, GF_RK4, GF_SSP22, GF_SSP33, GF_SSP34 = 1, 2, 3, 4, 22, 33, 34
GF_ENS_RK, GF_ENS_CG = 0, 1
# gf_integrate_noalloc: fixed scratch of GF_NOALLOC_MAX_BLOCKS blocks of GF_NOALLOC_CHUNK
GF_NOALLOC_CHUNK, GF_NOALLOC_MAX_BLOCKS = 4096, 32768
GF_NOALLOC_MAX_N = GF_NOALLOC_CHUNK * GF_NOALLOC_MAX_BLOCKS


class ProblemDesc(C.Structure):
    _fields_ = [
        ("dim", c_int), ("ne", c_int64), ("n", c_int),
        ("D", P_double), ("W", P_double), ("geom", c_int),
        ("elem_geom", P_double), ("node_geom", P_double), ("mask", P_double),
        ("nclass", c_int64), ("class_ptr", P_int32), ("members", P_int32),
        ("box_ne", c_int * 3), ("box_periodic", c_int * 3), ("node_xyz", P_double),
    ]


class CGTraits(C.Structure):
    _fields_ = [
        ("maxit", c_int), ("normtype", c_int), ("tol", c_double), ("precond", c_int),
        ("precision", c_int), ("inner_tol", c_double), ("max_refine", c_int),
        ("check_every", c_int), ("relative", c_int), ("mixed_apply", c_int),
        ("poly_degree", c_int), ("poly_ratio", c_double),
    ]


class RKTraits(C.Structure):
    _fields_ = [("eqn", c_int), ("nu", c_double), ("nstate", c_int), ("scheme", c_int)]


class GioHeader(C.Structure):
    _fields_ = [
        ("ivers", c_int), ("dim", c_int), ("nelems", C.c_uint64), ("gtype", c_int),
        ("cycle", C.c_uint64), ("time", c_double), ("multivar", c_int),
        ("float_bytes", c_int), ("header_bytes", C.c_uint64), ("ndata", C.c_uint64),
        ("porder_rows", c_int64),
    ]


# name -> (restype, argtypes); every symbol declared in include/gfgpu.h
SIGNATURES = {
    "gf_abi_version": (c_int, []),
    "gf_ctx_create": (c_int, [c_int, c_void_p, P_void]),
    "gf_ctx_destroy": (c_int, [c_void_p]),
    "gf_ctx_last_error": (C.c_char_p, [c_void_p]),
    "gf_ctx_synchronize": (c_int, [c_void_p]),
    "gf_gll_basis": (c_int, [c_int, P_double, P_double, P_double]),
    "gf_box_grid": (c_int, [c_int, P_int, c_int, P_double, P_double, P_int, C.POINTER(P_double),
                            P_double, P_double]),
    "gf_box_classes": (c_int64, [c_int, P_int, c_int, P_int, P_int32, P_int32, P_int32]),
    "gf_classes_from_coords": (c_int64, [c_int, c_int64, C.POINTER(P_double), c_double, P_int32,
                                         P_int32, P_int32]),
    "gf_box_classes_device": (c_int64, [c_void_p, c_int, P_int, c_int, P_int, c_void_p, c_void_p,
                                        c_void_p]),
    "gf_classes_from_coords_device": (c_int64, [c_void_p, c_int, c_int64, P_void, c_double,
                                                c_void_p, c_void_p, c_void_p]),
    "gf_problem_create": (c_int, [c_void_p, C.POINTER(ProblemDesc), P_void]),
    "gf_problem_destroy": (c_int, [c_void_p]),
    "gf_problem_sizes": (c_int, [c_void_p, C.POINTER(c_int64), C.POINTER(c_int64)]),
    "gf_problem_stats": (c_int, [c_void_p, C.POINTER(c_int64)]),
    "gf_set_fp32_apply": (c_int, [c_int]),
    "gf_gather": (c_int, [c_void_p, c_int, c_int64, c_void_p, c_void_p, c_void_p]),
    "gf_dss_fold_copies": (c_int, [c_void_p, c_int, c_int, c_int, c_void_p, c_void_p, c_int64,
                                   c_void_p, c_void_p, c_void_p]),
    "gf_rk_stage_sum": (c_int, [c_void_p, c_int, c_void_p, c_int, c_void_p, c_void_p, c_void_p,
                                c_double, c_double, c_double, c_void_p]),
    "gf_rk_update": (c_int, [c_void_p, c_int, c_void_p, c_double, c_void_p, c_double, c_void_p,
                             c_double, c_double, c_void_p, c_double]),
    "gf_rk_accum": (c_int, [c_void_p, c_int, c_void_p, c_void_p, c_double]),
    "gf_problem_set_imass": (c_int, [c_void_p, P_double]),
    "gf_icos_sizes": (c_int, [c_int, c_int, c_int, C.POINTER(c_int64), C.POINTER(c_int64)]),
    "gf_icos_grid": (c_int, [c_int, c_int, c_double, c_int, C.POINTER(P_double), P_double]),
    "gf_helmholtz_apply": (c_int, [c_void_p, c_int, c_double, c_void_p, c_double, c_void_p, c_int,
                                   c_void_p, c_void_p]),
    "gf_helmholtz_apply_T": (c_int, [c_void_p, c_int, c_double, c_double, c_int, c_void_p,
                                     c_void_p]),
    "gf_mass_apply": (c_int, [c_void_p, c_int, c_int, c_void_p, c_void_p]),
    "gf_grefderiv": (c_int, [c_void_p, c_int, c_void_p, c_int, c_int, c_void_p]),
    "gf_grefdiv": (c_int, [c_void_p, c_int, P_void, c_int, c_void_p]),
    "gf_deriv": (c_int, [c_void_p, c_int, c_void_p, c_int, c_void_p]),
    "gf_advect_apply": (c_int, [c_void_p, c_int, c_void_p, c_int, P_void, c_void_p]),
    "gf_dudt": (c_int, [c_void_p, c_int, c_int, c_double, c_int, P_void, P_void, P_void]),
    "gf_dss": (c_int, [c_void_p, c_int, c_int, c_void_p]),
    "gf_mult": (c_int, [c_void_p, c_int, c_void_p]),
    "gf_integrate": (c_int, [c_void_p, c_int, c_void_p, P_double]),
    "gf_cg_solve": (c_int, [c_void_p, C.POINTER(CGTraits), c_double, c_double, c_int, c_void_p,
                            c_void_p, c_void_p, P_int, P_double, P_double]),
    "gf_cg_solve_host": (c_int, [c_void_p, C.POINTER(CGTraits), c_double, c_double, c_int,
                                 P_double, P_double, P_double, P_int, P_double]),
    "gf_pmg_launch": (c_int, [c_void_p, C.POINTER(CGTraits), c_double, c_double, c_int, c_int,
                              c_int]),
    "gf_rk_advance": (c_int, [c_void_p, c_int, C.POINTER(RKTraits), P_void, P_void, c_double,
                              c_double, c_int]),
    "gf_rk_advance_host": (c_int, [c_void_p, c_int, C.POINTER(RKTraits), P_void, P_void, c_double,
                                   c_double, c_int]),
    "gf_integrate_noalloc": (c_int, [c_int64, c_void_p, c_void_p, c_void_p, c_void_p]),
    "gf_constrain2sphere": (c_int, [c_void_p, c_int, P_void, P_void]),
    "gf_tensor_apply": (c_int, [c_void_p, c_int, P_double, P_double, P_double, c_void_p,
                                c_void_p]),
    "gf_rk_graph_create": (c_int, [c_void_p, c_int, C.POINTER(RKTraits), P_void, P_void, c_double,
                                   c_int, P_void]),
    "gf_filter_matrix": (c_int, [c_int, c_int, c_int, c_double, P_double]),
    "gf_filter_apply": (c_int, [c_void_p, c_int, P_double, P_double, P_double, c_int, P_void]),
    "gf_gio_header_bytes": (c_int64, [c_int, c_int, C.c_uint64, c_int]),
    "gf_gio_write": (c_int, [c_void_p, C.c_char_p, C.POINTER(GioHeader), c_void_p, c_void_p,
                             c_int, c_void_p, C.c_uint64]),
    "gf_gio_write_header": (c_int, [c_void_p, C.c_char_p, C.POINTER(GioHeader), c_void_p,
                                    c_void_p, c_int]),
    "gf_gio_write_data": (c_int, [c_void_p, C.c_char_p, c_int, c_void_p, C.c_uint64,
                                  C.c_uint64]),
    "gf_gio_read_data": (c_int, [c_void_p, C.c_char_p, c_int, c_void_p, C.c_uint64,
                                 C.c_uint64]),
    "gf_gio_read_header": (c_int, [c_void_p, C.c_char_p, c_int, C.POINTER(GioHeader), c_void_p,
                                   c_int64, c_void_p, c_int64]),
    "gf_gio_read": (c_int, [c_void_p, C.c_char_p, c_int, c_void_p, C.c_uint64,
                            C.POINTER(GioHeader)]),
    "gf_graph_ensemble": (c_int, [c_int, P_void, P_void]),
    "gf_graph_launch": (c_int, [c_void_p]),
    "gf_graph_nodes": (c_int, [c_void_p]),
    "gf_graph_destroy": (c_int, [c_void_p]),
    "gf_dudt_vjp": (c_int, [c_void_p, c_int, c_int, c_double, c_int, P_void, P_void, P_void,
                            P_void]),
    "gf_dss_T": (c_int, [c_void_p, c_int, c_int, c_void_p]),
    "gf_rk_step_vjp": (c_int, [c_void_p, c_int, C.POINTER(RKTraits), P_void, P_void, c_double,
                               P_void]),
    "gf_adjoint_gradient": (c_int, [c_void_p, C.POINTER(RKTraits), P_void, P_void, P_void,
                                    c_double, c_int, c_int, P_double, P_void]),
    "gf_ensemble_create": (c_int, [c_void_p, c_int, P_void, P_void]),
    "gf_ensemble_destroy": (c_int, [c_void_p]),
    "gf_ensemble_kind": (c_int, [c_void_p]),
    "gf_ensemble_launches": (C.c_uint64, [c_void_p]),
    "gf_ensemble_rk_advance": (c_int, [c_void_p, c_int, C.POINTER(RKTraits), P_void, P_void,
                                       P_double, c_int]),
    "gf_ensemble_cg_solve": (c_int, [c_void_p, C.POINTER(CGTraits), c_double, c_double, P_void,
                                     P_void, P_int, P_double, P_int]),
    "gf_ensemble_tune": (c_int, [c_void_p, c_int, c_int]),
    "gf_ensemble_shape": (c_int, [c_void_p, c_int, P_int, P_int, P_int, P_int, P_double]),
    "gf_ensemble_set_shape": (c_int, [c_void_p, c_int, c_int, c_int, P_int]),
}

_lib = None


class GFError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"libgfgpu error {code}: {msg}")
        self.code = code


def lib_path() -> Path:
    return _LIB_PATH


def load() -> C.CDLL:
    """Load libgfgpu.so and bind every entry point; raises if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not _LIB_PATH.exists():
        raise ImportError(f"{_LIB_PATH} is missing: build it with `python -m geoflow_b200.build` "
                          "(there is no CPU fallback)")
    lib = C.CDLL(str(_LIB_PATH), mode=os.RTLD_NOW | getattr(os, "RTLD_GLOBAL", 0))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def ptr(a):
    """Pointer of a numpy array (as the matching ctypes type) or torch tensor (void*)."""
    import numpy as np
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        if a.dtype == np.float64:
            return a.ctypes.data_as(P_double)
        if a.dtype == np.int32:
            return a.ctypes.data_as(P_int32)
        if a.dtype == np.intc:
            return a.ctypes.data_as(P_int)
        return a.ctypes.data_as(c_void_p)
    return c_void_p(a.data_ptr())


def ptr_array(items):
    arr = (c_void_p * max(1, len(items)))()
    for i, t in enumerate(items):
        arr[i] = None if t is None else t.data_ptr()
    return arr
