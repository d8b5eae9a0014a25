"""ctypes binding of libfmm3dbie_b200.so (declarations in include/fmm3dbie_b200.h).

The library is built in-tree (``python -m fmm3dbie_b200.build``); importing
this module without it raises immediately -- there is no fallback path.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libfmm3dbie_b200.so")

I64 = C.c_int64
DBL = C.c_double
PI64 = C.POINTER(C.c_int64)
PDBL = C.POINTER(C.c_double)
VP = C.c_void_p

STATUS = {
    0: "ok", 1: "bad argument", 2: "CUDA error", 3: "not converged", 4: "breakdown",
    5: "out of memory", 6: "node tables missing", 7: "singular matrix", 8: "timeout",
}


class BieError(RuntimeError):
    def __init__(self, status: int, where: str, msg: str):
        super().__init__(f"{where}: {STATUS.get(status, status)} ({msg})")
        self.status = status


_SIGS = {
    "bie_version": (C.c_char_p, []),
    "bie_last_error": (C.c_char_p, []),
    "bie_init": (C.c_int, [C.c_char_p]),
    "bie_get_npols": (C.c_int, [I64, I64, PI64]),
    "bie_get_disc_exps": (C.c_int, [I64, I64, I64, PDBL, PDBL, PDBL, PDBL]),
    "bie_get_basis_pols": (C.c_int, [PDBL, I64, I64, I64, PDBL]),
    "bie_icosa_npatches": (I64, [I64]),
    "bie_surf_icosa_ellipsoid": (C.c_int, [I64, I64, PDBL, PDBL, PI64, PI64, PI64, PDBL, PDBL]),
    "bie_surf_torus_quad": (C.c_int, [I64, I64, I64, DBL, DBL, DBL, I64, PI64, PI64, PI64,
                                      PDBL, PDBL]),
    "bie_get_centroid_rads": (C.c_int, [I64, PI64, PI64, PI64, I64, PDBL, PDBL, PDBL]),
    "bie_get_rfacs": (C.c_int, [I64, I64, PDBL, PDBL]),
    "bie_get_qwts": (C.c_int, [I64, PI64, PI64, PI64, I64, PDBL, PDBL]),
    "bie_findnearmem": (C.c_int, [PDBL, I64, PDBL, I64, PDBL, I64, PI64]),
    "bie_findnear": (C.c_int, [PDBL, I64, PDBL, I64, PDBL, I64, PI64, PI64]),
    "bie_findnear_gpu": (C.c_int, [PDBL, I64, PDBL, I64, PDBL, I64, PI64, PI64, I64]),
    "bie_get_far_order_gpu": (C.c_int, [DBL, I64, PI64, PI64, PI64, PDBL, PDBL, I64, PDBL, I64,
                                        I64, PDBL, I64, PDBL, I64, PI64, PI64, DBL, PI64, PI64]),
    "bie_oversample_geom_gpu": (C.c_int, [I64, PI64, PI64, PI64, I64, PDBL, PDBL, PI64, PI64, I64,
                                          PDBL]),
    "bie_get_iquad_rsc": (C.c_int, [I64, PI64, I64, I64, PI64, PI64, PI64]),
    "bie_get_far_order": (C.c_int, [DBL, I64, PI64, PI64, PI64, PDBL, PDBL, I64, PDBL, I64, I64,
                                    PDBL, I64, PDBL, I64, PI64, PI64, DBL, PI64, PI64]),
    "bie_oversample_geom": (C.c_int, [I64, PI64, PI64, PI64, I64, PDBL, PDBL, PI64, PI64, I64,
                                      PDBL]),
    "bie_oversample_fun_surf": (C.c_int, [I64, I64, PI64, PI64, PI64, I64, PDBL, PI64, PI64, I64,
                                          PDBL]),
    "bie_get_fmm_thresh": (C.c_int, [I64, I64, PDBL, I64, I64, PDBL, PDBL]),
    "bie_get_patch_id_uvs": (C.c_int, [I64, PI64, PI64, PI64, I64, PI64, PDBL]),
    "bie_hkrand": (DBL, [I64]),
    "bie_getnearquad_lap_comb_dir_eval": (C.c_int, [I64, PI64, PI64, PI64, I64, PDBL, PDBL, I64,
                                                    I64, PDBL, PI64, PDBL, DBL, PDBL, I64, I64,
                                                    PI64, PI64, PI64, DBL, I64, PDBL]),
    "bie_getnearquad_helm_comb_dir_eval": (C.c_int, [I64, PI64, PI64, PI64, I64, PDBL, PDBL, I64,
                                                     I64, PDBL, PI64, PDBL, DBL, PDBL, I64, I64,
                                                     PI64, PI64, PI64, DBL, I64, PDBL]),
    "bie_getnearquad_lap_comb_dir_eval_gpu": (C.c_int, [I64, PI64, PI64, PI64, I64, PDBL, PDBL,
                                                        I64, I64, PDBL, PI64, PDBL, DBL, PDBL,
                                                        I64, I64, PI64, PI64, PI64, DBL, I64,
                                                        PDBL, PI64]),
    "bie_getnearquad_helm_comb_dir_eval_gpu": (C.c_int, [I64, PI64, PI64, PI64, I64, PDBL, PDBL,
                                                         I64, I64, PDBL, PI64, PDBL, DBL, PDBL,
                                                         I64, I64, PI64, PI64, PI64, DBL, I64,
                                                         PDBL, PI64]),
    "bie_set_nearquad_engine": (C.c_int, [I64]),
    "bie_get_nearquad_engine": (I64, []),
    "bie_lpcomp_lap_comb_dir_addsub": (C.c_int, [I64, PI64, PI64, PI64, I64, PDBL, PDBL, DBL, I64,
                                                 PDBL, I64, PDBL, I64, PI64, I64, PI64, PI64, PI64,
                                                 I64, I64, PDBL, PI64, I64, PI64, PDBL, PDBL, I64,
                                                 PDBL, I64, PDBL, PDBL]),
    "bie_lpcomp_helm_comb_dir_addsub": (C.c_int, [I64, PI64, PI64, PI64, I64, PDBL, PDBL, DBL, I64,
                                                  PDBL, I64, PDBL, I64, PI64, I64, PI64, PI64,
                                                  PI64, I64, I64, PDBL, PI64, I64, PI64, PDBL, PDBL,
                                                  I64, PDBL, I64, PDBL, PDBL]),
    "bie_lap_comb_dir_eval_addsub": (C.c_int, [I64, PI64, PI64, PI64, I64, PDBL, PDBL, I64, I64,
                                               PDBL, DBL, PDBL, I64, PI64, PI64, PI64, I64, PDBL,
                                               PI64, I64, PI64, PDBL, PDBL, PDBL, PDBL]),
    "bie_helm_comb_dir_eval_addsub": (C.c_int, [I64, PI64, PI64, PI64, I64, PDBL, PDBL, I64, I64,
                                                PDBL, DBL, PDBL, I64, PI64, PI64, PI64, I64, PDBL,
                                                PI64, I64, PI64, PDBL, PDBL, PDBL, PDBL]),
    "bie_lap_comb_dir_eval": (C.c_int, [I64, PI64, PI64, PI64, I64, PDBL, PDBL, I64, I64, PDBL,
                                        PI64, PDBL, DBL, PDBL, PDBL, PDBL]),
    "bie_helm_comb_dir_eval": (C.c_int, [I64, PI64, PI64, PI64, I64, PDBL, PDBL, I64, I64, PDBL,
                                         PI64, PDBL, DBL, PDBL, PDBL, PDBL]),
    "bie_lap_comb_dir_solver_guru": (C.c_int, [I64, PI64, PI64, PI64, I64, PDBL, PDBL, DBL, PDBL,
                                               I64, I64, PDBL, I64, PI64, PI64, PI64, I64, I64,
                                               PDBL, PI64, I64, PI64, PDBL, PDBL, DBL, PI64, PDBL,
                                               PDBL, PDBL]),
    "bie_helm_comb_dir_solver_guru": (C.c_int, [I64, PI64, PI64, PI64, I64, PDBL, PDBL, DBL, PDBL,
                                                I64, I64, PDBL, I64, PI64, PI64, PI64, I64, I64,
                                                PDBL, PI64, I64, PI64, PDBL, PDBL, DBL, PI64, PDBL,
                                                PDBL, PDBL]),
    "bie_lap_comb_dir_solver": (C.c_int, [I64, PI64, PI64, PI64, I64, PDBL, PDBL, DBL, PDBL, I64,
                                          I64, PDBL, DBL, PI64, PDBL, PDBL, PDBL]),
    "bie_helm_comb_dir_solver": (C.c_int, [I64, PI64, PI64, PI64, I64, PDBL, PDBL, DBL, PDBL, I64,
                                           I64, PDBL, DBL, PI64, PDBL, PDBL, PDBL]),
    "bie_helm_comb_dir_solver_guru_ext": (C.c_int, [I64, PI64, PI64, PI64, I64, PDBL, PDBL, DBL,
                                                    PDBL, I64, I64, I64, PDBL, I64, PI64, PI64,
                                                    PI64, I64, PDBL, PI64, I64, PI64, PDBL, PDBL,
                                                    DBL, I64, PI64, PDBL, PDBL]),
    "bie_plan_create": (C.c_int, [I64, PDBL, I64, PI64, PI64, PI64, I64, PDBL, PDBL, I64, I64,
                                  PDBL, I64, PI64, PI64, PI64, I64, PDBL, PI64, I64, PI64, PDBL,
                                  PDBL, C.POINTER(VP)]),
    "bie_plan_destroy": (C.c_int, [VP]),
    "bie_plan_info": (C.c_int, [VP, PI64]),
    "bie_plan_matvec": (C.c_int, [VP, I64, I64, VP, VP, VP]),
    "bie_plan_solve": (C.c_int, [VP, I64, I64, PDBL, VP, VP, I64, DBL, VP, PI64, PDBL, PDBL, VP]),
    "bie_plan_timing": (C.c_int, [VP, I64, PDBL]),
    "bie_set_oversample_engine": (C.c_int, [I64]),
    "bie_get_oversample_engine": (C.c_int, []),
    "bie_plan_oversample": (C.c_int, [VP, I64, I64, VP, VP, VP]),
    "bie_set_mixed_residual": (C.c_int, [I64]),
    "bie_get_mixed_residual": (C.c_int, []),
    "bie_last_mixed_stats": (C.c_int, [PDBL]),
    "bie_plan_set_far": (C.c_int, [VP, I64, I64, I64, I64]),
    "bie_plan_get_far": (C.c_int, [VP, I64, I64, PI64]),
    "bie_plan_set_far_method": (C.c_int, [VP, I64, I64, DBL, I64, I64, I64, VP]),
    "bie_plan_get_far_method": (C.c_int, [VP, I64, PDBL]),
    "bie_tree_check": (C.c_int, [I64, PDBL, I64, PDBL, DBL, I64, DBL, I64, I64, PDBL]),
    "bie_farfield_dev": (C.c_int, [I64, PDBL, I64, VP, VP, VP, VP, I64, VP, DBL, I64, VP, VP]),
    "bie_farfield_dev_noalloc": (C.c_int, [I64, PDBL, I64, VP, VP, VP, VP, I64, VP, DBL, I64, VP,
                                           VP]),
    "bie_batch_create": (C.c_int, [C.POINTER(VP)]),
    "bie_batch_destroy": (C.c_int, [VP]),
    "bie_batch_add": (C.c_int, [VP, VP]),
    "bie_batch_finalize": (C.c_int, [VP, VP]),
    "bie_batch_info": (C.c_int, [VP, PI64]),
    "bie_batch_set_graph": (C.c_int, [VP, I64]),
    "bie_batch_matvec": (C.c_int, [VP, I64, I64, VP, VP, VP]),
    "bie_batch_solve": (C.c_int, [VP, I64, I64, PDBL, VP, VP, I64, DBL, VP, PI64, PDBL, PDBL, VP]),
    "bie_mlp_create": (C.c_int, [I64, C.POINTER(VP)]),
    "bie_mlp_destroy": (C.c_int, [VP]),
    "bie_mlp_info": (C.c_int, [VP, PI64]),
    "bie_mlp_set_engine": (C.c_int, [VP, I64]),
    "bie_mlp_set_params": (C.c_int, [VP, VP, VP]),
    "bie_mlp_get_params": (C.c_int, [VP, VP, VP]),
    "bie_mlp_forward": (C.c_int, [VP, VP, I64, VP, VP]),
    "bie_mlp_grad": (C.c_int, [VP, VP, VP, I64, VP, VP, VP]),
    "bie_mlp_train_step": (C.c_int, [VP, VP, VP, I64, DBL, VP, VP]),
    "bie_mlp_gather": (C.c_int, [VP, I64, VP, I64, VP, PDBL, C.c_uint64, I64, VP, VP, VP]),
    "bie_mlp_demodulate": (C.c_int, [VP, I64, VP, I64, VP, VP, VP]),
    "bie_mlp_predict_density": (C.c_int, [VP, VP, I64, VP, I64, PDBL, VP, VP]),
    "bie_launch_count": (I64, []),
    "bie_measure_fp32_peak": (C.c_int, [PDBL, PDBL]),
    "bie_measure_mufu_peak": (C.c_int, [PDBL, PDBL]),
}

_lib = None


def lib():
    """Load the shared library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with "
                              "`python -m fmm3dbie_b200.build`")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def exported_symbols():
    return list(_SIGS)


def check(status: int, where: str):
    if status != 0:
        raise BieError(status, where, lib().bie_last_error().decode())


# ---- numpy marshalling helpers ---------------------------------------------
def i64(a):
    a = np.ascontiguousarray(a, dtype=np.int64)
    return a, a.ctypes.data_as(PI64)


def f64(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(PDBL)


def c128(a):
    """complex array -> interleaved float64 view and pointer."""
    a = np.ascontiguousarray(a, dtype=np.complex128)
    v = a.view(np.float64)
    return a, v.ctypes.data_as(PDBL)


def ptr(a):
    if a is None:
        return None
    if a.dtype == np.int64:
        return a.ctypes.data_as(PI64)
    return a.ctypes.data_as(PDBL)
