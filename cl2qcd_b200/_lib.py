"""ctypes binding of ``libc2q_b200.so`` (the C ABI of ``include/cl2qcd_b200.h``).

The library is built in-tree by ``cl2qcd_b200/build.py``; there is no CPU
fallback: if the library is missing or no CUDA device is present, the calls
that need one fail with an exception.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libc2q_b200.so")

OK, SOLVER_STUCK, DID_NOT_SOLVE, TIMEOUT, OOM, BAD_ARG, CUDA_ERROR, NO_DEVICE = 0, -1, -2, -3, -4, -5, -6, -7
EVEN, ODD = 0, 1
WILSON, TWISTEDMASS = 1, 3
OP_AEE, OP_AEE_MINUS, OP_QPLUS_EO, OP_QMINUS_EO, OP_QPLUSQMINUS_EO, OP_AEE_AND_GAMMA5_EO, \
    OP_AEE_MINUS_AND_GAMMA5_EO = range(7)
DIAG_M_TM, DIAG_M_TM_INVERSE, DIAG_M_TM_MINUS, DIAG_M_TM_INVERSE_MINUS, DIAG_M_TM_AND_GAMMA5, \
    DIAG_M_TM_MINUS_AND_GAMMA5 = range(6)
SOLVER_CG, SOLVER_BICGSTAB, SOLVER_BICGSTAB_SAVE = 1, 2, 3
FULL_M_TM_PLUS, FULL_M_TM_MINUS, FULL_QPLUS, FULL_QMINUS, FULL_QPLUSQMINUS = range(5)


class CLattice(C.Structure):
    _fields_ = [("ns", C.c_int), ("nt", C.c_int), ("theta_t", C.c_double), ("theta_s", C.c_double),
                ("use_cp_re", C.c_int), ("use_cp_im", C.c_int), ("cp_re", C.c_double), ("cp_im", C.c_double)]


class CSolverParams(C.Structure):
    _fields_ = [("solver", C.c_int), ("prec", C.c_double), ("rel_tol", C.c_double), ("cgmax", C.c_int),
                ("iter_refresh", C.c_int), ("resid_check_every", C.c_int), ("min_iter", C.c_int),
                ("precision", C.c_int), ("reliable_delta", C.c_double), ("use_rec12", C.c_int),
                ("use_graph", C.c_int), ("use_temporal_gauge", C.c_int)]


class CParams(C.Structure):
    """c2q_params: the reference's inverter input keys (c2q_params_from_kv)."""
    _fields_ = [("lat", CLattice), ("fermion_action", C.c_int), ("kappa", C.c_double), ("mu", C.c_double),
                ("mubar", C.c_double), ("use_eo", C.c_int), ("precision", C.c_int),
                ("use_merge_kernels_fermion", C.c_int), ("use_merge_kernels_spinor", C.c_int),
                ("solver", CSolverParams), ("start_condition", C.c_int), ("initial_conf", C.c_char * 1024),
                ("ignore_checksum_errors", C.c_int), ("source_type", C.c_int), ("source_content", C.c_int),
                ("n_sources", C.c_int), ("source_pos", C.c_int * 4), ("measure_correlators", C.c_int),
                ("correlator_direction", C.c_int)]


class CSolveReport(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int), ("reliable_updates", C.c_int),
                ("resid_sq", C.c_double), ("true_resid_rel", C.c_double), ("seconds", C.c_double),
                ("dslash_applications", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class CRequest(C.Structure):
    _fields_ = [("lat", CLattice), ("gauge_id", C.c_ulonglong), ("kappa", C.c_double), ("mu", C.c_double),
                ("nsrc", C.c_int), ("source_kind", C.c_int), ("source_seed", C.c_ulonglong),
                ("params", CSolverParams), ("solutions", C.c_void_p)]


class CRequestResult(C.Structure):
    _fields_ = [("status", C.c_int), ("nsrc", C.c_int), ("t_submit", C.c_double), ("t_admit", C.c_double),
                ("t_done", C.c_double), ("iterations_max", C.c_int), ("true_resid_rel_max", C.c_double),
                ("solution_norm2", C.c_double), ("footprint_bytes", C.c_longlong)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class CServerStats(C.Structure):
    _fields_ = [("budget_bytes", C.c_longlong), ("gauge_bytes", C.c_longlong), ("reserved_bytes", C.c_longlong),
                ("queued", C.c_int), ("running", C.c_int), ("slots", C.c_int), ("completed", C.c_longlong),
                ("seconds", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


_D = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_P = C.c_void_p

# name -> (restype, argtypes); the declarations of include/cl2qcd_b200.h
SIGNATURES = {
    "c2q_version": (C.c_char_p, []),
    "c2q_params_default": (None, [C.POINTER(CParams)]),
    "c2q_params_from_kv": (C.c_int, [C.c_char_p, C.POINTER(CParams)]),
    "c2q_params_last_error": (C.c_char_p, []),
    "c2q_ctx_create": (C.c_int, [C.POINTER(_P), C.c_int, _P]),
    "c2q_ctx_destroy": (C.c_int, [_P]),
    "c2q_last_error": (C.c_char_p, [_P]),
    "c2q_ctx_synchronize": (C.c_int, [_P]),
    "c2q_ctx_launch_count": (C.c_longlong, [_P]),
    "c2q_ctx_profile": (C.c_int, [_P, C.c_int]),
    "c2q_ctx_profile_read": (C.c_int, [_P, C.c_int, C.POINTER(C.c_longlong), C.POINTER(C.c_double),
                                       C.POINTER(C.c_double)]),
    "c2q_gauge_create": (C.c_int, [_P, C.POINTER(CLattice), C.POINTER(_P)]),
    "c2q_gauge_upload": (C.c_int, [_P, _D]),
    "c2q_gauge_download": (C.c_int, [_P, _D]),
    "c2q_gauge_destroy": (C.c_int, [_P]),
    "c2q_gauge_device_bytes": (C.c_size_t, [_P]),
    "c2q_gauge_unitarity": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "c2q_gauge_reunitarize": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "c2q_spinor_eo_create": (C.c_int, [_P, C.POINTER(CLattice), C.POINTER(_P)]),
    "c2q_spinor_eo_create_precision": (C.c_int, [_P, C.POINTER(CLattice), C.c_int, C.POINTER(_P)]),
    "c2q_spinor_eo_precision": (C.c_int, [_P]),
    "c2q_spinor_eo_convert": (C.c_int, [_P, _P]),
    "c2q_ctx_set_link_format": (C.c_int, [_P, C.c_int]),
    "c2q_ctx_set_autotune": (C.c_int, [_P, C.c_int]),
    "c2q_ctx_set_sweep_choice": (C.c_int, [_P, C.c_int]),
    "c2q_ctx_tune_report": (C.c_int, [_P, C.c_char_p, C.c_int]),
    "c2q_spinor_eo_destroy": (C.c_int, [_P]),
    "c2q_spinor_eo_upload": (C.c_int, [_P, _D]),
    "c2q_spinor_eo_download": (C.c_int, [_P, _D]),
    "c2q_spinor_eo_upload_async": (C.c_int, [_P, _D, _P]),
    "c2q_spinor_eo_download_async": (C.c_int, [_P, _D, _P]),
    "c2q_spinor_eo_zero": (C.c_int, [_P]),
    "c2q_spinor_eo_cold": (C.c_int, [_P]),
    "c2q_convert_to_eoprec": (C.c_int, [_P, _P, _D]),
    "c2q_convert_from_eoprec": (C.c_int, [_D, _P, _P]),
    "c2q_dslash_eo": (C.c_int, [_P, _P, _P, C.c_int, C.c_double]),
    "c2q_dslash_AND_M_tm_inverse_sitediagonal_eo": (C.c_int, [_P, _P, _P, C.c_int, C.c_double, C.c_double,
                                                             C.c_int]),
    "c2q_tm_sitediagonal": (C.c_int, [_P, _P, C.c_double, C.c_int]),
    "c2q_gamma5_eo": (C.c_int, [_P]),
    "c2q_apply_eo": (C.c_int, [C.c_int, _P, _P, _P, C.c_double, C.c_double, C.c_int, C.c_int]),
    "c2q_apply_full": (C.c_int, [C.c_int, _P, _P, _P, _P, _P, C.c_double, C.c_double, C.c_int]),
    "c2q_saxpy": (C.c_int, [_P, C.c_double, C.c_double, _P, _P]),
    "c2q_saxpy_AND_gamma5_eo": (C.c_int, [_P, C.c_double, C.c_double, _P, _P]),
    "c2q_sax": (C.c_int, [_P, C.c_double, C.c_double, _P]),
    "c2q_saxsbypz": (C.c_int, [_P, C.c_double, C.c_double, _P, C.c_double, C.c_double, _P, _P]),
    "c2q_copyData": (C.c_int, [_P, _P]),
    "c2q_scalar_product": (C.c_int, [_P, _P, C.POINTER(C.c_double), C.POINTER(C.c_double)]),
    "c2q_squarenorm": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "c2q_saxpy_AND_squarenorm": (C.c_int, [_P, C.c_double, C.c_double, _P, _P, C.POINTER(C.c_double)]),
    "c2q_scalar_product_eo_noalloc": (C.c_int, [_P, _P, C.c_int, C.c_int, _P, _P]),
    "c2q_solver_params_default": (None, [C.POINTER(CSolverParams)]),
    "c2q_cg": (C.c_int, [_P, C.c_int, _P, _P, C.c_double, C.c_double, C.c_int, C.POINTER(CSolverParams),
                         C.POINTER(CSolveReport)]),
    "c2q_bicgstab": (C.c_int, [_P, C.c_int, _P, _P, C.c_double, C.c_double, C.c_int,
                               C.POINTER(CSolverParams), C.POINTER(CSolveReport)]),
    "c2q_cg_multi": (C.c_int, [C.POINTER(_P), C.c_int, _P, C.POINTER(_P), C.c_int, C.c_double, C.c_double,
                               C.c_int, C.POINTER(CSolverParams), C.POINTER(CSolveReport)]),
    "c2q_perform_inversion_eo": (C.c_int, [_P, _D, _P, _D, C.c_double, C.c_double, C.c_int,
                                           C.POINTER(CSolverParams), C.POINTER(CSolveReport)]),
    "c2q_perform_inversion_eo_fields": (C.c_int, [_P, _P, _P, _P, _D, C.c_double, C.c_double, C.c_int,
                                                  C.POINTER(CSolverParams), C.POINTER(CSolveReport)]),
    "c2q_correlator_ps": (C.c_int, [C.POINTER(_P), C.POINTER(_P), C.c_int, C.c_double, C.c_int, _D]),
    "c2q_cg_full": (C.c_int, [_P, _P, C.c_int, _P, _P, _P, C.c_double, C.c_double, C.c_int,
                              C.POINTER(CSolverParams), C.POINTER(CSolveReport)]),
    "c2q_bicgstab_full": (C.c_int, [_P, _P, C.c_int, _P, _P, _P, C.c_double, C.c_double, C.c_int,
                                    C.POINTER(CSolverParams), C.POINTER(CSolveReport)]),
    "c2q_perform_inversion_full": (C.c_int, [_P, _D, _P, _D, C.c_double, C.c_double, C.c_int,
                                             C.POINTER(CSolverParams), C.POINTER(CSolveReport)]),
    "c2q_gaugemomenta_create": (C.c_int, [_P, C.POINTER(CLattice), C.POINTER(_P)]),
    "c2q_gaugemomenta_destroy": (C.c_int, [_P]),
    "c2q_gaugemomenta_zero": (C.c_int, [_P]),
    "c2q_gaugemomenta_upload": (C.c_int, [_P, _D]),
    "c2q_gaugemomenta_download": (C.c_int, [_P, _D]),
    "c2q_gaugemomenta_squarenorm": (C.c_int, [_P, C.POINTER(C.c_double)]),
    "c2q_fermion_force_eo": (C.c_int, [_P, _P, _P, _P, C.c_int, C.c_double]),
    "c2q_gauge_generate": (C.c_int, [_D, C.c_int, C.c_int, C.c_double, C.c_ulonglong]),
    "c2q_source_generate": (C.c_int, [_D, C.c_size_t, C.c_int, C.c_ulonglong]),
    "c2q_spinor_eo_source": (C.c_int, [_P, C.c_int, C.c_ulonglong]),
    "c2q_ildg_read": (C.c_int, [C.c_char_p, C.c_void_p, C.c_size_t, C.POINTER(C.c_int), C.POINTER(C.c_int),
                                C.POINTER(C.c_int), C.c_char_p, C.c_int, C.POINTER(C.c_uint), C.POINTER(C.c_uint),
                                C.POINTER(C.c_int)]),
    "c2q_server_create": (C.c_int, [C.POINTER(_P), C.c_int, C.c_int, C.c_size_t, C.c_int, C.c_int]),
    "c2q_server_add_gauge": (C.c_int, [_P, C.c_ulonglong, C.POINTER(CLattice), _D]),
    "c2q_server_set_heavy_limit": (C.c_int, [_P, C.c_longlong, C.c_int]),
    "c2q_server_submit": (C.c_int, [_P, C.POINTER(CRequest), C.POINTER(C.c_longlong)]),
    "c2q_server_wait": (C.c_int, [_P, C.c_longlong, C.POINTER(CRequestResult)]),
    "c2q_server_get_stats": (C.c_int, [_P, C.POINTER(CServerStats)]),
    "c2q_server_destroy": (C.c_int, [_P]),
    "c2q_request_footprint": (C.c_size_t, [C.POINTER(CLattice), C.c_int, C.c_int]),
}

_lib = None


def load(path: str | None = None) -> C.CDLL:
    """Load the CUDA library (once).  Raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python cl2qcd_b200/build.py` "
                          "(there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class C2QError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code
