"""ctypes binding of libuassa.so (the C-ABI declared in include/ua_ssa.h).

The shared library is built in-tree (``uasource_b200/libuassa.so``) by
``python -m uasource_b200.build`` or ``make -C uasource_b200/csrc``.  There is
no fallback: if the library or a CUDA device is missing, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
# UASOURCE_B200_LIBRARY selects another build of the library (the bounds-checked libuassa_debug.so)
LIB_PATH = os.environ.get("UASOURCE_B200_LIBRARY") or os.path.join(_HERE, "libuassa.so")

UA_OK = 0
UA_ERR_INVALID = -1
UA_ERR_NAN_INPUT = -2
UA_ERR_NOT_CONVERGED = -3
UA_ERR_OOM = -4
UA_ERR_TIMEOUT = -5
UA_ERR_BAD_MESH = -6
UA_ERR_CUDA = -7
UA_ERR_KRYLOV = -8
UA_ERR_NO_DEVICE = -9

UA_PREC_FP64 = 0
UA_ADJ_LOGC, UA_ADJ_PREMUL_M = 1, 2
UA_SLIDING_WEERTMAN, UA_SLIDING_BUDD, UA_SLIDING_TSAI, UA_SLIDING_COULOMB = 0, 1, 2, 3
UA_SLIDING_CORNFORD, UA_SLIDING_UMBI, UA_SLIDING_JOUGHIN = 4, 5, 6
# CtrlVar.SlidingLaw names (Ua2D_DefaultParameters.m:172) -> UA_SLIDING_*
SLIDING_LAWS = {"Weertman": 0, "W": 0, "Budd": 1, "W-N0": 1, "Tsai": 2, "minCW-N0": 2, "Coulomb": 3, "C": 3,
                "Cornford": 4, "rpCW-N0": 4, "Umbi": 5, "rCW-N0": 5, "Joughin": 6, "rCW-V0": 6}
UA_PREC_MIXED = 1
UA_PC_JACOBI = 0
UA_PC_AMG = 1
UA_KRYLOV_GMRES = 0
UA_KRYLOV_BICGSTAB = 1
UA_ASM_R = 0
UA_ASM_RK = 1
UA_ASM_ZERO_R = 2
UA_HOST = 0
UA_DEVICE = 1

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_lp = C.POINTER(C.c_int64)


class ua_mesh_desc(C.Structure):
    _fields_ = [("nnodes", C.c_int32), ("nele", C.c_int32), ("nod", C.c_int32), ("index_base", C.c_int32),
                ("coordinates", _dp), ("connectivity", _ip)]


class ua_params(C.Structure):
    _fields_ = [
        ("kH", C.c_double), ("Hh0", C.c_double),
        ("SpeedZero", C.c_double), ("EpsZero", C.c_double), ("etaZero", C.c_double),
        ("Czero", C.c_double), ("Cmin", C.c_double), ("AGlenmin", C.c_double),
        ("Picard", C.c_int32), ("NRviscosity", C.c_double),
        ("NRitmax", C.c_int32), ("NRitmin", C.c_int32),
        ("NewtonAcceptRatio", C.c_double), ("BacktrackingGammaMin", C.c_double),
        ("LineSearchAllowedToUseExtrapolation", C.c_int32),
        ("BackTrackBeta", C.c_double), ("BackTrackMaxIterations", C.c_int32),
        ("BackTrackMaxExtrapolations", C.c_int32), ("BackTrackExtrapolationRatio", C.c_double),
        ("BackTrackMinXfrac", C.c_double), ("BackTrackMaxFuncSame", C.c_int32),
        ("BackTrackGuardLower", C.c_double), ("BackTrackGuardUpper", C.c_double),
        ("NLtol", C.c_double),
        ("uvDesiredWorkAndForceTolerances", C.c_double * 2),
        ("uvDesiredWorkOrForceTolerances", C.c_double * 2),
        ("uvExitBackTrackingStepLength", C.c_double),
        ("uvAcceptableWorkAndForceTolerances", C.c_double * 2),
        ("uvAcceptableWorkOrForceTolerances", C.c_double * 2),
        ("ModifiedNRuvIntervalCriterion", C.c_int32), ("ModifiedNRuvReductionCriterion", C.c_double),
        ("theta", C.c_double), ("SUPG_beta0", C.c_double), ("uvh_SUPG_tauMultiplier", C.c_double),
        ("uvh_SUPG_tau", C.c_int32),
        ("uvhDesiredWorkAndForceTolerances", C.c_double * 2),
        ("uvhDesiredWorkOrForceTolerances", C.c_double * 2),
        ("uvhExitBackTrackingStepLength", C.c_double),
        ("uvhAcceptableWorkAndForceTolerances", C.c_double * 2),
        ("uvhAcceptableWorkOrForceTolerances", C.c_double * 2),
        ("krylov_rtol", C.c_double), ("krylov_maxit", C.c_int32), ("precision", C.c_int32),
        ("patch_nodes", C.c_int32), ("verbose", C.c_int32), ("profile", C.c_int32),
        ("krylov_adaptive", C.c_int32), ("krylov_precond", C.c_int32), ("spmv_lanes", C.c_int32), ("asm_threads", C.c_int32),
        ("asm_regs", C.c_int32),
        ("uvh_krylov", C.c_int32), ("krylov_restart", C.c_int32),
        ("krylov_eta_c", C.c_double), ("krylov_eta_max", C.c_double), ("precond_bf16", C.c_int32),
        ("amg_smoothed", C.c_int32), ("krylov_full_grid", C.c_int32),
        ("amg_P_refresh", C.c_int32),
        ("uvh_h_sweeps", C.c_int32), ("krylov_sell", C.c_int32),
        ("SlidingLaw", C.c_int32), ("Nzero", C.c_double), ("IncludeMelangeModelPhysics", C.c_int32),
        ("ThicknessConstraints", C.c_int32), ("ThickMin", C.c_double), ("ThicknessConstraintsItMax", C.c_int32),
        ("MaxNumberOfNewlyIntroducedActiveThicknessConstraints", C.c_int32),
        ("MinNumberOfNewlyIntroducedActiveThicknessConstraints", C.c_int32),
    ]


class ua_fields(C.Structure):
    _fields_ = [("location", C.c_int32),
                ("h", _dp), ("S", _dp), ("B", _dp), ("rho", _dp), ("AGlen", _dp), ("n", _dp), ("C", _dp),
                ("m", _dp), ("ub", _dp), ("vb", _dp),
                ("rhow", C.c_double), ("g", C.c_double), ("alpha", C.c_double),
                ("h0", _dp), ("u0", _dp), ("v0", _dp), ("as0", _dp), ("ab0", _dp), ("as1", _dp), ("ab1", _dp),
                ("dadh", _dp), ("h1", _dp), ("dt", C.c_double),
                ("q", _dp), ("muk", _dp), ("V0", _dp),
                ("uo", _dp), ("vo", _dp), ("Co", _dp), ("mo", _dp), ("ua", _dp), ("va", _dp), ("Ca", _dp),
                ("ma", _dp), ("ub_out", _dp), ("vb_out", _dp)]


class ua_measurements(C.Structure):
    _fields_ = [("us", _dp), ("vs", _dp), ("usErr", _dp), ("vsErr", _dp)]


class ua_bcs(C.Structure):
    _fields_ = [("n_ufixed", C.c_int32), ("ufixed_node", _ip), ("ufixed_value", _dp),
                ("n_vfixed", C.c_int32), ("vfixed_node", _ip), ("vfixed_value", _dp),
                ("n_utied", C.c_int32), ("utied_a", _ip), ("utied_b", _ip),
                ("n_vtied", C.c_int32), ("vtied_a", _ip), ("vtied_b", _ip),
                ("n_hfixed", C.c_int32), ("hfixed_node", _ip), ("hfixed_value", _dp),
                ("n_hpos", C.c_int32), ("hpos_node", _ip),
                ("n_normal", C.c_int32), ("normal_node", _ip), ("normal_value", _dp)]


class ua_newton_iter(C.Structure):
    _fields_ = [("iteration", C.c_int32), ("iarm", C.c_int32), ("krylov_its", C.c_int32), ("direction", C.c_int32),
                ("gamma", C.c_double), ("r0", C.c_double), ("r", C.c_double), ("rForce", C.c_double),
                ("rWork", C.c_double)]


class ua_newton_report(C.Structure):
    _fields_ = [("converged", C.c_int32), ("iterations", C.c_int32), ("backtrack_steps", C.c_int32),
                ("krylov_its_total", C.c_int32), ("cauchy_fallbacks", C.c_int32), ("retried", C.c_int32),
                ("r", C.c_double), ("rForce", C.c_double), ("rWork", C.c_double),
                ("assembly_ms", C.c_double), ("solve_ms", C.c_double), ("total_ms", C.c_double),
                ("device_ms", C.c_double), ("kasmK_ms", C.c_double), ("kasmR_ms", C.c_double),
                ("kspmv_ms", C.c_double), ("kasmK_n", C.c_int32), ("kasmR_n", C.c_int32), ("kspmv_n", C.c_int32),
                ("kamgR_ms", C.c_double), ("kamgP_ms", C.c_double), ("kamgR_n", C.c_int32), ("kamgP_n", C.c_int32),
                ("kwork_nnz", C.c_double * 5), ("kwork_rows", C.c_double * 5),
                ("gpu_launches", C.c_int32),
                ("n_iter_records", C.c_int32), ("iters_capacity", C.c_int32),
                ("iters", C.POINTER(ua_newton_iter)),
                ("updates", C.POINTER(C.c_double)), ("update_stride", C.c_int64),
                ("active_set_iterations", C.c_int32), ("active_set_cyclical", C.c_int32),
                ("active_set_converged", C.c_int32), ("n_hpos", C.c_int32), ("hpos_capacity", C.c_int32),
                ("hpos_node", _ip), ("ksetup_ms", C.c_double), ("kkrylov_ms", C.c_double),
                ("ksetup_n", C.c_int32), ("kkrylov_n", C.c_int32)]


UA_TUNE_MAX = 48


class ua_tune_report(C.Structure):
    _fields_ = [("n_candidates", C.c_int32), ("div", C.c_int32 * UA_TUNE_MAX), ("cap", C.c_int32 * UA_TUNE_MAX),
                ("threads", C.c_int32 * UA_TUNE_MAX), ("regs", C.c_int32 * UA_TUNE_MAX),
                ("ms", C.c_double * UA_TUNE_MAX), ("chosen", C.c_int32),
                ("default_ms", C.c_double)]


# symbol -> (restype, argtypes); every function declared in include/ua_ssa.h
SIGNATURES = {
    "ua_version": (C.c_char_p, []),
    "ua_last_error": (C.c_char_p, []),
    "ua_device_count": (C.c_int, []),
    "ua_struct_sizes": (C.c_int, [_lp, C.c_int32]),
    "ua_params_default": (None, [C.POINTER(ua_params)]),
    "ua_mesh_create": (C.c_int, [C.POINTER(ua_mesh_desc), C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]),
    "ua_mesh_create_batch": (C.c_int, [C.POINTER(ua_mesh_desc), C.c_int32, C.c_int32, C.c_int32,
                                       C.POINTER(C.c_void_p)]),
    "ua_mesh_destroy": (None, [C.c_void_p]),
    "ua_mesh_pattern": (C.c_int, [C.c_void_p, C.c_int32, _lp, _lp, _lp]),
    "ua_mesh_info": (C.c_int, [C.c_void_p, C.c_int32, _ip, _ip, _ip, _lp]),
    "ua_mesh_flipped": (C.c_int, [C.c_void_p, _ip]),
    "ua_uv_assemble": (C.c_int, [C.c_void_p, C.POINTER(ua_params), C.POINTER(ua_fields), C.POINTER(ua_bcs),
                                 C.c_int32, _dp, _dp, _dp, _dp]),
    "ua_uv_newton": (C.c_int, [C.c_void_p, C.POINTER(ua_params), C.POINTER(ua_fields), C.POINTER(ua_bcs), _dp,
                               C.c_int32, C.POINTER(ua_newton_report), _dp, _dp]),
    "ua_uv_newton_batch": (C.c_int, [C.c_void_p, C.POINTER(ua_params), C.POINTER(ua_fields), C.POINTER(ua_bcs),
                                     C.POINTER(ua_newton_report)]),
    "ua_uvh_assemble": (C.c_int, [C.c_void_p, C.POINTER(ua_params), C.POINTER(ua_fields), C.c_int32, _dp, _dp, _dp,
                                  _dp]),
    "ua_uvh_newton": (C.c_int, [C.c_void_p, C.POINTER(ua_params), C.POINTER(ua_fields), C.POINTER(ua_bcs), _dp,
                                C.c_int32, C.POINTER(ua_newton_report)]),
    "ua_uvh_newton_batch": (C.c_int, [C.c_void_p, C.POINTER(ua_params), C.POINTER(ua_fields), C.POINTER(ua_bcs),
                                      C.POINTER(ua_newton_report)]),
    "ua_serve_setup": (C.c_int, [C.c_void_p, C.POINTER(ua_params), C.POINTER(ua_bcs)]),
    "ua_serve_begin": (C.c_int, [C.c_void_p, C.POINTER(ua_params), C.c_int32, _ip, C.POINTER(ua_fields)]),
    "ua_serve_step": (C.c_int, [C.c_void_p, C.POINTER(ua_params), _ip, _ip]),
    "ua_serve_result": (C.c_int, [C.c_void_p, C.c_int32, _dp, _dp, C.POINTER(ua_newton_report)]),
    "ua_mem_info": (C.c_int, [C.c_int32, _lp, _lp]),
    "ua_constraint_count": (C.c_int, [C.c_void_p, C.POINTER(ua_bcs), C.c_int32, _ip]),
    "ua_constraint_matrix": (C.c_int, [C.c_void_p, C.POINTER(ua_bcs), _ip, _ip, _dp, _dp]),
    "ua_serve_cancel": (C.c_int, [C.c_void_p, C.c_int32, _ip]),
    "ua_debug_bounds": (C.c_int, [C.c_void_p, _ip, _ip, _lp]),
    "ua_autotune": (C.c_int, [C.c_void_p, C.POINTER(ua_params), C.POINTER(ua_fields), C.c_int32, C.c_int32,
                              C.POINTER(ua_tune_report)]),
    "ua_uv_adjoint_dIdC": (C.c_int, [C.c_void_p, C.POINTER(ua_params), C.POINTER(ua_fields), C.POINTER(ua_bcs),
                                     C.POINTER(ua_measurements), C.c_int32, _dp, _dp, _dp, _dp, _ip]),
    "ua_solve_kape_symmetric": (C.c_int, [C.c_int32, _lp, _lp, _dp, C.c_int32, _lp, _lp, _dp, _dp, _dp, _dp, _dp,
                                          C.c_double, C.c_int32, _ip, C.c_int32]),
    "ua_solve_kape_symmetric_noalloc": (C.c_int, [C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int32,
                                                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                                  C.c_void_p, C.c_double, C.c_int32, _ip, C.c_int32]),
}

_lib = None


class UaError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"libuassa error {code}: {msg}")
        self.code = code


def load():
    """Load libuassa.so (raises if it is missing: there is no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing; build it with `python -m uasource_b200.build`")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc, allow=()):
    if rc != UA_OK and rc not in allow:
        raise UaError(rc, load().ua_last_error().decode())
    return rc


def dptr(a):
    return a.ctypes.data_as(_dp) if a is not None else None


def iptr(a):
    return a.ctypes.data_as(_ip) if a is not None else None


def lptr(a):
    return a.ctypes.data_as(_lp) if a is not None else None
