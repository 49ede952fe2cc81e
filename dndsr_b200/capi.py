"""ctypes binding of the C-ABI declared in include/dndsb.h.

The shared library is built in-tree (``dndsr_b200/libdndsb.so``) by
``dndsr_b200/build.py``.  Loading fails loudly when it is missing or when no
CUDA device is present: there is no CPU path.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libdndsb.so")

DNDSB_OK = 0
NOALLOC_SCRATCH_DOUBLES = 1 << 20  # DNDSB_NOALLOC_SCRATCH_DOUBLES in include/dndsb.h
ERRORS = {-1: "BADARG", -2: "CUDA", -3: "NONFINITE", -4: "NONPHYSICAL", -5: "UNSUPPORTED", -6: "DIVERGED", -7: "TIMEOUT"}


class DndsbError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class VRSettings(ctypes.Structure):
    _fields_ = [
        ("maxOrder", ctypes.c_int), ("intOrder", ctypes.c_int), ("jacobiRelax", ctypes.c_double), ("SORInstead", ctypes.c_int),
        ("anisotropicLengths", ctypes.c_int), ("scaleType", ctypes.c_int), ("scaleMultiplier", ctypes.c_double),
        ("dirWeightScheme", ctypes.c_int), ("manualDirWeights", ctypes.c_double * 4), ("geomWeightScheme", ctypes.c_int),
        ("geomWeightBias", ctypes.c_double), ("geomWeightPower", ctypes.c_double), ("geomWeightPower1", ctypes.c_double),
        ("geomWeightPower2", ctypes.c_double), ("bcWeight", ctypes.c_double),
    ]


class EulerSettings(ctypes.Structure):
    _fields_ = [
        ("nVars", ctypes.c_int), ("rsType", ctypes.c_int), ("rsFixScale", ctypes.c_double), ("rsIncFScale", ctypes.c_double),
        ("gamma", ctypes.c_double), ("Rgas", ctypes.c_double), ("muGas", ctypes.c_double), ("prGas", ctypes.c_double),
        ("TRef", ctypes.c_double), ("CSutherland", ctypes.c_double), ("muModel", ctypes.c_int), ("ignoreVis", ctypes.c_int),
        ("rsMeanValueEig", ctypes.c_int),
    ]


class LinearSettings(ctypes.Structure):
    _fields_ = [
        ("gmresCode", ctypes.c_int), ("jacobiCode", ctypes.c_int), ("sgsIter", ctypes.c_int), ("nGmresSpace", ctypes.c_int),
        ("nGmresIter", ctypes.c_int), ("precision", ctypes.c_int), ("useGraph", ctypes.c_int), ("meanScale", ctypes.c_double * 8),
    ]


# every function the header declares, with its ctypes signature
_P = ctypes.c_void_p
_PP = ctypes.POINTER(ctypes.c_void_p)
_D = ctypes.POINTER(ctypes.c_double)
_I64 = ctypes.POINTER(ctypes.c_int64)
_I32 = ctypes.POINTER(ctypes.c_int32)
_i = ctypes.c_int
_d = ctypes.c_double
_l = ctypes.c_int64
SIGNATURES = {
    "dndsb_mesh_create": [_PP, _i, _i, _i, _l, _D, _l, _i, _I64, _D, _l, _i, _I64, _D, _I64, _I32, _D, _i, _I64],
    "dndsb_mesh_destroy": [_P],
    "dndsb_mesh_colors": [_P, ctypes.POINTER(ctypes.c_int), _I32],
    "dndsb_vr_create": [_PP, _P, ctypes.POINTER(VRSettings)],
    "dndsb_vr_destroy": [_P],
    "dndsb_vr_construct_metrics": [_P],
    "dndsb_vr_construct_base_and_weight": [_P, _D, _i],
    "dndsb_vr_construct_rec_coeff": [_P],
    "dndsb_vr_sizes": [_P, _I64],
    "dndsb_vr_get_array": [_P, ctypes.c_char_p, _D, _l, _I64],
    "dndsb_vr_do_reconstruction_iter": [_P, _P, _P, _P, _i, _i, _i, _i, _i, _P],
    "dndsb_eval_create": [_PP, _P, ctypes.POINTER(EulerSettings)],
    "dndsb_eval_destroy": [_P],
    "dndsb_eval_initialize_udof": [_P, _i, _d, _P, _P],
    "dndsb_eval_evaluate_dt": [_P, _P, _d, _d, _i, _P, _D, _P],
    "dndsb_eval_evaluate_rhs": [_P, _P, _P, _P, _P],
    "dndsb_eval_evaluate_rhs_full": [_P, _P, _P, _P, _P, _P, _P, _P, _i, _d, ctypes.c_uint64, _P],
    "dndsb_eval_set_deferred_errors": [_P, _i],
    "dndsb_eval_check_errors": [_P, _P],
    "dndsb_eval_lusgs_matrix_init": [_P, _P, _d, _d, _P, _P],
    "dndsb_eval_set_jacobian_mode": [_P, _i, _i],
    "dndsb_eval_lusgs_matrix_to_jacobian_lu": [_P, _d, _P, _P, _P],
    "dndsb_eval_lusgs_matrix_solve_jacobian_lu": [_P, _d, _P, _P, _P, _P, _P, _i, _D, _P],
    "dndsb_eval_lusgs_matrix_init_full": [_P, _P, _d, _d, _P, _P, _i, _d, _P, _P],
    "dndsb_eval_update_sgs": [_P, _d, _P, _P, _P, _P, _P, _i, _i, _i, _D, _P],
    "dndsb_eval_lusgs_matrix_vec": [_P, _d, _P, _P, _P, _P, _P],
    "dndsb_eval_update_lusgs_forward": [_P, _d, _P, _P, _P, _P, _P, _P],
    "dndsb_eval_update_lusgs_backward": [_P, _d, _P, _P, _P, _P, _P, _P],
    "dndsb_eval_fix_umax_filter": [_P, _P, _P],
    "dndsb_eval_lusgs_matrix_vec_t": [_P, _d, _P, _P, _P, _P, _P],
    "dndsb_eval_update_sgs_t": [_P, _d, _P, _P, _P, _P, _P, _i, _i, _i, _P],
    "dndsb_eval_pressure_force": [_P, _i, _D, _P, _P, _D, _P, _P, _P],
    "dndsb_eval_pressure_force_coords": [_P, _i, _D, _P, _P, _P, _P],
    "dndsb_vr_smooth_indicator": [_P, _P, _P, _i, _P, _P],
    "dndsb_eval_limiter_wbap_c": [_P, _P, _P, _P, _P, _d, _d, _i, _P],
    "dndsb_eval_cell_rhs_alpha": [_P, _P, _P, _P, _d, _d, _d, _i, _d, _i, _i, _P, _P, _P],
    "dndsb_eval_cell_rhs_alpha_expansion": [_P, _P, _P, _P, _d, _d, _d, _P],
    "dndsb_eval_add_fixed_increment": [_P, _P, _P, _d, _d, _d, _i, _P, _P],
    "dndsb_eval_evaluate_norm": [_P, _P, _i, _i, _D, _P],
    "dndsb_eval_solve_linear": [_P, _P, _d, _P, _d, _P, _P, _P, _P],
    "dndsb_vr_set_boundary": [_P, _i, _I32, _D, _i, _d, _d],
    "dndsb_eval_set_bc": [_P, _i, _I32, _D],
    "dndsb_eval_set_wall_distance": [_P, _D],
    "dndsb_vr_iter_vjp": [_P, _P, _P, _P, _i, _P, _P, _P],
    "dndsb_vr_iter_jvp": [_P, _P, _P, _P, _P, _i, _P, _P],
    "dndsb_eval_rhs_vjp": [_P, _P, _P, _P, _P, _P, _P],
    "dndsb_eval_rhs_jvp": [_P, _P, _P, _P, _P, _P, _P],
    "dndsb_eval_wall_flux_vjp": [_P, _D, _P, _P, _P, _P, _P],
    "dndsb_vr_iter_vjp_coords": [_P, _P, _P, _P, _i, _P, _P],
    "dndsb_vr_iter_jvp_coords": [_P, _P, _P, _P, _i, _P, _P],
    "dndsb_eval_rhs_vjp_coords": [_P, _P, _P, _P, _P, _P],
    "dndsb_eval_rhs_jvp_coords": [_P, _P, _P, _P, _P, _P],
    "dndsb_eval_residual_vjp_coords": [_P, _P, _P, _P, _P, _P, _P],
    "dndsb_eval_get_array": [_P, ctypes.c_char_p, _D, _l, _I64],
    "dndsb_eval_set_delta_lambda": [_P, _P, _P],
    "dndsb_eval_evaluate_rhs_noalloc": [_P, _P, _P, _P, _P],
    "dndsb_krylov_ld": [_l],
    "dndsb_krylov_work_bytes": [],
    "dndsb_krylov_start": [_i, _l, _i, _P, _P, _P, _P, _P, _P],
    "dndsb_krylov_arnoldi": [_i, _l, _i, _i, _P, _P, _P, _P, _P, _P, _P],
    "dndsb_krylov_update": [_i, _l, _i, _P, _P, _P, _P, _P],
    "dndsb_last_error": [],
    "dndsb_version": [],
}
_RESTYPES = {"dndsb_last_error": ctypes.c_char_p, "dndsb_krylov_ld": ctypes.c_int64, "dndsb_krylov_work_bytes": ctypes.c_size_t}

_lib = None


def load(require_device=True):
    """Load libdndsb.so; raise if it is missing (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run dndsr_b200/build.py (nvcc, sm_100a)")
        L = ctypes.CDLL(LIB_PATH)
        for name, args in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = _RESTYPES.get(name, ctypes.c_int)
        _lib = L
    if require_device:
        import torch
        if not torch.cuda.is_available():
            raise RuntimeError("dndsr_b200 needs a CUDA device; there is no CPU path")
    return _lib


def call(name, *args):
    rc = getattr(load(), name)(*args)
    if rc != DNDSB_OK:
        raise DndsbError(rc, _lib.dndsb_last_error().decode())
    return rc


def dptr(a):
    return ctypes.cast(a.ctypes.data, _D) if isinstance(a, np.ndarray) else a
