"""ctypes binding of ``libzm_b200.so`` (declarations in ``include/zm_b200.h``).

The library is built in-tree (``python -m zhenmode_b200.build``); importing
this module never compiles anything.  A missing library is an error, not a
fallback: there is no CPU implementation of the step in the product.
"""
from __future__ import annotations

import ctypes
import os

LIB_NAME = "libzm_b200.so"
LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), LIB_NAME)

ZM_OK = 0
ZM_ERR_INVALID = 1
ZM_ERR_UNSUPPORTED = 2
ZM_ERR_CUDA = 3
ZM_ERR_TIMEOUT = 4
ZM_ERR_MONITOR = 5

KERNEL_CLASSES = ("nu_sub", "inner_lap", "lin_finish", "implicit", "fz", "madv", "dealias", "tracer_adv",
                  "tracer_rest", "pgf", "barotropic", "final", "closure", "projection")

_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)


class ZmGrid(ctypes.Structure):
    _fields_ = [("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
                ("dy", ctypes.c_double), ("dx_2d", _dp), ("cos_lat", _dp), ("f", _dp),
                ("z", _dp), ("dz", _dp), ("wet_mask", _dp), ("wet_mask_3d", _dp)]


class ZmParams(ctypes.Structure):
    _fields_ = [("dt", ctypes.c_double), ("dt_bt", ctypes.c_double),
                ("nu_h", ctypes.c_double), ("nu_v", ctypes.c_double), ("kappa_h", ctypes.c_double),
                ("kappa_v", ctypes.c_double), ("kappa_conv", ctypes.c_double), ("nu_bi", ctypes.c_double),
                ("kappa_bi", ctypes.c_double), ("T_ref", ctypes.c_double), ("S_ref", ctypes.c_double),
                ("r_bot", ctypes.c_double), ("lambda_bulk", ctypes.c_double),
                ("restore_coef_S", ctypes.c_double), ("ice_salt_flux", ctypes.c_double),
                ("ice_freeze_temp_c", ctypes.c_double),
                ("nu_nsub", ctypes.c_int32), ("polar_cap_rows", ctypes.c_int32),
                ("polar_cap_taper", ctypes.c_int32), ("limiter", ctypes.c_int32),
                ("localize_conv", ctypes.c_int32), ("conservative_kv", ctypes.c_int32),
                ("freeze_adv_vel", ctypes.c_int32), ("vertical_diffusion", ctypes.c_int32),
                ("bt_kernel", ctypes.c_int32), ("autotune", ctypes.c_int32),
                ("tau_x", _dp), ("tau_y", _dp), ("q_heat", _dp), ("t_atm", _dp), ("s_ref", _dp),
                ("coastal_restore_coef", _dp), ("coastal_restore_t", _dp),
                ("coastal_bulk_lambda", _dp), ("coastal_kappa_h", _dp), ("coastal_kappa_v", _dp),
                ("project_adv_vel", ctypes.c_int32), ("projection_niter", ctypes.c_int32),
                ("projection_preconditioner", ctypes.c_int32), ("projection_max_refinements", ctypes.c_int32),
                ("projection_rtol", ctypes.c_double),
                ("sponge_rate", _dp), ("T_clim", _dp), ("S_clim", _dp), ("eta_relax_mask", _dp),
                ("eta_relax_rate", ctypes.c_double)]


class ZmState(ctypes.Structure):
    _fields_ = [("u", ctypes.c_void_p), ("v", ctypes.c_void_p), ("T", ctypes.c_void_p),
                ("S", ctypes.c_void_p), ("eta", ctypes.c_void_p)]


EXPORTS = {
    "zm_create": (ctypes.c_int, [ctypes.POINTER(ZmGrid), ctypes.POINTER(ZmParams), ctypes.POINTER(ctypes.c_void_p)]),
    "zm_info": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32), ctypes.c_int32]),
    "zm_load_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ZmState)]),
    "zm_advance": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32]),
    "zm_store_state": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ZmState)]),
    "zm_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ZmState),
                               ctypes.POINTER(ZmState), ctypes.c_int32]),
    "zm_step_host": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ZmState),
                                    ctypes.POINTER(ZmState), ctypes.c_int32]),
    "zm_set_forcing": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p]),
    "zm_run_stage": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(ZmState),
                                    ctypes.POINTER(ZmState)]),
    "zm_profile": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_float),
                                  ctypes.POINTER(ctypes.c_int32), ctypes.c_int32]),
    "zm_barrier_probe": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                        ctypes.c_int32]),
    "zm_status": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)]),
    "zm_projection_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32), ctypes.c_int32]),
    "zm_ledger_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ZmState), ctypes.POINTER(ZmState),
                                      ctypes.POINTER(ctypes.c_double), ctypes.c_int32]),
    "zm_diagnostics": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ZmState), ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "zm_mlp_forward_bf16": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32] + [ctypes.c_void_p] * 8
                            + [ctypes.c_void_p]),
    "zm_mlp_pack_bf16": (ctypes.c_int, [ctypes.c_void_p] * 5),
    "zm_mlp_trainer_create": (ctypes.c_int, [ctypes.c_int32, ctypes.POINTER(ctypes.c_void_p)]),
    "zm_mlp_trainer_destroy": (None, [ctypes.c_void_p]),
    "zm_mlp_grad": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32] + [ctypes.c_void_p] * 3
                    + [ctypes.c_double, ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)]),
    "zm_mlp_train_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32] + [ctypes.c_void_p] * 3
                          + [ctypes.c_double] + [ctypes.c_void_p] * 3
                          + [ctypes.c_int32, ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                             ctypes.POINTER(ctypes.c_double)]),
    "zm_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32),
                                   ctypes.POINTER(ctypes.c_int32)]),
    "zm_set_forcing_seasonal": (ctypes.c_int, [ctypes.c_void_p] * 5 + [ctypes.c_double, ctypes.c_double]),
    "zm_set_closure": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float]),
    "zm_closure_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint32),
                                        ctypes.POINTER(ctypes.c_uint32)]),
    "zm_closure_kappa": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ZmState), ctypes.c_void_p]),
    "zm_closure_features": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ZmState),
                                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "zm_ensemble_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int32,
                                          ctypes.POINTER(ctypes.c_void_p)]),
    "zm_ensemble_advance": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                           ctypes.POINTER(ctypes.c_int32)]),
    "zm_ensemble_destroy": (None, [ctypes.c_void_p]),
    "zm_tracer_terms": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ZmState), ctypes.c_void_p]),
    "zm_budgets": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                  ctypes.c_double, ctypes.c_double, ctypes.POINTER(ctypes.c_double)]),
    "zm_classify_state_noalloc": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float, ctypes.c_float,
                                                 ctypes.c_int32,
                                                 ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_int32)]),
    "zm_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "zm_destroy": (None, [ctypes.c_void_p]),
}

_LIB = None


def load():
    """Load the in-tree library once; raise if it has not been built."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_NAME} is not built; run `python -m zhenmode_b200.build` "
                           "(the B200 step has no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (restype, argtypes) in EXPORTS.items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    _LIB = lib
    return lib


def dptr(array):
    """float64 C pointer of a contiguous NumPy array (None stays NULL)."""
    if array is None:
        return None
    return array.ctypes.data_as(_dp)
