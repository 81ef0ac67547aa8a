"""ctypes binding of the C ABI in include/dnsbox.h (libdnsbox_gpu.so).

The library is built in-tree (``dnsbox_b200/_lib/libdnsbox_gpu.so``); loading
fails loudly when it is missing -- there is no CPU path.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libdnsbox_gpu.so")

DNSBOX_OK = 0
ERRORS = {
    -1: "DNSBOX_ERR_ARG", -2: "DNSBOX_ERR_SIZE", -3: "DNSBOX_ERR_CUDA", -4: "DNSBOX_ERR_OOM",
    -5: "DNSBOX_ERR_NONFINITE", -6: "DNSBOX_ERR_TIMEOUT", -7: "DNSBOX_ERR_STATE",
    -8: "DNSBOX_ERR_UNSUPPORTED",
}


class DnsboxError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class Params(ctypes.Structure):
    """``dnsbox_params`` (parameters.f90:11-50 as a runtime struct)."""
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("precision", ctypes.c_int32), ("stepper", ctypes.c_int32), ("ab2_mode", ctypes.c_int32),
        ("bandlim", ctypes.c_int32), ("spherical", ctypes.c_int32), ("tstep_fix", ctypes.c_int32),
        ("hminone", ctypes.c_int32), ("spectrum_mode", ctypes.c_int32), ("adj_phat", ctypes.c_int32),
        ("device", ctypes.c_int32), ("nbatch", ctypes.c_int32), ("no_prune", ctypes.c_int32),
        ("implicit_max_iter", ctypes.c_int32),
        ("alpha_x", ctypes.c_double), ("alpha_y", ctypes.c_double), ("alpha_z", ctypes.c_double),
        ("nu", ctypes.c_double), ("Q", ctypes.c_double), ("kCutOff", ctypes.c_double),
        ("Pin", ctypes.c_double), ("Deltak", ctypes.c_double),
        ("courant_min", ctypes.c_double), ("courant_max", ctypes.c_double),
        ("dt_max", ctypes.c_double), ("dt", ctypes.c_double), ("implicit_c", ctypes.c_double),
        ("implicit_tol", ctypes.c_double), ("reserved_d", ctypes.c_double * 2),
    ]


class Diag(ctypes.Structure):
    """``dnsbox_diag``: the Ekin.dat quantities of one step (io.f90:651-658)."""
    _fields_ = [
        ("t", ctypes.c_double), ("dt", ctypes.c_double), ("ekin", ctypes.c_double),
        ("dissipation", ctypes.c_double), ("production_literal", ctypes.c_double),
        ("injected_power", ctypes.c_double), ("courant", ctypes.c_double),
        ("umax", ctypes.c_double * 3), ("eband", ctypes.c_double),
        ("nonfinite", ctypes.c_int32), ("step", ctypes.c_int32),
    ]


class Schedule(ctypes.Structure):
    """``dnsbox_schedule``: the right-hand side's kernel choices."""
    _fields_ = [
        ("tc_kernel", ctypes.c_int32 * 4), ("x_kernel", ctypes.c_int32), ("tuned", ctypes.c_int32),
        ("ms_default", ctypes.c_double), ("ms_tuned", ctypes.c_double),
    ]


NPASS = 8
PASS_NAMES = ["z_inv", "y_inv", "x_nl", "y_fwd", "z_fin", "small", "other", "z_fwd"]


class Profile(ctypes.Structure):
    """``dnsbox_profile``: per-pass event time and launch counts."""
    _fields_ = [("ms", ctypes.c_double * NPASS), ("launches", ctypes.c_int64 * NPASS),
                ("total_launches", ctypes.c_int64)]


# (name, argtypes) of every entry point declared in include/dnsbox.h
_VP = ctypes.c_void_p
_DP = ctypes.POINTER(ctypes.c_double)
SIGNATURES = {
    "dnsbox_default_params": (None, [ctypes.POINTER(Params)]),
    "dnsbox_create": (ctypes.c_int, [ctypes.POINTER(Params), ctypes.POINTER(_VP)]),
    "dnsbox_destroy": (ctypes.c_int, [_VP]),
    "dnsbox_set_stream": (ctypes.c_int, [_VP, _VP]),
    "dnsbox_last_error": (ctypes.c_char_p, []),
    "dnsbox_supported_size": (ctypes.c_int, [ctypes.c_int]),
    "dnsbox_abi_version": (ctypes.c_int, []),
    "dnsbox_field_bytes": (ctypes.c_int, [_VP, ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_size_t)]),
    "dnsbox_nspec": (ctypes.c_int, [_VP]),
    "dnsbox_set_dt": (ctypes.c_int, [_VP, ctypes.c_double]),
    "dnsbox_get_dt": (ctypes.c_int, [_VP, _DP]),
    "dnsbox_set_time": (ctypes.c_int, [_VP, ctypes.c_double]),
    "dnsbox_get_time": (ctypes.c_int, [_VP, _DP]),
    "dnsbox_reset_history": (ctypes.c_int, [_VP]),
    "dnsbox_rhs_nonlinear": (ctypes.c_int, [_VP, _VP, _VP, _DP]),
    "dnsbox_step": (ctypes.c_int, [_VP, _VP, ctypes.c_int, ctypes.POINTER(Diag)]),
    "dnsbox_project": (ctypes.c_int, [_VP, _VP]),
    "dnsbox_dealias": (ctypes.c_int, [_VP, _VP]),
    "dnsbox_spectrum": (ctypes.c_int, [_VP, _VP, _DP, _DP, _DP, _DP]),
    "dnsbox_kinetic": (ctypes.c_int, [_VP, _VP, _DP]),
    "dnsbox_dissipation": (ctypes.c_int, [_VP, _VP, _DP]),
    "dnsbox_courant": (ctypes.c_int, [_VP, _VP, ctypes.c_double, _DP, _DP]),
    "dnsbox_divergence": (ctypes.c_int, [_VP, _VP, _DP]),
    "dnsbox_eband": (ctypes.c_int, [_VP, _VP, _DP]),
    "dnsbox_r2c": (ctypes.c_int, [_VP, _VP, _VP]),
    "dnsbox_c2r": (ctypes.c_int, [_VP, _VP, _VP]),
    "dnsbox_c2r_noalloc": (ctypes.c_int, [ctypes.c_int] * 4 + [_VP, _VP, _VP]),
    "dnsbox_state_alloc": (ctypes.c_int, [_VP, ctypes.POINTER(_VP)]),
    "dnsbox_state_free": (ctypes.c_int, [_VP, _VP]),
    "dnsbox_upload_state": (ctypes.c_int, [_VP, _VP, _VP]),
    "dnsbox_download_state": (ctypes.c_int, [_VP, _VP, _VP]),
    "dnsbox_upload_physical": (ctypes.c_int, [_VP, _VP, _VP]),
    "dnsbox_download_physical": (ctypes.c_int, [_VP, _VP, _VP]),
    "dnsbox_rhs_adj": (ctypes.c_int, [_VP, _VP, _VP, _VP]),
    "dnsbox_rhs_nonlinear_vjp": (ctypes.c_int, [_VP, _VP, _VP, _VP]),
    "dnsbox_set_forcing": (ctypes.c_int, [_VP, _VP]),
    "dnsbox_residual": (ctypes.c_int, [_VP, _VP, _DP]),
    "dnsbox_residual_grad": (ctypes.c_int, [_VP, _VP, _VP, _DP]),
    "dnsbox_adjoint_descent": (ctypes.c_int, [_VP, _VP, ctypes.c_int, _DP, _DP]),
    "dnsbox_heun_step_vjp": (ctypes.c_int, [_VP, _VP, _VP, _VP]),
    "dnsbox_step_pruned": (ctypes.c_int, [_VP]),
    "dnsbox_implicit_iterations": (ctypes.c_int, [_VP]),
    "dnsbox_init_yoffe": (ctypes.c_int, [_VP, _VP, ctypes.c_uint64, _VP]),
    "dnsbox_init_beltrami": (ctypes.c_int, [_VP, ctypes.c_double, _VP]),
    "dnsbox_set_step_projection": (ctypes.c_int, [_VP, ctypes.c_int]),
    "dnsbox_heun_steps_vjp": (ctypes.c_int, [_VP, _VP, ctypes.c_int, ctypes.c_int, _VP, _VP, _VP]),
    "dnsbox_orbit_residual": (ctypes.c_int, [_VP, _VP, ctypes.c_int, ctypes.c_int, _VP, _DP]),
    "dnsbox_batch_size": (ctypes.c_int, [_VP]),
    "dnsbox_set_batch_nu": (ctypes.c_int, [_VP, _DP]),
    "dnsbox_diag_read": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.POINTER(Diag)]),
    "dnsbox_ensemble_create": (ctypes.c_int, [ctypes.POINTER(_VP), ctypes.POINTER(_VP), ctypes.c_int,
                                              ctypes.POINTER(_VP)]),
    "dnsbox_ensemble_run": (ctypes.c_int, [_VP, ctypes.c_int]),
    "dnsbox_ensemble_destroy": (ctypes.c_int, [_VP]),
    "dnsbox_ensemble_pruned": (ctypes.c_int, [_VP]),
    "dnsbox_profile_enable": (ctypes.c_int, [_VP, ctypes.c_int]),
    "dnsbox_sync": (ctypes.c_int, [_VP]),
    "dnsbox_get_schedule": (ctypes.c_int, [_VP, ctypes.POINTER(Schedule)]),
    "dnsbox_set_schedule": (ctypes.c_int, [_VP, ctypes.POINTER(Schedule)]),
    "dnsbox_autotune": (ctypes.c_int, [_VP, _VP, ctypes.c_int, ctypes.POINTER(Schedule)]),
    "dnsbox_profile_read": (ctypes.c_int, [_VP, ctypes.POINTER(Profile), ctypes.c_int]),
    "dnsbox_slab_create": (ctypes.c_int, [ctypes.c_int] * 7 + [ctypes.POINTER(_VP)]),
    "dnsbox_slab_destroy": (None, [_VP]),
    "dnsbox_slab_dims": (ctypes.c_int, [_VP] + [ctypes.POINTER(ctypes.c_int)] * 4 + [ctypes.POINTER(ctypes.c_size_t)]),
    "dnsbox_slab_ftran_local": (ctypes.c_int, [_VP, _VP, _VP, _VP]),
    "dnsbox_slab_ftran_finish": (ctypes.c_int, [_VP, _VP, _VP, _VP]),
    "dnsbox_slab_btran_local": (ctypes.c_int, [_VP, _VP, _VP, _VP]),
    "dnsbox_slab_btran_finish": (ctypes.c_int, [_VP, _VP, _VP, _VP]),
    "dnsbox_slab_rhs_setup": (ctypes.c_int, [_VP, _VP]),
    "dnsbox_slab_rhs_begin": (ctypes.c_int, [_VP, _VP, _VP, _VP, _VP]),
    "dnsbox_slab_rhs_middle": (ctypes.c_int, [_VP, _VP, _VP, _VP, _VP]),
    "dnsbox_slab_rhs_finish": (ctypes.c_int, [_VP, _VP, _VP, _VP, _VP, _VP]),
    "dnsbox_slab_heun_finish": (ctypes.c_int, [_VP, _VP, _VP, _VP, ctypes.c_int, ctypes.c_double, _VP, _VP, _VP]),
}

_lib = None


def load():
    """Load libdnsbox_gpu.so (raises if it is not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is not built; run `python -c 'import __graft_entry__ as g; g.build()'`")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(rc):
    if rc != DNSBOX_OK:
        msg = load().dnsbox_last_error()
        raise DnsboxError(rc, msg.decode() if msg else "")
    return rc
