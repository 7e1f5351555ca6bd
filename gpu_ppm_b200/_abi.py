"""ctypes mirror of include/ppm.h and the loader for the in-tree libppm_b200.so.

The shared library is built by gpu_ppm_b200/build.py (nvcc, sm_100a) into
gpu_ppm_b200/_build/.  Importing this module never falls back to anything:
if the library is missing, `lib()` raises.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int32, c_int64, c_uint64, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libppm_b200.so")

# status codes (include/ppm.h)
PPM_OK = 0
PPM_E_INVALID = 1
PPM_E_IO = 2
PPM_E_RANGE = 3
PPM_E_OOM = 4
PPM_E_TIMEOUT = 5
PPM_E_CUDA = 6
PPM_E_STATE = 7
STATUS_NAMES = {
    0: "PPM_OK", 1: "PPM_E_INVALID", 2: "PPM_E_IO", 3: "PPM_E_RANGE", 4: "PPM_E_OOM",
    5: "PPM_E_TIMEOUT", 6: "PPM_E_CUDA", 7: "PPM_E_STATE",
}

SPOT_HEALPIX, SPOT_POINT = 0, 1
ATM_NSX, ATM_BLACKBODY = 0, 1
INTERP_4C, INTERP_4C_SG, INTERP_4C_LE, INTERP_2L2C_LE, INTERP_4L = 0, 1, 2, 3, 4
BEAM_ISO, BEAM_SIN2, BEAM_COS2 = 0, 1, 2
PREC_FP32, PREC_FP64 = 0, 1
FOLD_BF16X3, FOLD_FP32, FOLD_FP64 = 0, 1, 2

DP = POINTER(c_double)


class LensingDesc(ctypes.Structure):
    _fields_ = [
        ("u_min", c_double), ("u_max", c_double), ("n_u", c_int32),
        ("cos_psi_min", c_double), ("cos_psi_max", c_double), ("n_cos_psi", c_int32),
        ("cos_alpha_min", c_double), ("cos_alpha_max", c_double), ("n_cos_alpha", c_int32),
        ("cos_alpha_of_u_cos_psi", DP), ("lf_of_u_cos_psi", DP), ("cdt_over_R_of_u_cos_alpha", DP),
    ]


class LensingSpec(ctypes.Structure):
    _fields_ = [
        ("u_min", c_double), ("u_max", c_double), ("n_u", c_int32),
        ("cos_psi_min", c_double), ("cos_psi_max", c_double), ("n_cos_psi", c_int32),
        ("cos_alpha_min", c_double), ("cos_alpha_max", c_double), ("n_cos_alpha", c_int32),
        ("n_threads", c_int32),
    ]


class NsxDesc(ctypes.Structure):
    _fields_ = [
        ("n_logT", c_int32), ("n_logg", c_int32), ("n_logEkT", c_int32), ("n_mu", c_int32),
        ("logT_min", c_double), ("logT_max", c_double),
        ("logg_min", c_double), ("logg_max", c_double),
        ("logEkT_min", c_double), ("logEkT_max", c_double),
        ("mu", DP), ("log_I_T3", DP),
    ]


class Spot(ctypes.Structure):
    _fields_ = [
        ("theta1", c_double), ("phi1", c_double), ("angrad1", c_double),
        ("theta2", c_double), ("phi2", c_double), ("angrad2", c_double),
        ("logT", c_double), ("kT_keV", c_double),
        ("kind", c_int32), ("reserved", c_int32),
    ]


class Params(ctypes.Structure):
    _fields_ = [
        ("mass_msun", c_double), ("r_eq_km", c_double), ("spin_hz", c_double),
        ("inclination_rad", c_double), ("distance_kpc", c_double), ("exposure_s", c_double),
        ("spots", Spot * 2),
        ("n_spots", c_int32), ("atmosphere", c_int32), ("interp", c_int32), ("beaming", c_int32),
        ("n_side", c_int32), ("n_bins", c_int32), ("n_gl", c_int32), ("n_fine", c_int32),
        ("energy_grid", c_int32), ("response", c_int32), ("precision", c_int32), ("fold", c_int32),
    ]


class ResultInfo(ctypes.Structure):
    _fields_ = [
        ("n_active", c_int64), ("n_rings", c_int64), ("n_dropped_rings", c_int64),
        ("n_points", c_int64), ("n_clamped", c_int64), ("n_active_integrated", c_int64),
        ("status", c_int32), ("reserved", c_int32),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


class ServeBatchTrace(ctypes.Structure):
    _fields_ = [
        ("t_admit", c_double), ("t_launched", c_double), ("t_finished", c_double), ("t_published", c_double),
        ("n_requests", c_int32), ("stream_slot", c_int32), ("staging_bytes", c_int64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Fit(ctypes.Structure):
    _fields_ = [("chi2", c_double), ("loglike", c_double), ("model_total", c_double), ("n_zero_model", c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class EngineConfig(ctypes.Structure):
    _fields_ = [
        ("device", c_int32), ("max_batch", c_int32), ("memory_budget", c_int64),
        ("autotune", c_int32), ("n_streams", c_int32),
    ]


# Every symbol include/ppm.h declares, with its ctypes signature.
SIGNATURES = {
    "ppm_engine_create": (c_int32, [POINTER(EngineConfig), POINTER(c_void_p)]),
    "ppm_engine_destroy": (None, [c_void_p]),
    "ppm_engine_load_lensing": (c_int32, [c_void_p, POINTER(LensingDesc)]),
    "ppm_engine_load_lensing_dir": (c_int32, [c_void_p, c_char_p]),
    "ppm_engine_load_nsx": (c_int32, [c_void_p, POINTER(NsxDesc)]),
    "ppm_engine_load_nsx_file": (c_int32, [c_void_p, c_char_p, POINTER(NsxDesc)]),
    "ppm_engine_add_energy_grid": (c_int32, [c_void_p, c_int32, DP, POINTER(c_int32)]),
    "ppm_engine_add_response": (c_int32, [c_void_p, c_int32, c_int32, DP, POINTER(c_int32)]),
    "ppm_engine_load_ism_inst_dir": (c_int32, [c_void_p, c_char_p, POINTER(c_int32), POINTER(c_int32)]),
    "ppm_profile": (c_int32, [c_void_p, POINTER(Params), DP, DP, POINTER(ResultInfo)]),
    "ppm_profile_batch": (c_int32, [c_void_p, c_int32, POINTER(Params), DP, DP, POINTER(ResultInfo)]),
    "ppm_batch_create": (c_int32, [c_void_p, c_int32, POINTER(Params), POINTER(c_void_p)]),
    "ppm_batch_launch": (c_int32, [c_void_p, c_void_p, c_void_p]),
    "ppm_batch_device_outputs": (c_int32, [c_void_p, POINTER(c_void_p), POINTER(c_int64), POINTER(c_void_p),
                                           POINTER(c_int64)]),
    "ppm_batch_collect": (c_int32, [c_void_p, c_void_p, DP, DP, POINTER(ResultInfo)]),
    "ppm_batch_destroy": (None, [c_void_p, c_void_p]),
    "ppm_batch_launch_timed": (c_int32, [c_void_p, c_void_p, c_void_p, POINTER(ctypes.c_float)]),
    "ppm_batch_kernel_count": (c_int32, [c_void_p, c_void_p, POINTER(c_int32)]),
    "ppm_profile_noalloc": (c_int32, [c_void_p, POINTER(Params), c_void_p, c_void_p, c_void_p]),
    "ppm_profile_noalloc_result": (c_int32, [c_void_p, c_void_p, POINTER(ResultInfo)]),
    "ppm_batch_create_rings": (c_int32, [c_void_p, c_int32, POINTER(Params), c_int32, c_int32, POINTER(c_void_p)]),
    "ppm_profile_rings": (c_int32, [c_void_p, POINTER(Params), c_int32, c_int32, DP, DP, POINTER(ResultInfo)]),
    "ppm_engine_add_observed": (c_int32, [c_void_p, c_int32, c_int32, DP, POINTER(c_int32)]),
    "ppm_batch_fit": (c_int32, [c_void_p, c_void_p, c_int32, POINTER(Fit), c_void_p]),
    "ppm_profile_fit": (c_int32, [c_void_p, POINTER(Params), c_int32, POINTER(Fit), POINTER(ResultInfo)]),
    "ppm_engine_autotune": (c_int32, [c_void_p, c_int32, POINTER(Params), c_char_p, c_int32]),
    "ppm_output_sizes": (c_int32, [c_void_p, POINTER(Params), POINTER(c_int64), POINTER(c_int64)]),
    "ppm_fold": (c_int32, [c_void_p, c_int32, c_int32, c_int32, c_int32, DP, DP, DP]),
    "ppm_fold_device": (c_int32, [c_void_p, c_int32, c_int32, c_int32, c_int32, DP, c_void_p, c_void_p, c_void_p]),
    "ppm_submit": (c_int32, [c_void_p, POINTER(Params), DP, DP, POINTER(c_uint64)]),
    "ppm_poll": (c_int32, [c_void_p, c_uint64, POINTER(c_int32)]),
    "ppm_wait": (c_int32, [c_void_p, c_uint64, c_int32, POINTER(ResultInfo)]),
    "ppm_ticket_latency_us": (c_int32, [c_void_p, c_uint64, POINTER(c_double)]),
    "ppm_ticket_release": (c_int32, [c_void_p, c_uint64]),
    "ppm_serve_trace": (c_int32, [c_void_p, c_void_p, c_int32, POINTER(c_int32)]),
    "ppm_lensing_generate": (c_int32, [POINTER(LensingSpec), DP, DP, DP]),
    "ppm_response_prepare": (c_int32, [c_int32, c_int32, DP, DP, DP, DP, DP, c_int32, DP, DP]),
    "ppm_ism_inst_prepare": (c_int32, [c_char_p, c_char_p, c_char_p, c_int32, c_int32, c_int32, c_int32, c_int32,
                                       c_char_p]),
    "ppm_write_counts": (c_int32, [c_char_p, c_int32, c_int32, DP, c_int32]),
    "ppm_write_row": (c_int32, [c_char_p, c_int32, DP, c_int32]),
    "ppm_last_error_string": (c_char_p, []),
    "ppm_version": (c_char_p, []),
}

_LIB = None


class PpmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS_NAMES.get(code, code)}: {msg}")
        self.code = code


def lib():
    """Loads gpu_ppm_b200/_build/libppm_b200.so (raises if it was not built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -c 'import __graft_entry__ as g; g.build()'` "
                "(there is no fallback implementation)")
        h = ctypes.CDLL(LIB_PATH)
        missing = []
        for name, (res, args) in SIGNATURES.items():
            try:
                f = getattr(h, name)
            except AttributeError:
                missing.append(name)
                continue
            f.restype = res
            f.argtypes = args
        h.missing_symbols = missing
        _LIB = h
    return _LIB


def check(code):
    if code != PPM_OK:
        msg = lib().ppm_last_error_string()
        raise PpmError(code, msg.decode() if msg else "")
    return code


def dptr(a):
    """Pointer to a C-contiguous float64 numpy array (or None)."""
    if a is None:
        return None
    assert a.dtype.name == "float64" and a.flags["C_CONTIGUOUS"], "need C-contiguous float64"
    return a.ctypes.data_as(DP)
