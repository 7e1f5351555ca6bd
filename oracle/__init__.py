"""ctypes binding of the FP64 oracle (oracle/ppm_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker.  The engine package never
imports it.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from gpu_ppm_b200 import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF = os.path.join(HERE, "_ref")

_LIBS = {}


def build(ref=False):
    """Builds the oracle (and, when the reference sources exist, the reference harness)."""
    targets = ["oracle"] + (["ref"] if ref else [])  # "ref" needs PPM_REFERENCE_DIR
    subprocess.run(["make", "-s", "-C", HERE] + targets, check=True)


def _load(fast=False):
    name = "libppm_oracle_fast.so" if fast else "libppm_oracle.so"
    if name not in _LIBS:
        path = os.path.join(BUILD, name)
        if not os.path.exists(path):
            build()
        L = ctypes.CDLL(path)
        L.oracle_create.restype = ctypes.c_void_p
        L.oracle_create.argtypes = [ctypes.POINTER(_abi.LensingDesc), ctypes.POINTER(_abi.NsxDesc)]
        L.oracle_destroy.argtypes = [ctypes.c_void_p]
        L.oracle_profile.restype = ctypes.c_int
        L.oracle_profile.argtypes = [ctypes.c_void_p, ctypes.POINTER(_abi.Params), ctypes.c_int, _abi.DP, _abi.DP,
                                     ctypes.POINTER(_abi.ResultInfo)]
        L.oracle_profile_rings.restype = ctypes.c_int
        L.oracle_profile_rings.argtypes = [ctypes.c_void_p, ctypes.POINTER(_abi.Params), ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, _abi.DP, _abi.DP, ctypes.POINTER(_abi.ResultInfo)]
        L.oracle_profile_batch.restype = ctypes.c_int
        L.oracle_profile_batch.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(_abi.Params), ctypes.c_int,
                                           _abi.DP, _abi.DP, ctypes.POINTER(_abi.ResultInfo), ctypes.c_int]
        L.oracle_fold.restype = None
        L.oracle_fold.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _abi.DP, _abi.DP, ctypes.c_double, _abi.DP]
        L.oracle_interp.restype = ctypes.c_double
        L.oracle_interp.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                    ctypes.c_double]
        L.oracle_count_active.restype = ctypes.c_int64
        L.oracle_count_active.argtypes = [ctypes.POINTER(_abi.Spot), ctypes.c_int]
        _LIBS[name] = L
    return _LIBS[name]


class Oracle:
    """FP64 reference computation on fixed tables."""

    def __init__(self, lens, nsx=None, fast=False):
        self.L = _load(fast)
        self._ld = lens.desc()
        self._nd = nsx.desc() if nsx is not None else None
        self.ctx = self.L.oracle_create(ctypes.byref(self._ld), ctypes.byref(self._nd) if self._nd else None)
        if not self.ctx:
            raise RuntimeError("oracle_create failed")

    def __del__(self):
        if getattr(self, "ctx", None):
            self.L.oracle_destroy(self.ctx)
            self.ctx = None

    def profile(self, p, e_obs):
        e = np.ascontiguousarray(e_obs, dtype=np.float64)
        flux = np.zeros((p.n_bins, len(e)))
        info = _abi.ResultInfo()
        rc = self.L.oracle_profile(self.ctx, ctypes.byref(p), len(e), _abi.dptr(e), _abi.dptr(flux), ctypes.byref(info))
        if rc != 0:
            raise RuntimeError(f"oracle_profile failed: {rc}")
        return flux, info

    def profile_rings(self, p, e_obs, ring_begin, ring_end):
        """The profile over HEALPix rings ring_begin <= i < ring_end only (point source: ring 0)."""
        e = np.ascontiguousarray(e_obs, dtype=np.float64)
        flux = np.zeros((p.n_bins, len(e)))
        info = _abi.ResultInfo()
        rc = self.L.oracle_profile_rings(self.ctx, ctypes.byref(p), ring_begin, ring_end, len(e), _abi.dptr(e),
                                         _abi.dptr(flux), ctypes.byref(info))
        if rc != 0:
            raise RuntimeError(f"oracle_profile_rings failed: {rc}")
        return flux, info

    def profile_batch(self, plist, e_obs, n_threads=1):
        e = np.ascontiguousarray(e_obs, dtype=np.float64)
        n = len(plist)
        arr = (_abi.Params * n)(*plist)
        flux = np.zeros((n, plist[0].n_bins, len(e)))
        infos = (_abi.ResultInfo * n)()
        self.L.oracle_profile_batch(self.ctx, n, arr, len(e), _abi.dptr(e), _abi.dptr(flux), infos, n_threads)
        return flux, list(infos)

    def interp(self, mode, logT, logg, logEkT, mu):
        return self.L.oracle_interp(self.ctx, mode, logT, logg, logEkT, mu)


def fold(rsp, flux, exposure):
    """counts[ch][b] = sum_E flux[b][E] rsp[ch][E] * exposure / n_bins (FP64)."""
    L = _load()
    rsp = np.ascontiguousarray(rsp, dtype=np.float64)
    flux = np.ascontiguousarray(flux, dtype=np.float64)
    n_ch, n_e = rsp.shape
    n_bins = flux.shape[0]
    counts = np.zeros((n_ch, n_bins))
    L.oracle_fold(n_ch, n_e, n_bins, _abi.dptr(rsp), _abi.dptr(flux), exposure, _abi.dptr(counts))
    return counts


def cal_chi2(data, model):
    """p_devarshi24st.py:43-49 (cal_chi2): both arrays scaled so the model sums to
    1e6, chi2 = sum (data_ - model_)^2 / model_.  Entries with model <= 0 are left
    out, as the engine's fit statistics document (numpy gives inf/nan there)."""
    data = np.asarray(data, dtype=np.float64).ravel()
    model = np.asarray(model, dtype=np.float64).ravel()
    fac = 1e6 / np.sum(model)
    keep = model > 0
    model_ = model[keep] * fac
    data_ = data[keep] * fac
    return float(np.sum((data_ - model_) ** 2 / model_))


def poisson_loglike(data, model):
    """sum(d ln m - m - lgamma(d + 1)); entries with m <= 0 add -m when d == 0 and
    give -inf otherwise."""
    from math import lgamma

    d = np.asarray(data, dtype=np.float64).ravel()
    m = np.asarray(model, dtype=np.float64).ravel()
    pos = m > 0
    if np.any(~pos & (d != 0)):
        return float("-inf")
    lg = sum(lgamma(x + 1.0) for x in d)
    return float(np.sum(d[pos] * np.log(m[pos]) - m[pos]) - np.sum(m[~pos]) - lg)


def count_active(spot_struct, n_side):
    return _load().oracle_count_active(ctypes.byref(spot_struct), n_side)
