"""Python host layer over libppm_b200.so (include/ppm.h).

`Engine` owns one device's resident tables (lensing, NSX, energy grids,
responses) and runs profiles through the C ABI:

* `profile(p)`            plain form: one profile, one pass of the kernels
  (replaces calc_one_star, gpu/devarshi24st_gpu.cu:432-511);
* `profile_batch(ps)`     batched form: one persistent launch over all profiles;
* `submit / wait`         serving form (continuous batching).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from ._abi import check, dptr, lib


class Engine:
    def __init__(self, device=0, max_batch=65536, memory_budget=0, autotune=0, n_streams=3):
        cfg = _abi.EngineConfig(device, max_batch, memory_budget, autotune, n_streams)
        h = ctypes.c_void_p()
        check(lib().ppm_engine_create(ctypes.byref(cfg), ctypes.byref(h)))
        self._lib = lib()  # kept for close() at interpreter exit, when module globals are gone
        self.h = h
        self.grids = {}      # id -> energies
        self.responses = {}  # id -> (grid, n_ch)

    def close(self):
        if getattr(self, "h", None):
            self._lib.ppm_engine_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    # ---- tables
    def load_lensing(self, tables):
        d = tables.desc()
        check(lib().ppm_engine_load_lensing(self.h, ctypes.byref(d)))

    def load_lensing_dir(self, path):
        check(lib().ppm_engine_load_lensing_dir(self.h, str(path).encode()))

    def load_nsx(self, table):
        d = table.desc()
        check(lib().ppm_engine_load_nsx(self.h, ctypes.byref(d)))

    def load_nsx_file(self, path, axes):
        check(lib().ppm_engine_load_nsx_file(self.h, str(path).encode(), ctypes.byref(axes)))

    def add_energy_grid(self, energies):
        e = np.ascontiguousarray(energies, dtype=np.float64)
        gid = ctypes.c_int32()
        check(lib().ppm_engine_add_energy_grid(self.h, len(e), dptr(e), ctypes.byref(gid)))
        self.grids[gid.value] = e.copy()
        return gid.value

    def add_response(self, grid, rsp):
        r = np.ascontiguousarray(rsp, dtype=np.float64)
        rid = ctypes.c_int32()
        check(lib().ppm_engine_add_response(self.h, grid, r.shape[0], dptr(r), ctypes.byref(rid)))
        self.responses[rid.value] = (grid, r.shape[0])
        return rid.value

    def load_ism_inst_dir(self, path):
        g = ctypes.c_int32()
        r = ctypes.c_int32()
        check(lib().ppm_engine_load_ism_inst_dir(self.h, str(path).encode(), ctypes.byref(g), ctypes.byref(r)))
        e = np.loadtxt(f"{path}/E_obs.txt", ndmin=1)
        self.grids[g.value] = e
        n_ch = int(open(f"{path}/num.txt").read().split()[0])
        self.responses[r.value] = (g.value, n_ch)
        return g.value, r.value

    # ---- sizes
    def sizes(self, p):
        n_e = len(self.grids[p.energy_grid])
        n_ch = self.responses[p.response][1] if p.response >= 0 else 0
        return (p.n_bins, n_e), (n_ch, p.n_bins)

    # ---- profiles
    def profile(self, p, want_flux=True, want_counts=None):
        fs, cs = self.sizes(p)
        if want_counts is None:
            want_counts = p.response >= 0
        flux = np.zeros(fs) if want_flux else None
        counts = np.zeros(cs) if want_counts else None
        info = _abi.ResultInfo()
        check(lib().ppm_profile(self.h, ctypes.byref(p), dptr(flux), dptr(counts), ctypes.byref(info)))
        return flux, counts, info

    def fold(self, response, flux, alpha, mode):
        """The response fold alone (ppm_fold): flux [n_profiles][n_bins][n_e] or [n_bins][n_e], alpha per
        profile (exposure / n_bins in the plain form); returns counts [.., n_ch, n_bins]."""
        f = np.ascontiguousarray(flux, dtype=np.float64)
        one = f.ndim == 2
        if one:
            f = f[None]
        n_prof, n_bins, _ = f.shape
        a = np.ascontiguousarray(np.broadcast_to(np.asarray(alpha, dtype=np.float64), (n_prof,)))
        n_ch = self.responses[response][1]
        counts = np.zeros((n_prof, n_ch, n_bins))
        check(lib().ppm_fold(self.h, response, mode, n_prof, n_bins, dptr(a), dptr(f), dptr(counts)))
        return counts[0] if one else counts

    def add_observed(self, response, n_bins, counts):
        """Observed counts [n_ch][n_bins] for fit statistics (ppm_engine_add_observed)."""
        c = np.ascontiguousarray(counts, dtype=np.float64).ravel()
        oid = ctypes.c_int32()
        check(lib().ppm_engine_add_observed(self.h, response, n_bins, dptr(c), ctypes.byref(oid)))
        return oid.value

    def profile_fit(self, p, observed):
        """One profile's fit statistics only (ppm_profile_fit): (ppm_fit as dict, info)."""
        out = _abi.Fit()
        info = _abi.ResultInfo()
        check(lib().ppm_profile_fit(self.h, ctypes.byref(p), observed, ctypes.byref(out), ctypes.byref(info)))
        return out.as_dict(), info

    def profile_batch(self, plist, want_flux=True, want_counts=None):
        n = len(plist)
        arr = (_abi.Params * n)(*plist)
        fsz = [self.sizes(p) for p in plist]
        nf = sum(a[0] * a[1] for a, _ in fsz)
        nc = sum(b[0] * b[1] for _, b in fsz)
        if want_counts is None:
            want_counts = nc > 0
        flux = np.zeros(nf) if want_flux else None
        counts = np.zeros(max(nc, 1)) if want_counts else None
        infos = (_abi.ResultInfo * n)()
        check(lib().ppm_profile_batch(self.h, n, arr, dptr(flux), dptr(counts), infos))
        out_f, out_c = [], []
        of = oc = 0
        for (fa, ca) in fsz:
            if want_flux:
                out_f.append(flux[of:of + fa[0] * fa[1]].reshape(fa))
            if want_counts:
                out_c.append(counts[oc:oc + ca[0] * ca[1]].reshape(ca) if ca[0] else None)
            of += fa[0] * fa[1]
            oc += ca[0] * ca[1]
        return out_f, out_c, list(infos)

    def autotune(self, plist):
        """Times candidate integrand launch shapes on these profiles and keeps the fastest."""
        n = len(plist)
        arr = (_abi.Params * n)(*plist)
        buf = ctypes.create_string_buffer(8192)
        check(lib().ppm_engine_autotune(self.h, n, arr, buf, len(buf)))
        return buf.value.decode()

    def batch(self, plist, rings=None):
        """A device-resident batch: planned once, launched any number of times.
        rings=(begin, end) keeps only HEALPix rings begin <= i < end (ppm_batch_create_rings)."""
        return Batch(self, plist, rings)

    def profile_rings(self, p, ring_begin, ring_end, want_flux=True, want_counts=None):
        """One profile restricted to rings [ring_begin, ring_end) (ppm_profile_rings)."""
        fs, cs = self.sizes(p)
        if want_counts is None:
            want_counts = p.response >= 0
        flux = np.zeros(fs) if want_flux else None
        counts = np.zeros(cs) if want_counts else None
        info = _abi.ResultInfo()
        check(lib().ppm_profile_rings(self.h, ctypes.byref(p), ring_begin, ring_end, dptr(flux), dptr(counts),
                                      ctypes.byref(info)))
        return flux, counts, info

    # ---- serving
    def submit(self, p, flux, counts):
        t = ctypes.c_uint64()
        check(lib().ppm_submit(self.h, ctypes.byref(p), dptr(flux), dptr(counts), ctypes.byref(t)))
        return t.value

    def poll(self, ticket):
        d = ctypes.c_int32()
        check(lib().ppm_poll(self.h, ticket, ctypes.byref(d)))
        return bool(d.value)

    def wait(self, ticket, timeout_ms=-1):
        info = _abi.ResultInfo()
        check(lib().ppm_wait(self.h, ticket, timeout_ms, ctypes.byref(info)))
        return info

    def latency_us(self, ticket):
        v = ctypes.c_double()
        check(lib().ppm_ticket_latency_us(self.h, ticket, ctypes.byref(v)))
        return v.value

    def release(self, ticket):
        """Forgets a finished ticket (ppm_ticket_release)."""
        check(lib().ppm_ticket_release(self.h, ticket))

    def serve_trace(self, cap=4096):
        """The most recent served batches (ppm_serve_trace), oldest first, as dicts."""
        buf = (_abi.ServeBatchTrace * cap)()
        n = ctypes.c_int32()
        check(lib().ppm_serve_trace(self.h, buf, cap, ctypes.byref(n)))
        return [buf[i].as_dict() for i in range(n.value)]


class Batch:
    """Wraps ppm_batch: uploads/plans once; `launch(stream)` replays a CUDA graph
    of plan -> integrand -> fold; outputs stay on the device until `collect`."""

    def __init__(self, engine, plist, rings=None):
        self.engine = engine
        self.n = len(plist)
        self.params = (_abi.Params * self.n)(*plist)
        h = ctypes.c_void_p()
        if rings is None:
            check(lib().ppm_batch_create(engine.h, self.n, self.params, ctypes.byref(h)))
        else:
            check(lib().ppm_batch_create_rings(engine.h, self.n, self.params, int(rings[0]), int(rings[1]),
                                               ctypes.byref(h)))
        self._lib = lib()
        self.h = h
        f = ctypes.c_void_p()
        c = ctypes.c_void_p()
        nf = ctypes.c_int64()
        nc = ctypes.c_int64()
        check(lib().ppm_batch_device_outputs(self.h, ctypes.byref(f), ctypes.byref(nf), ctypes.byref(c),
                                             ctypes.byref(nc)))
        self.flux_ptr, self.n_flux, self.counts_ptr, self.n_counts = f.value, nf.value, c.value, nc.value

    def launch(self, stream=0):
        check(lib().ppm_batch_launch(self.engine.h, self.h, ctypes.c_void_p(stream)))

    def fit(self, observed, stream=0):
        """Fit statistics of every profile after the last launch (ppm_batch_fit): list of dicts."""
        out = (_abi.Fit * self.n)()
        check(lib().ppm_batch_fit(self.engine.h, self.h, observed, out, ctypes.c_void_p(stream)))
        return [f.as_dict() for f in out]

    def collect(self, want_flux=False, want_counts=True):
        flux = np.zeros(self.n_flux) if want_flux else None
        counts = np.zeros(max(self.n_counts, 1)) if want_counts else None
        infos = (_abi.ResultInfo * self.n)()
        check(lib().ppm_batch_collect(self.engine.h, self.h, dptr(flux), dptr(counts), infos))
        return flux, counts, list(infos)

    def close(self):
        if getattr(self, "h", None):
            self._lib.ppm_batch_destroy(self.engine.h, self.h)
            self.h = None

    def __del__(self):
        self.close()
