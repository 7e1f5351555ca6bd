"""FP64 oracle flux of the two full-size NSX configurations, for the GPU parity
tests that compare the engine with the oracle at the sizes those
configurations name (tests/test_config_sizes.py):

  config2   ring (0.1 / 0.3 rad, colatitude 30 deg) + crescent (0.35 / 0.2 rad,
            offset 0.1 rad, colatitude 120 deg); M = 1.6 Msun, R_eq = 12.5 km,
            400 Hz, i = 60 deg; N_side 256, 64 bins x 2 GL, 300 energies
            0.2-12 keV; NSX 2l2c_le on synth.nsx("v171019", seed=0);
            synth.lensing("std")
  config3   the same star and spots at N_side 512 and 128 bins

The oracle (oracle/ppm_oracle.c, the FP64 restatement of
cpu/devarshi24st_cpu.cpp:25-241, pinned to the reference's own CPU programs by
tests/test_oracle_golden.py) integrates each profile over ring windows on all
host threads; flux and counts are linear in the rings, so the windows sum to
the whole profile.  The file also keeps fingerprints of every input (tables,
energy grid, responses, parameters) so that the tests can check that they
rebuild the same inputs.  About a minute (config 2) and a few minutes
(config 3) on 8 cores:

    python tests/golden/make_config_golden.py
"""
from __future__ import annotations

import ctypes
import os
import sys
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from gpu_ppm_b200 import _abi, synth  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "config_sizes_oracle.npz")
INFO_FIELDS = ("n_active", "n_rings", "n_dropped_rings", "n_points", "n_clamped", "n_active_integrated")


def inputs():
    """The tables, energy grid, responses and the two parameter sets (energy grid 0, responses 0 / 1)."""
    lens, nsx = synth.lensing("std"), synth.nsx("v171019", seed=0)
    E = synth.energy_grid(300, 0.2, 12.0)
    rsp2 = synth.response(300, 1000, E, seed=0)
    rsp3 = synth.response(1500, 3000, E, seed=0)
    p2 = synth.config2_params(0, 0)
    p3 = synth.config3_params(0, 1)
    return lens, nsx, E, rsp2, rsp3, p2, p3


def fingerprint(lens, nsx, E, rsp2, rsp3, p2, p3):
    """Sums and sums of squares of every input array plus the parameter structs' bytes."""
    arrays = {"lens_ca": lens.ca, "lens_lf": lens.lf, "lens_cdt": lens.cdt, "nsx_log_I": nsx.log_I, "nsx_mu": nsx.mu,
              "E": E, "rsp2": rsp2, "rsp3": rsp3}
    fp = {}
    for k, a in arrays.items():
        a = np.asarray(a, dtype=np.float64).ravel()
        fp[k] = np.array([a.size, a.sum(), (a * a).sum()])
    fp["p2"] = np.frombuffer(ctypes.string_at(ctypes.addressof(p2), ctypes.sizeof(p2)), dtype=np.uint8).copy()
    fp["p3"] = np.frombuffer(ctypes.string_at(ctypes.addressof(p3), ctypes.sizeof(p3)), dtype=np.uint8).copy()
    return fp


def profile_by_windows(ora, p, E, n_threads, n_windows=96):
    """The oracle's profile summed over ring windows evaluated on a thread pool."""
    n_rings = 4 * p.n_side
    edges = np.linspace(0, n_rings, n_windows + 1).round().astype(int)
    windows = [(int(a), int(b)) for a, b in zip(edges[:-1], edges[1:]) if b > a]

    def one(w):
        return ora.profile_rings(p, E, w[0], w[1])

    flux = np.zeros((p.n_bins, len(E)))
    info = dict.fromkeys(INFO_FIELDS, 0)
    with ThreadPoolExecutor(n_threads) as ex:
        for f, inf in ex.map(one, windows):
            flux += f
            for k in INFO_FIELDS:
                info[k] += getattr(inf, k)
    return flux, info


def main():
    lens, nsx, E, rsp2, rsp3, p2, p3 = inputs()
    ora = oracle.Oracle(lens, nsx)
    n_threads = os.cpu_count() or 1
    out = {}
    for name, p in (("config2", p2), ("config3", p3)):
        t0 = time.time()
        flux, info = profile_by_windows(ora, p, E, n_threads)
        out[f"{name}_flux"] = flux
        out[f"{name}_info"] = np.array([info[k] for k in INFO_FIELDS], dtype=np.int64)
        print(f"{name}: N_side {p.n_side}, {p.n_bins} bins, {info['n_active']} active elements, "
              f"{info['n_points']} phase points, {time.time() - t0:.1f} s on {n_threads} threads", flush=True)
    for k, v in fingerprint(lens, nsx, E, rsp2, rsp3, p2, p3).items():
        out["fp_" + k] = v
    np.savez_compressed(OUT, **out)
    print(OUT)


if __name__ == "__main__":
    main()
