"""Times the reference's OWN CUDA program (gpu/devarshi24st_gpu.cu, built unchanged
for sm_100a into oracle/_ref/ref_devarshi_gpu by oracle/Makefile) and the engine
on the same GPU, tables and scenarios, and prints one JSON line per scenario.

The reference program hard-codes its star (gpu/devarshi24st_gpu.cu:22-44: M = 1.4,
R_eq = 12 km, 300 Hz, inclination 2.391, 32 phase bins, logT = 6, D = 0.15 kpc), so
the scenarios are fixed-star ones: its four std stars at its own N_side
(:123-127, :520-524) and the two-spot ring/crescent at N_side 256, with 300
energies over 0.2-12 keV and a 300-channel response.

* reference: calc_one_star's own CUDA-event time of its kernel and cuBLAS fold
  (:452-483), read from its output; the first scenario is the program's warm-up.
* engine device: one plan + integrand + fold pass of a one-profile batch,
  CUDA events around each phase (ppm_batch_launch_timed).
* engine plain: the synchronous ppm_profile call, host wall clock, counts
  downloaded to the host.

Also reports the largest relative difference between the two programs' counts
(floor 1e-6 of the maximum; informative: the reference's GPU lookups do not
clamp where its CPU does, and the engine follows the CPU).  MEASUREMENT
INFRASTRUCTURE ONLY; runs on a GPU with the reference program prebuilt.

    python oracle/time_reference_gpu.py [--repeats 3]
    python oracle/time_reference_gpu.py --layout DIR [--only NAME]   # tables + scen.txt only (for a profiler)
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import re
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

PI = math.pi
# name, N_side, N_fine, N_pts, setting, theta1, phi1, angrad1, theta2, phi2, angrad2
SCENARIOS = [
    ("Ring_Eq", 173, 192, 2, "std", 0.5 * PI, -0.2, 0.5, 0.5 * PI, 0.0, 0.25),
    ("Ring_Polar", 1708, 192, 2, "std", PI - 0.001, -0.02, 0.05, PI - 0.001, 0.0, 0.025),
    ("Crescent_Eq", 128, 192, 2, "std", 1.0, -1.0, 1.4, 0.5, 0.0, 0.5 * PI - 0.001),
    ("Crescent_Polar", 189, 192, 2, "std", 1.15, -0.1, 1.3, 1.75, 0.0, 0.5 * PI - 0.001),
    ("Cfg2_Ring", 256, 192, 2, "std", 30 * PI / 180, 0.0, 0.3, 30 * PI / 180, 0.0, 0.1),
    ("Cfg2_Crescent", 256, 192, 2, "std", 120 * PI / 180, 0.0, 0.35, 120 * PI / 180 - 0.1, 0.0, 0.2),
]


def max_rel(a, ref, floor=1e-6):
    scale = np.abs(ref).max()
    if scale == 0:
        return float(np.abs(a).max())
    denom = np.where(np.abs(ref) >= floor * scale, np.abs(ref), scale)
    return float((np.abs(a - ref) / denom).max())


def write_layout(d, lens, nsx, E, rsp, lines):
    """The reference program's working directory: tables, NSX file, output/ and scen.txt."""
    lens.write_dir(os.path.join(d, "tables", "lensing", "std"))
    nsx.write_file(os.path.join(d, "ext", "model_data", "nsx_H_v200804.out"))
    synth_mod().write_ism_inst(os.path.join(d, "tables", "ism_inst", "std"), E, rsp)
    os.makedirs(os.path.join(d, "output"), exist_ok=True)
    path = os.path.join(d, "scen.txt")
    with open(path, "w") as f:
        for ln in lines:
            f.write(" ".join(repr(x) if isinstance(x, float) else str(x) for x in ln) + "\n")
    return path


def synth_mod():
    from gpu_ppm_b200 import synth

    return synth


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--repeats", type=int, default=3)
    ap.add_argument("--layout", help="only write the reference program's working directory here and exit")
    ap.add_argument("--only", help="scenario name for --layout")
    args = ap.parse_args()
    if args.layout:
        synth = synth_mod()
        E = synth.energy_grid(300, 0.2, 12.0)
        scen = [s for s in SCENARIOS if args.only in (None, s[0])]
        if not scen:
            raise SystemExit(f"unknown scenario {args.only}")
        write_layout(args.layout, synth.lensing("std"), synth.nsx("v200804", seed=0), E,
                     synth.response(300, 1000, E, seed=0), scen)
        return
    prog = os.path.join(ROOT, "oracle", "_ref", "ref_devarshi_gpu")
    if not os.path.exists(prog):
        raise SystemExit(f"{prog} is missing: build it with `make -C oracle ref` where the reference sources are")
    import torch

    from gpu_ppm_b200 import _abi, synth
    from gpu_ppm_b200.engine import Engine

    lens, nsx = synth.lensing("std"), synth.nsx("v200804", seed=0)
    E = synth.energy_grid(300, 0.2, 12.0)
    rsp = synth.response(300, 1000, E, seed=0)
    ref_ms, ref_counts = {}, {}
    with tempfile.TemporaryDirectory() as tmp:
        lines = [("Warmup",) + SCENARIOS[0][1:]] + [s for s in SCENARIOS for _ in range(args.repeats)]
        path = write_layout(tmp, lens, nsx, E, rsp, lines)
        p = subprocess.run([prog, path], cwd=tmp, capture_output=True, text=True, timeout=1200)
        if p.returncode != 0:
            raise SystemExit(f"reference program failed ({p.returncode}): {p.stderr[-2000:]}")
        times = [float(m) for m in re.findall(r"Time taken: ([0-9.eE+-]+) ms", p.stdout)]
        assert len(times) == len(lines), (len(times), len(lines))
        for (name, *_), t in zip(lines[1:], times[1:]):
            ref_ms.setdefault(name, []).append(t)
        for s in SCENARIOS:
            ref_counts[s[0]] = np.loadtxt(os.path.join(tmp, "output", f"{s[0]}_std_counts_gpu.txt"))

    eng = Engine(device=0)
    eng.load_lensing(lens)
    eng.load_nsx(nsx)
    g = eng.add_energy_grid(E)
    r = eng.add_response(g, rsp)
    stream = torch.cuda.Stream()
    for name, n_side, n_fine, n_pts, _set, t1, p1, a1, t2, p2, a2 in SCENARIOS:
        prm = synth.params(mass_msun=1.4, r_eq_km=12.0, spin_hz=300.0, inclination_rad=2.391, distance_kpc=0.15,
                           exposure_s=1e6, spots=[synth.spot(t1, p1, a1, t2, p2, a2, logT=6.0)],
                           atmosphere=_abi.ATM_NSX, interp=_abi.INTERP_2L2C_LE, n_side=n_side, n_bins=32,
                           n_gl=n_pts, n_fine=n_fine, energy_grid=g, response=r)
        batch = eng.batch([prm])
        ms3 = (ctypes.c_float * 3)()
        dev = []
        for k in range(args.repeats + 1):
            _abi.check(_abi.lib().ppm_batch_launch_timed(eng.h, batch.h, ctypes.c_void_p(stream.cuda_stream), ms3))
            if k:
                dev.append(float(sum(ms3)))
        batch.close()
        plain = []
        for k in range(args.repeats + 1):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            _, counts, info = eng.profile(prm, want_flux=False, want_counts=True)
            if k:
                plain.append(1000.0 * (time.perf_counter() - t0))
        ref = float(np.median(ref_ms[name]))
        print(json.dumps({
            "scenario": name, "n_side": n_side, "energies": len(E), "channels": rsp.shape[0], "bins": 32,
            "reference_gpu_ms": ref, "engine_device_ms": float(np.median(dev)), "engine_plain_ms": float(np.median(plain)),
            "speedup_device": ref / float(np.median(dev)), "speedup_plain": ref / float(np.median(plain)),
            "max_rel_diff_counts": max_rel(counts.reshape(ref_counts[name].shape), ref_counts[name]),
            "repeats": args.repeats, "visible_points": int(info.n_points),
        }), flush=True)
    eng.close()


if __name__ == "__main__":
    main()
