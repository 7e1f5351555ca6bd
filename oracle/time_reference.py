"""Calibrates the CPU baseline: times the reference's OWN CPU program
(cpu/devarshi24st_cpu.cpp, built unchanged with the reference's timing flags
into oracle/_ref/ref_devarshi_timed) against the FP64 restatement in
oracle/ppm_oracle.c (its timed build, one thread) on the same profiles and
tables, and prints both rates in integrand evaluations per second.

The reference program hard-codes its star (cpu/devarshi24st_cpu.cpp:48-59), so
it cannot evaluate the batching prior's varying stars; bench.py's reference arm
therefore times the restatement, and this ratio tells how far that stands for
the reference's own code.  TEST INFRASTRUCTURE ONLY; needs the reference
sources (the Makefile's REF) and runs on the host cores.

    python oracle/time_reference.py --ref <reference source tree>  (or set PPM_REFERENCE_DIR) [--n-side 96]
"""
from __future__ import annotations

import argparse
import json
import math
import os
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from gpu_ppm_b200 import _abi, synth  # noqa: E402

PI = math.pi


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("PPM_REFERENCE_DIR"), required="PPM_REFERENCE_DIR" not in os.environ,
                    help="reference source tree (default: $PPM_REFERENCE_DIR)")
    ap.add_argument("--n-side", type=int, default=96)
    args = ap.parse_args()
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={args.ref}"], check=True)
    prog = os.path.join(ROOT, "oracle", "_ref", "ref_devarshi_timed")
    N = args.n_side
    # the config-2 spots on the reference star (cpu/devarshi24st_cpu.cpp:48-59), 300 energies 0.2-12 keV
    scen = [("Cfg2_Ring", N, 192, 2, "std", 30 * PI / 180, 0.0, 0.3, 30 * PI / 180, 0.0, 0.1),
            ("Cfg2_Crescent", N, 192, 2, "std", 120 * PI / 180, 0.0, 0.35, 120 * PI / 180 - 0.1, 0.0, 0.2)]
    tiny = [("Tiny", 2, 192, 2, "std", 30 * PI / 180, 0.0, 0.3, 30 * PI / 180, 0.0, 0.1)]
    lens, nsx = synth.lensing("std"), synth.nsx("v200804", seed=0)
    E = synth.energy_grid(300, 0.2, 12.0)
    rsp = synth.response(300, 1000, E, seed=0)
    with tempfile.TemporaryDirectory() as tmp:
        lens.write_dir(os.path.join(tmp, "tables", "lensing", "std"))
        nsx.write_file(os.path.join(tmp, "ext", "model_data", "nsx_H_v200804.out"))
        synth.write_ism_inst(os.path.join(tmp, "tables", "ism_inst", "std"), E, rsp)
        os.makedirs(os.path.join(tmp, "output"))

        def run(lines):
            path = os.path.join(tmp, "scen.txt")
            with open(path, "w") as f:
                for ln in lines:
                    f.write(" ".join(repr(x) if isinstance(x, float) else str(x) for x in ln) + "\n")
            t = time.perf_counter()
            subprocess.run([prog, path], cwd=tmp, check=True, capture_output=True)
            return time.perf_counter() - t

        t_load = min(run(tiny) for _ in range(2))  # table loading and start-up
        t_ref = run(scen) - t_load

    ora = oracle.Oracle(lens, nsx, fast=True)
    plist = []
    for s in scen:
        name, n_side, n_fine, n_pts, _set, t1, p1, a1, t2, p2, a2 = s
        plist.append(synth.params(mass_msun=1.4, r_eq_km=12.0, spin_hz=300.0, inclination_rad=2.391,
                                  distance_kpc=0.15, exposure_s=1e6, spots=[synth.spot(t1, p1, a1, t2, p2, a2, logT=6.0)],
                                  atmosphere=_abi.ATM_NSX, interp=_abi.INTERP_2L2C_LE, n_side=n_side, n_bins=32,
                                  n_gl=n_pts, n_fine=n_fine, energy_grid=0, response=0))
    t = time.perf_counter()
    _, infos = ora.profile_batch(plist, E, n_threads=1)
    t_port = time.perf_counter() - t
    evals = sum(i.n_points for i in infos) * len(E)  # visible (element, phase node) pairs x energies
    out = {"n_side": N, "evaluations": evals, "reference_s": t_ref, "reference_evals_per_s": evals / t_ref,
           "restatement_s": t_port, "restatement_evals_per_s": evals / t_port, "restatement_over_reference": t_ref / t_port,
           "table_load_s": t_load}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
