"""Generates the golden vectors in tests/golden/reference_cpu.npz by running the
reference's OWN CPU programs (cpu/devarshi24st_cpu.cpp, cpu/os1_cpu.cpp,
cpu/t_interp.cpp from fizban007/gpu_ppm, compiled unchanged by oracle/Makefile
and driven by oracle/ref_harness.cpp) on seeded synthetic tables.

Run in a container that has the reference sources:
    python tests/golden/make_golden.py --ref <reference source tree>  (or set PPM_REFERENCE_DIR)

Inputs (all regenerated bit-identically by the tests from the same seeds):
  * tables/lensing/std      synth.lensing("std")               (c_lensing.py grid)
  * NSX file                synth.nsx("v200804", seed=0)       (shape the unmodified
                                                                 cpu/nsx.hpp:53 expects)
  * tables/ism_inst/std     40 log-spaced energies 0.3-8 keV, 24-channel synth.response
The reference programs hard-code their star (cpu/devarshi24st_cpu.cpp:48-59,
cpu/os1_cpu.cpp:30-36, cpu/t_interp.cpp:20-32); the scenarios below vary spots,
N_side, fine phases, GL points, beaming and NSX interpolator.
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

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from gpu_ppm_b200 import synth  # noqa: E402

OUT = os.path.join(ROOT, "tests", "golden", "reference_cpu.npz")

PI = math.pi
DEVARSHI = [
    # name N_side N_fine N_pts setting theta1 phi1 angrad1 theta2 phi2 angrad2
    # the four reference scenarios (cpu/devarshi24st_cpu.cpp:18-21) at reduced N_side
    ("Ring_Eq", 16, 192, 2, "std", 0.5 * PI, -0.2, 0.5, 0.5 * PI, 0.0, 0.25),
    ("Ring_Polar", 128, 192, 2, "std", PI - 0.001, -0.02, 0.05, PI - 0.001, 0.0, 0.025),
    ("Crescent_Eq", 12, 192, 2, "std", 1.0, -1.0, 1.4, 0.5, 0.0, 0.5 * PI - 0.001),
    ("Crescent_Polar", 16, 192, 2, "std", 1.15, -0.1, 1.3, 1.75, 0.0, 0.5 * PI - 0.001),
    # the config-2 spots on the reference star, and other GL / fine-phase counts
    ("Cfg2_Ring", 24, 192, 2, "std", 30 * PI / 180, 0.0, 0.3, 30 * PI / 180, 0.0, 0.1),
    ("Cfg2_Crescent", 24, 150, 3, "std", 120 * PI / 180, 0.0, 0.35, 120 * PI / 180 - 0.1, 0.0, 0.2),
    ("Disk_G1", 20, 96, 1, "std", 2.0, 0.4, 0.3, 0.0, 0.0, 0.0),
]
OS1 = [
    # cpu/os1_cpu.cpp:18-27: name nu theta_c obs_theta angular_radius beaming
    ("os1a", 600, 90, 90, 0.01, "i"), ("os1b", 600, 90, 90, 1.0, "i"), ("os1c", 200, 90, 90, 0.01, "i"),
    ("os1d", 1, 90, 90, 1.0, "i"), ("os1e", 600, 60, 30, 1.0, "i"), ("os1f", 600, 20, 80, 1.0, "i"),
    ("os1g", 600, 60, 30, 1.0, "c"), ("os1h", 600, 60, 30, 1.0, "s"), ("os1i", 600, 20, 80, 1.0, "c"),
    ("os1j", 600, 20, 80, 1.0, "s"),
]
TINTERP = [
    # cpu/t_interp.cpp:458-470: name N_fine N_pts obs_theta theta angrad interp_type
    (f"test{g}{k}", 1024, 2, ot, th, 0.01, k)
    for g, (ot, th) in ((1, (0.01, 1.983)), (2, (0.964, PI - 0.01)))
    for k in range(4)
]
ISM_E = (0.3, 8.0, 40)
ISM_CH, ISM_FINE = 24, 200
TINTERP_ROWS = slice(0, 256, 8)
TINTERP_COLS = slice(0, 1024, 8)


def ism_inst():
    e = synth.energy_grid(ISM_E[2], ISM_E[0], ISM_E[1])
    return e, synth.response(ISM_CH, ISM_FINE, e, seed=0)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("PPM_REFERENCE_DIR"), required="PPM_REFERENCE_DIR" not in os.environ,
                    help="reference source tree (default: $PPM_REFERENCE_DIR)")
    args = ap.parse_args()
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle"), "ref", f"REF={args.ref}"], check=True)
    bin_dir = os.path.join(ROOT, "oracle", "_ref")
    with tempfile.TemporaryDirectory() as tmp:
        t0 = time.time()
        synth.lensing("std").write_dir(os.path.join(tmp, "tables", "lensing", "std"))
        synth.nsx("v200804", seed=0).write_file(os.path.join(tmp, "ext", "model_data", "nsx_H_v200804.out"))
        e, rsp = ism_inst()
        synth.write_ism_inst(os.path.join(tmp, "tables", "ism_inst", "std"), e, rsp)
        os.makedirs(os.path.join(tmp, "output"))
        print(f"tables written in {time.time() - t0:.1f}s", flush=True)

        def run(prog, lines):
            path = os.path.join(tmp, prog + ".txt")
            with open(path, "w") as f:
                for ln in lines:
                    f.write(" ".join(repr(x) if isinstance(x, float) else str(x) for x in ln) + "\n")
            t = time.time()
            r = subprocess.run([os.path.join(bin_dir, prog), path], cwd=tmp, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(r.stderr[-2000:])
            print(prog, f"{time.time() - t:.1f}s", r.stderr.strip().splitlines()[-1], flush=True)

        run("ref_devarshi", DEVARSHI)
        run("ref_os1", [(n, float(nu), th * PI / 180, ot * PI / 180, float(ar), b) for n, nu, th, ot, ar, b in OS1])
        run("ref_tinterp", TINTERP)

        out = {}
        for s in DEVARSHI:
            out["devarshi/" + s[0]] = np.loadtxt(os.path.join(tmp, "output", f"{s[0]}_{s[4]}_counts_cpu.txt"))
        for s in OS1:
            out["os1/" + s[0]] = np.loadtxt(os.path.join(tmp, "output", f"{s[0]}_cpu.txt"))
        for s in TINTERP:
            full = np.loadtxt(os.path.join(tmp, "output", f"{s[0]}_flux.txt"))
            out["tinterp/" + s[0]] = full[TINTERP_ROWS, TINTERP_COLS]
        meta = dict(devarshi=DEVARSHI, os1=OS1, tinterp=TINTERP, ism_e=ISM_E, ism_ch=ISM_CH, ism_fine=ISM_FINE,
                    tinterp_rows=[0, 256, 8], tinterp_cols=[0, 1024, 8], nsx="v200804 seed 0", lensing="std",
                    generator="tests/golden/make_golden.py")
        np.savez_compressed(OUT, meta=json.dumps(meta), **out)
        print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()
