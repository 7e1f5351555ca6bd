"""Golden subset of the reference's own lensing tables: runs c_lensing.py
(fizban007/gpu_ppm, "std" setting, ~100 s) in a scratch directory and keeps
rows u[0,85,170,255] x every 16th cos psi / cos alpha column of the three
tables in tests/golden/lensing_std_subset.npz.

    python tests/golden/make_lensing_golden.py --ref <reference source tree>  (or set PPM_REFERENCE_DIR) [--from DIR]
"""
import argparse
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
ROWS = [0, 85, 170, 255]
COLS = slice(0, 512, 16)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("PPM_REFERENCE_DIR"), required="PPM_REFERENCE_DIR" not in os.environ,
                    help="reference source tree (default: $PPM_REFERENCE_DIR)")
    ap.add_argument("--from", dest="src", default=None, help="existing tables/lensing/std folder")
    a = ap.parse_args()
    with tempfile.TemporaryDirectory() as tmp:
        src = a.src
        if src is None:
            subprocess.run([sys.executable, os.path.join(a.ref, "c_lensing.py")], cwd=tmp, check=True,
                           stdout=subprocess.DEVNULL)
            src = os.path.join(tmp, "tables", "lensing", "std")
        out = {}
        for k in ("cos_alpha_of_u_cos_psi", "lf_of_u_cos_psi", "cdt_over_R_of_u_cos_alpha"):
            out[k] = np.loadtxt(os.path.join(src, k + ".txt"))[ROWS][:, COLS]
        np.savez_compressed(os.path.join(ROOT, "tests", "golden", "lensing_std_subset.npz"), rows=np.array(ROWS),
                            col_step=16, **out)


if __name__ == "__main__":
    main()
