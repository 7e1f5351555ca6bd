"""The engine's lensing-table generator against the reference's own
c_lensing.py output (golden subset, tests/golden/make_lensing_golden.py)."""
import os

import numpy as np

from gpu_ppm_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_std_tables_match_c_lensing():
    z = np.load(os.path.join(ROOT, "tests", "golden", "lensing_std_subset.npz"))
    t = synth.generate_lensing(0.3, 0.5, 256, 512)
    rows = z["rows"]
    step = int(z["col_step"])
    ca = t.ca[rows][:, ::step]
    lf = t.lf[rows][:, ::step]
    cdt = t.cdt[rows][:, ::step]
    # scipy.quad in the script stops at 1.49e-8; the lensing factor is a numerical gradient of it
    assert np.abs(ca - z["cos_alpha_of_u_cos_psi"]).max() < 1e-7
    assert np.abs(cdt - z["cdt_over_R_of_u_cos_alpha"]).max() < 1e-6
    assert (np.abs(lf - z["lf_of_u_cos_psi"]) / np.abs(z["lf_of_u_cos_psi"])).max() < 5e-5


def test_generator_rejects_undefined_turning_points():
    import pytest

    from gpu_ppm_b200._abi import PpmError

    with pytest.raises(PpmError):
        synth.generate_lensing(0.1, 0.6, 8, 16)
