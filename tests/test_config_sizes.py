"""The two full-size NSX configurations against the FP64 oracle, at the sizes
they name (oracle flux from tests/golden/make_config_golden.py):

  * config 2: N_side 256, 64 bins x 2 GL, 300 energies, 300-channel response;
    flux and counts of all three folds within 1e-4 relative of the oracle;
  * config 3 (precision): N_side 512, 128 bins, a 1500-channel response built
    from 3000 fine energies; each fold (FP64 SIMT, FP32 SIMT, BF16 hi/lo x 3 on
    the tensor cores) applied both to the engine's FP32 flux (ppm_profile) and
    to the oracle's FP64 flux (ppm_fold), against the oracle's FP64 fold of
    its own flux.  Max and median relative error per channel are printed for
    each; limits: FP64 fold of the oracle flux 1e-12, FP32 and BF16x3 folds
    1e-4, everything computed from the engine's flux 1e-4.

Error metric: tests/errors.py (relative, floor 1e-6 of the maximum)."""
import json
import os

import numpy as np
import pytest

import oracle
from gpu_ppm_b200 import _abi
from gpu_ppm_b200.engine import Engine
from tests.errors import max_rel, per_channel_summary
from tests.golden import make_config_golden as mcg

pytestmark = pytest.mark.gpu

TOL = 1e-4
FOLDS = {"fp64": _abi.FOLD_FP64, "fp32": _abi.FOLD_FP32, "bf16x3": _abi.FOLD_BF16X3}


@pytest.fixture(scope="module")
def setup():
    lens, nsx, E, rsp2, rsp3, p2, p3 = mcg.inputs()
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "config_sizes_oracle.npz"))
    fp = mcg.fingerprint(lens, nsx, E, rsp2, rsp3, p2, p3)
    for k, v in fp.items():  # the tests rebuild the inputs the oracle flux was computed from
        if k in ("p2", "p3"):
            assert np.array_equal(v, z["fp_" + k]), k
        else:
            assert np.allclose(v, z["fp_" + k], rtol=1e-12, atol=0), k
    e = Engine()
    e.load_lensing(lens)
    e.load_nsx(nsx)
    g = e.add_energy_grid(E)
    r2 = e.add_response(g, rsp2)
    r3 = e.add_response(g, rsp3)
    assert (g, r2, r3) == (0, 0, 1)
    yield e, z, E, rsp2, rsp3, p2, p3
    e.close()


def check_info(info, golden):
    """Active elements, integrated phase points, dropped rings and rings with active elements equal the oracle's."""
    want = dict(zip(mcg.INFO_FIELDS, (int(x) for x in golden)))
    for k in ("n_active", "n_points", "n_dropped_rings", "n_rings"):
        assert getattr(info, k) == want[k], (k, getattr(info, k), want[k])


def test_config2_full_size(setup):
    e, z, E, rsp2, _, p, _ = setup
    ref_flux = z["config2_flux"]
    ref_counts = oracle.fold(rsp2, ref_flux, p.exposure_s)
    for name, mode in FOLDS.items():
        p.fold = mode
        flux, counts, info = e.profile(p)
        check_info(info, z["config2_info"])
        assert max_rel(flux, ref_flux) < TOL, name
        assert max_rel(counts, ref_counts) < TOL, name
        print(f"config 2 {name}: flux {max_rel(flux, ref_flux):.2e}, counts {max_rel(counts, ref_counts):.2e}")


def test_config3_precision(setup):
    e, z, E, _, rsp3, _, p = setup
    ref_flux = z["config3_flux"]
    alpha = p.exposure_s / p.n_bins
    ref_counts = oracle.fold(rsp3, ref_flux, p.exposure_s)
    report = {}
    flux_err = None
    for name, mode in FOLDS.items():
        p.fold = mode
        flux, counts, info = e.profile(p)
        check_info(info, z["config3_info"])
        flux_err = max_rel(flux, ref_flux)
        assert flux_err < TOL
        on_oracle = e.fold(p.response, ref_flux, alpha, mode)
        report[name] = {"fold_of_oracle_flux": per_channel_summary(on_oracle, ref_counts),
                        "engine_counts": per_channel_summary(counts, ref_counts)}
    report["flux_max_rel"] = flux_err
    print("config 3 per-channel relative errors:\n" + json.dumps(report, indent=1))
    assert report["fp64"]["fold_of_oracle_flux"]["max_of_channel_max"] < 1e-12
    assert report["fp32"]["fold_of_oracle_flux"]["max_of_channel_max"] < TOL
    assert report["bf16x3"]["fold_of_oracle_flux"]["max_of_channel_max"] < TOL
    for name in FOLDS:
        assert report[name]["engine_counts"]["max_of_channel_max"] < TOL, name
