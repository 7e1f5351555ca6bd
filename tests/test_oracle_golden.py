"""Pins the FP64 oracle against golden vectors produced by the reference's own
CPU programs (tests/golden/make_golden.py)."""
import os

import numpy as np
import pytest

import oracle
from gpu_ppm_b200 import synth
from tests import golden_cases as gc


@pytest.fixture(scope="module")
def ora():
    return oracle.Oracle(synth.lensing("std"), synth.nsx("v200804", seed=0))


def rel_err(a, b, floor_frac=1e-6):
    """max |a-b| / |b| over entries with |b| >= floor_frac * max|b|, else normalised by max|b|."""
    b = np.asarray(b)
    scale = np.abs(b).max()
    big = np.abs(b) >= floor_frac * scale
    e = np.where(big, np.abs(a - b) / np.where(big, np.abs(b), 1.0), np.abs(a - b) / scale)
    return e.max()


def test_devarshi_counts(golden, ora):
    meta, z = golden
    e, rsp = gc.ism_inst(meta)
    for s in meta["devarshi"]:
        p = gc.devarshi_params(s)
        flux, info = ora.profile(p, e)
        counts = oracle.fold(rsp, flux, p.exposure_s)
        ref = z["devarshi/" + s[0]]
        # the reference writes 10 significant digits (cpu/devarshi24st_cpu.cpp:248)
        assert rel_err(counts, ref) < 2e-9, s[0]
        assert info.n_active > 0


def test_os1_lightcurves(golden, ora):
    meta, z = golden
    for s in meta["os1"]:
        p = gc.os1_params(s)
        flux, info = ora.profile(p, np.array([1.0]))
        ref = z["os1/" + s[0]]
        assert rel_err(flux[:, 0], ref) < 2e-9, s[0]


def test_tinterp_all_interpolators(golden, ora):
    meta, z = golden
    e = gc.tinterp_energies()
    r0, r1, rs = meta["tinterp_rows"]
    c0, c1, cs = meta["tinterp_cols"]
    for s in meta["tinterp"]:
        p = gc.tinterp_params(s)
        flux, _ = ora.profile(p, e)
        ref = z["tinterp/" + s[0]]
        assert rel_err(flux[r0:r1:rs, c0:c1:cs], ref) < 2e-9, s[0]


def test_config_size_fixture_inputs_rebuild():
    """The full-size configuration fixture (tests/golden/make_config_golden.py)
    was computed from the inputs this checkout rebuilds: same tables, grid,
    responses and parameter structs."""
    from tests.golden import make_config_golden as mcg

    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "config_sizes_oracle.npz"))
    fp = mcg.fingerprint(*mcg.inputs())
    for k, v in fp.items():
        if k in ("p2", "p3"):
            assert np.array_equal(v, z["fp_" + k]), k
        else:
            assert np.allclose(v, z["fp_" + k], rtol=1e-12, atol=0), k
    for name in ("config2", "config3"):
        flux = z[name + "_flux"]
        assert np.all(np.isfinite(flux)) and flux.max() > 0
