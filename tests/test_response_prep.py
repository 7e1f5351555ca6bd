"""Response preparation (ppm_response_prepare, ppm_ism_inst_prepare, ppm_run
ism_inst) against a restatement of c_ism_inst.py with scipy's CubicSpline, the
script's own dependency, on synthetic RMF / ARF / ISM files in the script's
input formats (the NICER files are not available).

Tolerance: 1e-12 of the largest entry (both sides FP64; the spline slopes come
from different tridiagonal solvers)."""
import ctypes
import os
import subprocess

import numpy as np
import pytest
from scipy.interpolate import CubicSpline

from gpu_ppm_b200 import _abi

BUILD = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "gpu_ppm_b200", "_build")


def spline_matrix(e_lo, e_hi, e_obs):
    """C[j][i] = integral over fine bin j of the spline through unit vector i (c_ism_inst.py:76-86)."""
    C = np.zeros((len(e_lo), len(e_obs)))
    for i in range(len(e_obs)):
        y = np.zeros(len(e_obs))
        y[i] = 1.0
        cs = CubicSpline(e_obs, y)
        for j in range(len(e_lo)):
            C[j, i] = cs.integrate(e_lo[j], e_hi[j])
    return C


def fine_bins(rng, n, lo=0.2, hi=12.0):
    edges = np.sort(np.concatenate(([lo, hi], rng.uniform(lo, hi, n - 1))))
    return edges[:-1], edges[1:]


@pytest.mark.parametrize("n_obs", [2, 3, 4, 7, 64])
def test_response_prepare_matches_scipy(n_obs):
    rng = np.random.default_rng(n_obs)
    n_ch, n_fine = 17, 120
    e_lo, e_hi = fine_bins(rng, n_fine)
    rmf = rng.uniform(0, 1, (n_ch, n_fine))
    area = rng.uniform(10, 300, n_fine)
    ism = rng.uniform(0.5, 1.0, n_fine)
    e_obs = np.geomspace(e_lo[0], e_hi[-1], n_obs)
    ref = (rmf * area * ism) @ spline_matrix(e_lo, e_hi, e_obs)
    out = np.zeros((n_ch, n_obs))
    _abi.check(_abi.lib().ppm_response_prepare(n_ch, n_fine, _abi.dptr(rmf), _abi.dptr(area), _abi.dptr(e_lo),
                                               _abi.dptr(e_hi), _abi.dptr(ism), n_obs, _abi.dptr(e_obs),
                                               _abi.dptr(out)))
    assert np.abs(out - ref).max() <= 1e-12 * np.abs(ref).max()
    # without the interstellar factor
    ref2 = (rmf * area) @ spline_matrix(e_lo, e_hi, e_obs)
    _abi.check(_abi.lib().ppm_response_prepare(n_ch, n_fine, _abi.dptr(rmf), _abi.dptr(area), _abi.dptr(e_lo),
                                               _abi.dptr(e_hi), None, n_obs, _abi.dptr(e_obs), _abi.dptr(out)))
    assert np.abs(out - ref2).max() <= 1e-12 * np.abs(ref2).max()


def test_response_prepare_rejects_bad_knots():
    e = np.array([1.0, 1.0, 2.0])
    x = np.ones(2)
    out = np.zeros(3)
    rc = _abi.lib().ppm_response_prepare(1, 2, _abi.dptr(x), _abi.dptr(x), _abi.dptr(x), _abi.dptr(x), None, 3,
                                         _abi.dptr(e), _abi.dptr(out))
    assert rc == _abi.PPM_E_INVALID


def write_inputs(tmp, rng, n_e=240, n_ch=60):
    """Synthetic RMF / ARF / ISM files in c_ism_inst.py's formats (3 header lines for RMF and ARF)."""
    edges = np.linspace(0.2, 12.0, n_e + 1)
    area = 150 + 100 * np.sin(edges[:-1])
    chan = np.linspace(0.2, 12.0, n_ch)
    rmf = np.exp(-0.5 * ((chan[None, :] - 0.5 * (edges[:-1] + edges[1:])[:, None]) / 0.3) ** 2)  # [E][CH]
    with open(tmp / "rmf.txt", "w") as f:
        f.write("# synthetic\n# ENERG CHAN\n# value\n")
        for ie in range(n_e):
            for ic in range(n_ch):
                f.write(f"{ie} {ic} {rmf[ie, ic]:.17g}\n")
    with open(tmp / "arf.txt", "w") as f:
        f.write("# synthetic\n# ENERG_LO ENERG_HI SPECRESP\n#\n")
        for ie in range(n_e):
            f.write(f"{edges[ie]:.17g} {edges[ie + 1]:.17g} {area[ie]:.17g}\n")
    ism_e = np.geomspace(0.1, 20.0, 50)
    with open(tmp / "ism.txt", "w") as f:
        for e in ism_e:
            f.write(f"{e:.17g} 0 {np.exp(-0.3 / e ** 2):.17g}\n")
    return n_e, n_ch


def script_restatement(tmp, i_e_min, i_e_max, i_ch_min, i_ch_max, n_obs, with_ism=True):
    """c_ism_inst.py:30-99 on the synthetic files."""
    arf = np.loadtxt(tmp / "arf.txt", skiprows=3)
    rmf = np.loadtxt(tmp / "rmf.txt", skiprows=3, usecols=-1)
    n_e = arf.shape[0]
    rmf = rmf.reshape((n_e, -1)).T
    rmf = rmf[i_ch_min:i_ch_max, i_e_min:i_e_max]
    arf = arf[i_e_min:i_e_max, :]
    e_lo, e_hi = arf[:, 0], arf[:, 1]
    e_mid = 0.5 * (e_lo + e_hi)
    e_edges = np.hstack((e_lo[0], e_hi))
    response = arf[:, 2] * rmf
    e_obs = np.geomspace(e_edges[0], e_edges[-1], n_obs)
    C = spline_matrix(e_lo, e_hi, e_obs)
    frac = np.ones(len(e_mid))
    if with_ism:
        ism = np.loadtxt(tmp / "ism.txt")
        frac = CubicSpline(ism[:, 0], ism[:, 2])(e_mid) ** 5
    ds = (response * frac) @ C
    ds[np.abs(ds) < 1e-300] = 0.0
    return e_obs, ds


def test_ism_inst_prepare_matches_script(tmp_path):
    rng = np.random.default_rng(3)
    write_inputs(tmp_path, rng)
    out = tmp_path / "out"
    out.mkdir()
    args = (10, 200, 5, 50, 48)
    _abi.check(_abi.lib().ppm_ism_inst_prepare(str(tmp_path / "rmf.txt").encode(), str(tmp_path / "arf.txt").encode(),
                                               str(tmp_path / "ism.txt").encode(), *args, str(out).encode()))
    e_obs, ds = script_restatement(tmp_path, *args)
    assert open(out / "num.txt").read().split() == [str(ds.shape[0]), str(ds.shape[1])]
    got_e = np.loadtxt(out / "E_obs.txt")
    got = np.loadtxt(out / "rsp.txt")
    assert np.allclose(got_e, e_obs, rtol=1e-14, atol=0)
    assert np.abs(got - ds).max() <= 1e-12 * np.abs(ds).max()
    # out-of-range trims are refused
    rc = _abi.lib().ppm_ism_inst_prepare(str(tmp_path / "rmf.txt").encode(), str(tmp_path / "arf.txt").encode(),
                                         None, 0, 999, 0, 10, 16, str(out).encode())
    assert rc == _abi.PPM_E_RANGE


def test_ppm_run_ism_inst(tmp_path):
    rng = np.random.default_rng(4)
    write_inputs(tmp_path, rng)
    out = tmp_path / "o"
    out.mkdir()
    subprocess.run([os.path.join(BUILD, "ppm_run"), "ism_inst", str(tmp_path / "rmf.txt"), str(tmp_path / "arf.txt"),
                    "-", "0", "240", "0", "60", "32", str(out)], check=True, timeout=120)
    e_obs, ds = script_restatement(tmp_path, 0, 240, 0, 60, 32, with_ism=False)
    got = np.loadtxt(out / "rsp.txt")
    assert np.abs(got - ds).max() <= 1e-12 * np.abs(ds).max()


@pytest.mark.gpu
def test_prepared_folder_drives_the_engine(tmp_path):
    """A folder written by ppm_ism_inst_prepare loads with
    ppm_engine_load_ism_inst_dir, and the engine's counts on it match the
    oracle's flux folded with the written response (1e-4, FP32 integrand)."""
    import oracle
    from gpu_ppm_b200 import synth
    from gpu_ppm_b200.engine import Engine
    from tests.errors import max_rel

    rng = np.random.default_rng(5)
    write_inputs(tmp_path, rng)
    out = tmp_path / "std"
    out.mkdir()
    _abi.check(_abi.lib().ppm_ism_inst_prepare(str(tmp_path / "rmf.txt").encode(), str(tmp_path / "arf.txt").encode(),
                                               str(tmp_path / "ism.txt").encode(), 0, 240, 0, 60, 64,
                                               str(out).encode()))
    lens, nsx = synth.lensing("std"), synth.nsx("v171019", seed=0)
    e = Engine()
    e.load_lensing(lens)
    e.load_nsx(nsx)
    g, r = e.load_ism_inst_dir(out)
    p = synth.config2_params(g, r, n_side=24, n_bins=16, fold=_abi.FOLD_FP64)
    flux, counts, _ = e.profile(p)
    E = np.loadtxt(out / "E_obs.txt")
    rsp = np.loadtxt(out / "rsp.txt")
    ref_flux, _ = oracle.Oracle(lens, nsx).profile(p, E)
    assert max_rel(counts, oracle.fold(rsp, ref_flux, p.exposure_s)) < 1e-4
    e.close()
