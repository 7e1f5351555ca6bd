"""ppm_profile_noalloc — the allocation-free plain form — against ppm_profile
and the FP64 oracle.

Callers such as a sampler that reserved all device memory for its own pool at
start-up, or a framework whose caching allocator owns the GPU, cannot let the
library call cudaMalloc mid-run.  For them ppm_profile_noalloc keeps its
working state in a fixed device array and writes only into buffers the caller
already owns.  This test (its own file, collected last) allocates the output
buffers itself and calls the entry point through the C ABI twice in a row
with different profiles, for each of
  * the NSX FP32 integrand with the FP64 fold and with the BF16x3 tensor-core fold
    (300 energies, and 128 energies: the two-slot home-cell kernel),
  * the blackbody integrand in FP32 and in FP64 (flux only),
and checks each result against ppm_profile (flux within 1e-12 relative, floor
1e-6 of the max: the same tiles and partial sums, added to the flux in another
order; counts within the fold's tolerance, 1e-4) and against the oracle at the
parity tests' tolerances (1e-4 FP32, 1e-6 FP64 blackbody).  It also checks that the calls leave the device's free memory
unchanged, that ppm_profile_noalloc_result reports the call's counters, that
a bounded wait of the fold that runs out is reported by
ppm_profile_noalloc_result and by no other call, and that an oversized profile
is refused with PPM_E_RANGE.
"""
import ctypes

import numpy as np
import pytest

import oracle
from gpu_ppm_b200 import _abi, synth
from gpu_ppm_b200.engine import Engine
from tests.errors import max_rel

pytestmark = pytest.mark.gpu

TOL32 = 1e-4
TOL64 = 1e-6


@pytest.fixture(scope="module")
def setup():
    import torch

    lens, nsx = synth.lensing("std"), synth.nsx("v171019", seed=0)
    e = Engine()
    e.load_lensing(lens)
    e.load_nsx(nsx)
    E = synth.energy_grid(300, 0.2, 12.0)
    g = e.add_energy_grid(E)
    rsp = synth.response(300, 1000, E, seed=0)
    r = e.add_response(g, rsp)
    E_bb = synth.energy_grid(64, 0.2, 10.0)
    g_bb = e.add_energy_grid(E_bb)
    E128 = synth.energy_grid(128, 0.2, 12.0)
    g128 = e.add_energy_grid(E128)
    rsp128 = synth.response(300, 1000, E128, seed=0)
    r128 = e.add_response(g128, rsp128)
    env = {"torch": torch, "e": e, "g": g, "r": r, "E": E, "rsp": rsp, "E_bb": E_bb, "g_bb": g_bb,
           "E128": E128, "g128": g128, "r128": r128, "rsp128": rsp128, "ora": oracle.Oracle(lens, nsx)}
    yield env
    e.close()


def run_noalloc(torch, e, p, n_e, n_ch, flux_d, counts_d):
    flux_d.fill_(123.0)  # the entry point must clear what it accumulates into
    stream = torch.cuda.current_stream().cuda_stream
    rc = _abi.lib().ppm_profile_noalloc(e.h, ctypes.byref(p), ctypes.c_void_p(flux_d.data_ptr()),
                                        ctypes.c_void_p(counts_d.data_ptr()) if counts_d is not None else None,
                                        ctypes.c_void_p(stream))
    _abi.check(rc)
    info = _abi.ResultInfo()
    _abi.check(_abi.lib().ppm_profile_noalloc_result(e.h, ctypes.c_void_p(stream), ctypes.byref(info)))
    flux = flux_d.cpu().numpy().reshape(p.n_bins, n_e)
    counts = counts_d.cpu().numpy().reshape(n_ch, p.n_bins) if counts_d is not None else None
    return flux, counts, info


def nsx_cases(env, grid="g", resp="r"):
    first = synth.config2_params(env[grid], env[resp], n_side=48, n_bins=16)
    second, _ = synth.draw_prior(1, seed=11, lens_u=(0.3, 0.5), n_side=40, n_bins=24, energy_grid=env[grid],
                                 response=env[resp])
    return [first, second[0]]


def bb_cases(env, precision):
    first = synth.config1_params(env["g_bb"])
    second = synth.config1_params(env["g_bb"])
    second.n_side, second.n_bins, second.inclination_rad = 40, 24, 1.1
    second.spots[0].kT_keV = 0.45
    for p in (first, second):
        p.precision = precision
    return [first, second]


CASES = [("nsx_fold_fp64", _abi.FOLD_FP64), ("nsx_fold_bf16x3", _abi.FOLD_BF16X3),
         ("nsx128_fold_bf16x3", _abi.FOLD_BF16X3), ("blackbody_fp32", _abi.PREC_FP32),
         ("blackbody_fp64", _abi.PREC_FP64)]


@pytest.mark.parametrize("case,mode", CASES, ids=[c[0] for c in CASES])
def test_noalloc_matches_plain_and_oracle_two_calls(setup, case, mode):
    env = setup
    torch, e = env["torch"], env["e"]
    nsx = case.startswith("nsx")
    if nsx:
        e128 = case.startswith("nsx128")  # at most two energies per NSX cell: the two-slot kernel
        plist = nsx_cases(env, "g128", "r128") if e128 else nsx_cases(env)
        for p in plist:
            p.fold = mode
        E, n_ch, tol = (env["E128"] if e128 else env["E"]), 300, TOL32
        rsp = env["rsp128"] if e128 else env["rsp"]
    else:
        plist = bb_cases(env, mode)
        E, n_ch, tol = env["E_bb"], 0, (TOL64 if mode == _abi.PREC_FP64 else TOL32)
    n_e = len(E)
    refs = []
    for p in plist:  # reference results first: ppm_profile allocates, the noalloc calls below must not
        flux_ref, counts_ref, info_ref = e.profile(p)
        ora_flux, oinfo = env["ora"].profile(p, E)
        refs.append((flux_ref, counts_ref, info_ref, ora_flux, oinfo))
    size_f = max(p.n_bins * n_e for p in plist)
    size_c = max(p.n_bins * n_ch for p in plist)
    bufs = [(torch.empty(p.n_bins * n_e, dtype=torch.float64, device="cuda"),
             torch.empty(p.n_bins * n_ch, dtype=torch.float64, device="cuda") if nsx else None) for p in plist]
    assert size_f > 0 and (size_c > 0) == nsx
    for p, (fd, cd) in zip(plist, bufs):  # first use loads the kernels of this case
        run_noalloc(torch, e, p, n_e, n_ch, fd, cd)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for p, (fd, cd), (flux_ref, counts_ref, info_ref, ora_flux, oinfo) in zip(plist, bufs, refs):
        flux, counts, info = run_noalloc(torch, e, p, n_e, n_ch, fd, cd)
        # the same tiles and partial sums as ppm_profile; only the order of the flux pool's
        # (uncompensated, here) additions differs
        assert max_rel(flux, flux_ref) < 1e-12, case
        assert max_rel(flux, ora_flux) < tol, case
        assert info.n_active == info_ref.n_active == oinfo.n_active, case
        assert info.n_points == info_ref.n_points == oinfo.n_points, case
        assert info.n_clamped == info_ref.n_clamped, case
        if nsx:
            assert max_rel(counts, counts_ref) < tol, case
            assert max_rel(counts, oracle.fold(rsp, ora_flux, p.exposure_s)) < tol, case
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before, "ppm_profile_noalloc changed the device's free memory"


def test_noalloc_fold_wait_runs_out_is_its_own(setup, monkeypatch):
    """A bounded wait of the tensor-core fold that runs out (the failure-path
    test setting: no copy or MMA is issued) is reported for that call only."""
    env = setup
    torch, e = env["torch"], env["e"]
    p = nsx_cases(env)[0]
    p.fold = _abi.FOLD_BF16X3
    n_e = len(env["E"])
    fd = torch.empty(p.n_bins * n_e, dtype=torch.float64, device="cuda")
    cd = torch.empty(p.n_bins * 300, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    monkeypatch.setenv("PPM_FOLD_TC_STALL_TEST", "64")
    _abi.check(_abi.lib().ppm_profile_noalloc(e.h, ctypes.byref(p), ctypes.c_void_p(fd.data_ptr()),
                                              ctypes.c_void_p(cd.data_ptr()), ctypes.c_void_p(stream)))
    info = _abi.ResultInfo()
    rc = _abi.lib().ppm_profile_noalloc_result(e.h, ctypes.c_void_p(stream), ctypes.byref(info))
    assert rc == _abi.PPM_E_TIMEOUT and info.status == _abi.PPM_E_TIMEOUT
    monkeypatch.delenv("PPM_FOLD_TC_STALL_TEST")
    flux_ref, counts_ref, _ = e.profile(p)  # the engine's other calls do not see that status
    flux, counts, _ = run_noalloc(torch, e, p, n_e, 300, fd, cd)
    assert max_rel(counts, counts_ref) < TOL32


def test_noalloc_rejects_oversized_profile(setup):
    env = setup
    torch, e = env["torch"], env["e"]
    n_e = len(env["E"])
    p = synth.config2_params(env["g"], env["r"], n_side=4096, n_bins=16)
    flux_d = torch.empty(16 * n_e, dtype=torch.float64, device="cuda")
    rc = _abi.lib().ppm_profile_noalloc(e.h, ctypes.byref(p), ctypes.c_void_p(flux_d.data_ptr()), None, None)
    assert rc == _abi.PPM_E_RANGE
    assert b"scratch" in _abi.lib().ppm_last_error_string()
