"""ppm_profile_noalloc — the allocation-free plain form — against ppm_profile.

Callers such as a sampler that reserved all device memory for its own pool at
start-up, or a framework whose caching allocator owns the GPU, cannot let the
library call cudaMalloc mid-run.  For them ppm_profile_noalloc keeps its
working state in a fixed device array and writes only into buffers the caller
already owns.  This test (its own file, collected last) allocates the output
buffers itself, calls the entry point through the C ABI twice in a row with
different profiles, and checks each result against ppm_profile within the
tolerance the other parity tests use (1e-4 relative, floor 1e-6 of the max).
It also checks that an oversized profile is refused with PPM_E_RANGE.
"""
import ctypes

import numpy as np
import pytest

from gpu_ppm_b200 import _abi, synth
from gpu_ppm_b200.engine import Engine
from tests.errors import max_rel

pytestmark = pytest.mark.gpu

TOL = 1e-4


@pytest.fixture(scope="module")
def setup():
    import torch

    lens, nsx = synth.lensing("std"), synth.nsx("v171019", seed=0)
    e = Engine()
    e.load_lensing(lens)
    e.load_nsx(nsx)
    E = synth.energy_grid(300, 0.2, 12.0)
    g = e.add_energy_grid(E)
    r = e.add_response(g, synth.response(300, 1000, E, seed=0))
    yield torch, e, g, r, len(E)
    e.close()


def run_noalloc(torch, e, p, n_e, n_ch):
    flux_d = torch.empty(p.n_bins * n_e, dtype=torch.float64, device="cuda")
    counts_d = torch.empty(n_ch * p.n_bins, dtype=torch.float64, device="cuda")
    flux_d.fill_(123.0)  # the entry point must clear what it accumulates into
    stream = torch.cuda.current_stream().cuda_stream
    rc = _abi.lib().ppm_profile_noalloc(e.h, ctypes.byref(p), ctypes.c_void_p(flux_d.data_ptr()),
                                        ctypes.c_void_p(counts_d.data_ptr()), ctypes.c_void_p(stream))
    _abi.check(rc)
    torch.cuda.synchronize()
    return flux_d.cpu().numpy().reshape(p.n_bins, n_e), counts_d.cpu().numpy().reshape(n_ch, p.n_bins)


def test_noalloc_matches_plain_two_calls(setup):
    torch, e, g, r, n_e = setup
    first = synth.config2_params(g, r, n_side=48, n_bins=16)
    second, _ = synth.draw_prior(1, seed=11, lens_u=(0.3, 0.5), n_side=40, n_bins=24, energy_grid=g, response=r)
    for p in (first, second[0]):
        p.fold = _abi.FOLD_FP64
        flux_ref, counts_ref, _ = e.profile(p)
        flux, counts = run_noalloc(torch, e, p, n_e, 300)
        assert max_rel(flux, flux_ref) < TOL
        assert max_rel(counts, counts_ref) < TOL


def test_noalloc_rejects_oversized_profile(setup):
    torch, e, g, r, n_e = setup
    p = synth.config2_params(g, r, n_side=4096, n_bins=16)
    flux_d = torch.empty(16 * n_e, dtype=torch.float64, device="cuda")
    rc = _abi.lib().ppm_profile_noalloc(e.h, ctypes.byref(p), ctypes.c_void_p(flux_d.data_ptr()), None, None)
    assert rc == _abi.PPM_E_RANGE
    assert b"scratch" in _abi.lib().ppm_last_error_string()
