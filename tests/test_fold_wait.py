"""Failure path of the tensor-core fold's bounded waits: every mbarrier wait of
fold_tc_kernel has an iteration limit after which the kernel records the
failure in an error word, waits (again bounded) for its own work in flight,
releases its tensor memory and returns.  The failure-path setting
PPM_FOLD_TC_STALL_TEST=<polls> makes the kernel issue no bulk copy and no MMA,
so its first wait has nothing to wait for and runs out after that many polls.
The call must report PPM_E_TIMEOUT, and the next call — on the same engine
and context — must succeed with correct counts."""
import numpy as np
import pytest

from gpu_ppm_b200 import _abi, synth
from gpu_ppm_b200.engine import Engine
from tests.errors import max_rel

pytestmark = pytest.mark.gpu


def test_fold_wait_runs_out_then_next_call_succeeds(monkeypatch):
    lens, nsx = synth.lensing("std"), synth.nsx("v171019", seed=0)
    e = Engine()
    try:
        e.load_lensing(lens)
        e.load_nsx(nsx)
        E = synth.energy_grid(300, 0.2, 12.0)
        g = e.add_energy_grid(E)
        r = e.add_response(g, synth.response(300, 1000, E, seed=0))
        p = synth.config2_params(g, r, n_side=32, n_bins=16)
        p.fold = _abi.FOLD_FP64
        _, counts_ref, _ = e.profile(p)
        p.fold = _abi.FOLD_BF16X3
        monkeypatch.setenv("PPM_FOLD_TC_STALL_TEST", "64")
        with pytest.raises(_abi.PpmError) as exc:
            e.profile(p)
        assert exc.value.code == _abi.PPM_E_TIMEOUT
        flux = np.zeros((16, 300))
        with pytest.raises(_abi.PpmError) as exc:  # the fold-only entry point reports it too
            e.fold(r, flux, 1.0, _abi.FOLD_BF16X3)
        assert exc.value.code == _abi.PPM_E_TIMEOUT
        monkeypatch.delenv("PPM_FOLD_TC_STALL_TEST")
        _, counts, _ = e.profile(p)
        assert max_rel(counts, counts_ref) < 1e-4
    finally:
        e.close()
