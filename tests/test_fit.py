"""Fit statistics after the fold (ppm_batch_fit / ppm_profile_fit) against the
oracle's restatements of cal_chi2 (p_devarshi24st.py:43-49) and the Poisson
log-likelihood, on counts collected from the same batch.

Tolerance: 1e-10 relative (both sides FP64; only the summation order differs)."""
import math

import numpy as np
import pytest

import oracle
from gpu_ppm_b200 import _abi, synth


def test_cal_chi2_restatement_matches_reference_expression():
    """The restatement equals the reference's expression on strictly positive models."""
    rng = np.random.default_rng(0)
    model = rng.uniform(0.5, 50.0, size=(30, 16))
    data = rng.poisson(model).astype(float)
    fac = 1e6 / np.sum(model)
    ref = np.sum((data * fac - model * fac) ** 2 / (model * fac))
    assert oracle.cal_chi2(data, model) == pytest.approx(ref, rel=1e-14)
    # zero-model entries are left out (with zero data), -inf log-likelihood with data
    model[0, 0] = 0.0
    data[0, 0] = 0.0
    assert math.isfinite(oracle.cal_chi2(data, model))
    data[0, 0] = 3.0
    assert oracle.poisson_loglike(data, model) == float("-inf")


@pytest.mark.gpu
def test_batch_and_plain_fit_match_oracle_statistics():
    from gpu_ppm_b200.engine import Engine

    lens, nsx = synth.lensing("std"), synth.nsx("v171019", seed=0)
    e = Engine()
    e.load_lensing(lens)
    e.load_nsx(nsx)
    E = synth.energy_grid(300, 0.2, 12.0)
    g = e.add_energy_grid(E)
    r = e.add_response(g, synth.response(300, 1000, E, seed=0))
    plist, _ = synth.draw_prior(8, seed=5, lens_u=(0.3, 0.5), n_side=32, n_bins=16, energy_grid=g, response=r,
                                fold=_abi.FOLD_FP64)
    batch = e.batch(plist)
    batch.launch()
    _, counts, _ = batch.collect(want_counts=True)
    n_el = 300 * 16
    rng = np.random.default_rng(1)
    # observed data: Poisson draws around the brightest profile's counts (scaled to ~1e5 counts)
    totals = [counts[k * n_el:(k + 1) * n_el].sum() for k in range(len(plist))]
    k0 = int(np.argmax(totals))
    assert totals[k0] > 0
    m0 = counts[k0 * n_el:(k0 + 1) * n_el]
    obs = rng.poisson(m0 * (1e5 / m0.sum())).astype(float)
    oid = e.add_observed(r, 16, obs.reshape(300, 16))
    fits = batch.fit(oid)
    for k in range(len(plist)):
        m = counts[k * n_el:(k + 1) * n_el]
        assert fits[k]["model_total"] == pytest.approx(m.sum(), rel=1e-12)
        if m.sum() > 0:
            assert fits[k]["chi2"] == pytest.approx(oracle.cal_chi2(obs, m), rel=1e-10), k
        else:  # no model counts at all (spot never visible): no chi2
            assert math.isnan(fits[k]["chi2"]), k
        ll = oracle.poisson_loglike(obs, m)
        if math.isinf(ll):
            assert fits[k]["loglike"] == ll, k
        else:
            assert fits[k]["loglike"] == pytest.approx(ll, rel=1e-10), k
        assert fits[k]["n_zero_model"] == int(np.sum(m <= 0)), k
    # the plain form gives the same statistics up to the FP32 partial sums of the
    # flux, which a one-profile launch splits into finer ring tiles than a batch
    f0, info = e.profile_fit(plist[k0], oid)
    assert f0["chi2"] == pytest.approx(fits[k0]["chi2"], rel=1e-6)
    assert f0["loglike"] == pytest.approx(fits[k0]["loglike"], rel=1e-9)
    assert info.n_points > 0
    # a profile with another bin count is rejected
    p = synth.draw_prior(1, seed=6, lens_u=(0.3, 0.5), n_side=32, n_bins=32, energy_grid=g, response=r)[0][0]
    with pytest.raises(_abi.PpmError):
        e.profile_fit(p, oid)
    batch.close()
    e.close()
