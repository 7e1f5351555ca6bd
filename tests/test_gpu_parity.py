"""Engine (sm_100a kernels, through the C ABI) against the FP64 oracle and the
reference's own golden vectors.

Tolerances (tests/errors.py metric, floor 1e-6 of the max):
  * FP32 NSX integrand: 1e-4 relative per bin and per channel;
  * FP64 blackbody integrand: 1e-6 relative."""
import math

import numpy as np
import pytest

import oracle
from gpu_ppm_b200 import _abi, synth
from gpu_ppm_b200.engine import Engine
from tests import golden_cases as gc
from tests.errors import max_rel

pytestmark = pytest.mark.gpu

TOL32 = 1e-4
TOL64 = 1e-6


@pytest.fixture(scope="module")
def tables_v200804():
    return synth.lensing("std"), synth.nsx("v200804", seed=0)


@pytest.fixture(scope="module")
def eng_v200804(tables_v200804, golden):
    lens, nsx = tables_v200804
    meta, _ = golden
    e = Engine()
    e.load_lensing(lens)
    e.load_nsx(nsx)
    E, rsp = gc.ism_inst(meta)
    g = e.add_energy_grid(E)
    r = e.add_response(g, rsp)
    e.ism = (g, r, E, rsp)
    e.g1 = e.add_energy_grid(np.array([1.0]))
    e.gti = e.add_energy_grid(gc.tinterp_energies())
    yield e
    e.close()


@pytest.fixture(scope="module")
def ora_v200804(tables_v200804):
    return oracle.Oracle(*tables_v200804)


def test_devarshi_scenarios(golden, eng_v200804, ora_v200804):
    meta, z = golden
    g, r, E, rsp = eng_v200804.ism
    for s in meta["devarshi"]:
        p = gc.devarshi_params(s, g, r)
        for fold in (_abi.FOLD_FP64, _abi.FOLD_FP32, _abi.FOLD_BF16X3):
            p.fold = fold
            flux, counts, info = eng_v200804.profile(p)
            ref_flux, oinfo = ora_v200804.profile(p, E)
            assert max_rel(flux, ref_flux) < TOL32, (s[0], fold)
            ref_counts = oracle.fold(rsp, ref_flux, p.exposure_s)
            assert max_rel(counts, ref_counts) < TOL32, (s[0], fold)
            assert max_rel(counts, z["devarshi/" + s[0]]) < TOL32, (s[0], fold)
            assert info.n_active == oinfo.n_active and info.n_points == oinfo.n_points, s[0]
            assert info.n_dropped_rings == oinfo.n_dropped_rings, s[0]


def test_os1_fp64_lightcurves(golden, eng_v200804, ora_v200804):
    meta, z = golden
    for s in meta["os1"]:
        p = gc.os1_params(s, eng_v200804.g1)
        flux, _, info = eng_v200804.profile(p)
        ref, oinfo = ora_v200804.profile(p, np.array([1.0]))
        assert max_rel(flux, ref) < TOL64, s[0]
        assert max_rel(flux[:, 0], z["os1/" + s[0]]) < TOL64, s[0]
        assert info.n_points == oinfo.n_points, s[0]


def test_all_interpolators(golden, eng_v200804, ora_v200804):
    meta, z = golden
    E = gc.tinterp_energies()
    r0, r1, rs = meta["tinterp_rows"]
    c0, c1, cs = meta["tinterp_cols"]
    for s in meta["tinterp"]:
        p = gc.tinterp_params(s, eng_v200804.gti)
        flux, _, _ = eng_v200804.profile(p)
        ref, _ = ora_v200804.profile(p, E)
        assert max_rel(flux, ref) < TOL32, s[0]
        assert max_rel(flux[r0:r1:rs, c0:c1:cs], z["tinterp/" + s[0]]) < TOL32, s[0]


def test_config1_blackbody_fp64():
    lens = synth.lensing("std")
    e = Engine()
    e.load_lensing(lens)
    E = synth.energy_grid(64, 0.2, 10.0)
    g = e.add_energy_grid(E)
    p = synth.config1_params(g)
    flux, _, info = e.profile(p)
    ref, oinfo = oracle.Oracle(lens).profile(p, E)
    assert info.n_active == oinfo.n_active > 700
    assert max_rel(flux, ref) < TOL64
    e.close()


def test_blackbody_pointwise_and_energy_paths(golden, eng_v200804, ora_v200804):
    """The blackbody kernel evaluates one phase point per thread when a grid has
    few energies (n_e * 4 <= threads) and walks compacted points per energy
    otherwise; both, in FP32 and FP64, against the oracle, alone and mixed in
    one batch (the path is chosen per tile)."""
    meta, _ = golden
    few = []
    for s in meta["os1"][:4]:
        for prec, tol in ((_abi.PREC_FP32, TOL32), (_abi.PREC_FP64, TOL64)):
            p = gc.os1_params(s, eng_v200804.g1)
            p.precision = prec
            flux, _, _ = eng_v200804.profile(p)
            ref, _ = ora_v200804.profile(p, np.array([1.0]))
            assert max_rel(flux, ref) < tol, (s[0], prec)
            few.append((p, ref))
    lens = synth.lensing("std")
    E = synth.energy_grid(300, 0.2, 10.0)
    e = Engine()
    e.load_lensing(lens)
    g300, g1 = e.add_energy_grid(E), e.add_energy_grid(np.array([1.0]))
    many = synth.config1_params(g300)
    flux, _, _ = e.profile(many)
    ref_many, _ = oracle.Oracle(lens).profile(many, E)
    assert max_rel(flux, ref_many) < TOL64
    p1 = few[1][0]
    p1.energy_grid = g1
    fb, _, _ = e.profile_batch([many, p1], want_flux=True, want_counts=False)
    assert max_rel(fb[0], ref_many) < TOL64
    assert max_rel(fb[1], few[1][1]) < TOL64
    e.close()


def test_fused_point_source_pass():
    """A batch whose spots are all point sources (one or two energies here,
    at most two flux additions per bin and energy) runs as one fused launch:
    each CTA clears, plans and integrates its profile.  It gives the bits and
    the counters of the planned pass (the same profile batched with a
    HEALPix spot), and matches the oracle; a point source hidden at phase 0
    is dropped and counted as the planner counts it."""
    lens = synth.lensing("std")
    e = Engine()
    e.load_lensing(lens)
    ora = oracle.Oracle(lens)
    E1, E2 = np.array([1.0]), np.array([0.8, 2.0])
    g1, g2 = e.add_energy_grid(E1), e.add_energy_grid(E2)
    cases = []
    for prec, tol in ((_abi.PREC_FP32, TOL32), (_abi.PREC_FP64, TOL64)):
        for g, E, n_gl, th, inc in ((g1, E1, 0, 90.0, 90.0), (g2, E2, 2, 60.0, 30.0), (g1, E1, 0, 178.0, 5.0)):
            p = synth.params(mass_msun=1.4, r_eq_km=12.0, spin_hz=600.0, inclination_rad=inc * math.pi / 180,
                             distance_kpc=0.2, spots=[synth.spot(th * math.pi / 180, 0.0, 0.01, kT_keV=0.35,
                                                                 kind=_abi.SPOT_POINT)],
                             atmosphere=_abi.ATM_BLACKBODY, n_side=64, n_bins=64, n_gl=n_gl, energy_grid=g,
                             precision=prec)
            cases.append((p, E, tol, th))
    for p, E, tol, th in cases:
        f_fused, _, info = e.profile(p, want_counts=False)
        q = synth.config1_params(p.energy_grid)
        q.precision = p.precision
        fb, _, infos = e.profile_batch([q, p], want_flux=True, want_counts=False)
        assert np.array_equal(np.asarray(f_fused).reshape(-1), np.asarray(fb[1]).reshape(-1)), th
        for k in ("n_active", "n_rings", "n_dropped_rings", "n_points", "n_clamped", "n_active_integrated"):
            assert getattr(info, k) == getattr(infos[1], k), (th, k)
        ref, oinfo = ora.profile(p, E)
        assert info.n_points == oinfo.n_points and info.n_dropped_rings == oinfo.n_dropped_rings, th
        if th > 170:
            assert info.n_dropped_rings == 1 and not np.asarray(f_fused).any()
        else:
            assert info.n_dropped_rings == 0 and max_rel(f_fused, ref) < tol, th
    e.close()


@pytest.fixture(scope="module")
def eng_v171019():
    lens, nsx = synth.lensing("std"), synth.nsx("v171019", seed=0)
    e = Engine()
    e.load_lensing(lens)
    e.load_nsx(nsx)
    E = synth.energy_grid(300, 0.2, 12.0)
    g = e.add_energy_grid(E)
    rsp = synth.response(300, 1000, E, seed=0)
    r = e.add_response(g, rsp)
    e.cfg2 = (g, r, E, rsp)
    e.ora = oracle.Oracle(lens, nsx)
    yield e
    e.close()


def test_config2_spots_small_nside(eng_v171019):
    g, r, E, rsp = eng_v171019.cfg2
    p = synth.config2_params(g, r, n_side=48, n_bins=16)
    ref_flux, oinfo = eng_v171019.ora.profile(p, E)
    ref_counts = oracle.fold(rsp, ref_flux, p.exposure_s)
    for fold in (_abi.FOLD_FP64, _abi.FOLD_FP32, _abi.FOLD_BF16X3):
        p.fold = fold
        flux, counts, info = eng_v171019.profile(p)
        assert info.n_active == oinfo.n_active and info.n_points == oinfo.n_points
        assert max_rel(flux, ref_flux) < TOL32
        assert max_rel(counts, ref_counts) < TOL32, fold


def test_batch_matches_plain(eng_v171019):
    g, r, E, rsp = eng_v171019.cfg2
    plist, _ = synth.draw_prior(12, seed=3, lens_u=(0.3, 0.5), n_side=32, n_bins=16, energy_grid=g, response=r)
    flux_b, counts_b, infos = eng_v171019.profile_batch(plist)
    for k, p in enumerate(plist):
        # the one-profile call splits the phase nodes over more tiles, but every
        # tile covers the same elements, a node's partial sums are formed in the
        # same order, and the flux pool's additions are compensated: the results
        # are the same bits
        f, c, info = eng_v171019.profile(p)
        assert np.array_equal(flux_b[k], f), (k, max_rel(flux_b[k], f))
        assert np.array_equal(counts_b[k], c), (k, max_rel(counts_b[k], c))
        assert infos[k].n_points == info.n_points
    # and against the oracle for a few
    for k in range(3):
        ref, _ = eng_v171019.ora.profile(plist[k], E)
        assert max_rel(flux_b[k], ref) < TOL32, k


def test_fold_precision_config3_shapes():
    """Config-3 response shape (1500 channels from a 3000-bin fine grid, 300
    energies, 128 bins): FP64 SIMT, FP32 SIMT and BF16x3 tensor-core folds of
    the same flux against the FP64 oracle fold."""
    lens, nsx = synth.lensing("std"), synth.nsx("v171019", seed=0)
    e = Engine()
    e.load_lensing(lens)
    e.load_nsx(nsx)
    E = synth.energy_grid(300, 0.2, 12.0)
    g = e.add_energy_grid(E)
    rsp = synth.response(1500, 3000, E, seed=0)
    r = e.add_response(g, rsp)
    p = synth.config3_params(g, r)
    p.n_side = 48
    errs = {}
    flux0 = None
    for fold in (_abi.FOLD_FP64, _abi.FOLD_FP32, _abi.FOLD_BF16X3):
        p.fold = fold
        flux, counts, _ = e.profile(p)
        if flux0 is None:
            flux0 = flux
        ref = oracle.fold(rsp, flux, p.exposure_s)
        errs[fold] = max_rel(counts, ref)
    assert errs[_abi.FOLD_FP64] < 1e-12
    assert errs[_abi.FOLD_FP32] < 1e-5
    assert errs[_abi.FOLD_BF16X3] < TOL32
    e.close()


def test_chunked_rings_and_small_batches(monkeypatch):
    """Rings split into many work tiles (32 candidate elements each) and small
    polynomial sub-batches give the oracle's result."""
    monkeypatch.setenv("PPM_CHUNK", "32")
    monkeypatch.setenv("PPM_PB", "10")
    lens, nsx = synth.lensing("std"), synth.nsx("v171019", seed=0)
    e = Engine()
    e.load_lensing(lens)
    e.load_nsx(nsx)
    E = synth.energy_grid(128, 0.2, 12.0)
    g = e.add_energy_grid(E)
    p = synth.config2_params(g, -1, n_side=40, n_bins=16)
    flux, _, info = e.profile(p, want_counts=False)
    ref, oinfo = oracle.Oracle(lens, nsx).profile(p, E)
    assert info.n_active == oinfo.n_active and info.n_points == oinfo.n_points
    assert max_rel(flux, ref) < TOL32
    e.close()


def test_node_splits_give_the_same_bits(monkeypatch):
    """The NSX home-cell kernel's tiles may split a ring chunk's phase nodes
    into any number of ranges (PPM_SPLITS forces 1, 3 or 16): every node's
    partial sums are formed the same way and the flux additions are
    compensated, so the flux and counts are the same bits; the blackbody
    kernel, which also sums in FP64, agrees to 1e-12."""
    lens, nsx = synth.lensing("std"), synth.nsx("v171019", seed=0)
    E = synth.energy_grid(300, 0.2, 12.0)
    rsp = synth.response(300, 1000, E, seed=0)
    E_bb = synth.energy_grid(3, 0.5, 4.0)
    out = {}
    for splits in ("1", "3", "16"):
        monkeypatch.setenv("PPM_SPLITS", splits)
        e = Engine()
        try:
            e.load_lensing(lens)
            e.load_nsx(nsx)
            g = e.add_energy_grid(E)
            r = e.add_response(g, rsp)
            g_bb = e.add_energy_grid(E_bb)
            plist, _ = synth.draw_prior(3, seed=7, lens_u=(0.3, 0.5), n_side=48, n_bins=32, energy_grid=g, response=r)
            bb = synth.config1_params(g_bb)
            bb.precision = _abi.PREC_FP32
            out[splits] = ([e.profile(p)[:2] for p in plist], e.profile(bb)[0])
        finally:
            e.close()
    for splits in ("3", "16"):
        for (f0, c0), (f1, c1) in zip(out["1"][0], out[splits][0]):
            assert np.array_equal(f0, f1), (splits, max_rel(f1, f0))
            assert np.array_equal(c0, c1), (splits, max_rel(c1, c0))
        assert max_rel(out[splits][1], out["1"][1]) < 1e-12, splits


def test_autotune_keeps_parity(eng_v171019):
    g, r, E, rsp = eng_v171019.cfg2
    plist, _ = synth.draw_prior(8, seed=21, lens_u=(0.3, 0.5), n_side=32, n_bins=16, energy_grid=g, response=r)
    report = eng_v171019.autotune(plist)
    assert "(chosen)" in report
    f, c, _ = eng_v171019.profile(plist[0])
    ref, _ = eng_v171019.ora.profile(plist[0], E)
    assert max_rel(f, ref) < TOL32


@pytest.mark.parametrize("kernel", ["0", "1"])
def test_table_edges_and_even_mu(monkeypatch, kernel):
    """Narrow logEkT axes put energies with large flux beyond the low end
    (0.6..1.4) or the high end (-0.3..0.5) of the table, where the edge value is
    held, and an even mu count exercises the padded slice rows; every
    interpolator, a log-spaced grid (home-cell kernel unless PPM_KERNEL=1) and a
    dense linear grid (pooled kernel), against the oracle."""
    monkeypatch.setenv("PPM_KERNEL", kernel)
    lens = synth.lensing("std")
    grids = (synth.energy_grid(200, 0.1, 20.0), np.linspace(0.1, 20.0, 700))
    for axis in ((0.6, 1.4), (-0.3, 0.5)):
        nsx = synth.nsx("v171019", seed=1, n_mu=66, dims={"n_logEkT": 41, "logEkT": axis})
        e = Engine()
        e.load_lensing(lens)
        e.load_nsx(nsx)
        ora = oracle.Oracle(lens, nsx)
        for E in grids:
            g = e.add_energy_grid(E)
            for interp in range(5):
                p = synth.config2_params(g, -1, n_side=24, n_bins=16)
                p.interp = interp
                flux, _, info = e.profile(p, want_counts=False)
                ref, oinfo = ora.profile(p, E)
                assert info.n_points == oinfo.n_points and info.n_clamped > 0
                assert max_rel(flux, ref) < TOL32, (axis, interp, len(E))
        e.close()


def test_ring_windows_sum_to_full_profile(monkeypatch):
    """ppm_profile_rings / ppm_batch_create_rings over a 3-way ring partition:
    each window matches the oracle on the same rings and the windows sum to the
    whole profile (FP64 fold, 1e-12, with one fixed tile size so that every
    call groups the FP32 partial sums alike); a point-source spot belongs to ring 0."""
    from gpu_ppm_b200 import dist as pdist

    monkeypatch.setenv("PPM_CHUNK", "64")
    monkeypatch.setenv("PPM_SMALL_CHUNK", "64")
    lens, nsx = synth.lensing("std"), synth.nsx("v171019", seed=0)
    eng = Engine()
    eng.load_lensing(lens)
    eng.load_nsx(nsx)
    E = synth.energy_grid(300, 0.2, 12.0)
    g = eng.add_energy_grid(E)
    rsp = synth.response(300, 1000, E, seed=0)
    r = eng.add_response(g, rsp)
    eng.ora = oracle.Oracle(lens, nsx)
    eng_v171019 = eng
    p = synth.config2_params(g, r, n_side=48, n_bins=16, fold=_abi.FOLD_FP64)
    full_f, full_c, _ = eng_v171019.profile(p)
    wins = pdist.ring_partition(pdist.ring_costs(p), 3)
    assert wins[0][0] == 0 and wins[-1][1] == 4 * 48
    sf, sc = np.zeros_like(full_f), np.zeros_like(full_c)
    for b, e in wins:
        f, c, info = eng_v171019.profile_rings(p, b, e)
        ref, oinfo = eng_v171019.ora.profile_rings(p, E, b, e)
        assert info.n_points == oinfo.n_points
        assert max_rel(f, ref) < TOL32, (b, e)
        sf += f
        sc += c
    assert np.allclose(sf, full_f, rtol=1e-12, atol=1e-12 * np.abs(full_f).max())
    assert np.allclose(sc, full_c, rtol=1e-12, atol=1e-12 * np.abs(full_c).max())
    batch = eng_v171019.batch([p], rings=wins[1])
    batch.launch()
    bf, bc, _ = batch.collect(want_flux=True, want_counts=True)
    f1, c1, _ = eng_v171019.profile_rings(p, *wins[1])
    assert np.allclose(bf.reshape(f1.shape), f1, rtol=1e-12, atol=1e-300)
    batch.close()
    # point source: ring 0 only
    q = synth.config2_params(g, r, n_side=48, n_bins=16, fold=_abi.FOLD_FP64)
    q.n_spots = 1
    q.spots[0].kind = _abi.SPOT_POINT
    q.spots[0].angrad1 = 0.05
    pf, _, _ = eng_v171019.profile(q)
    f0, _, _ = eng_v171019.profile_rings(q, 0, 1)
    f1, _, i1 = eng_v171019.profile_rings(q, 1, 4 * 48)
    assert np.array_equal(f0, pf) and not f1.any() and i1.n_points == 0
    eng.close()


def test_home_cell_kernel_shapes(eng_v171019):
    """Energy grids that select every home-cell kernel shape: at most 2 (the
    two-slot variant, its own kernel group; also over two warps of cells), up
    to 8 and up to 16 energies per NSX cell (fewer cells per lane), and a grid
    spanning two warps of cells (0.02-60 keV), each against the oracle."""
    ora = eng_v171019.ora
    for E in (synth.energy_grid(128, 0.2, 12.0), synth.energy_grid(160, 0.02, 60.0), synth.energy_grid(600, 0.2, 12.0),
              synth.energy_grid(1100, 0.2, 12.0), synth.energy_grid(400, 0.02, 60.0)):
        g = eng_v171019.add_energy_grid(E)
        p = synth.config2_params(g, -1, n_side=24, n_bins=16)
        flux, _, info = eng_v171019.profile(p, want_counts=False)
        ref, oinfo = ora.profile(p, E)
        assert info.n_points == oinfo.n_points
        assert max_rel(flux, ref) < TOL32, len(E)
