"""Serving (continuous batching): requests of mixed sizes submitted while
others are in flight give the same results as the same profile run alone, and
every ticket reports a latency.  The results are compared bit for bit: a
profile's work tiles cover the same elements in any batch (only their split
over the phase nodes changes), a phase node's partial sums are formed in the
same order, and the flux pool's atomic additions are compensated."""
import numpy as np
import pytest

from gpu_ppm_b200 import _abi, synth
from gpu_ppm_b200.engine import Engine
from tests.errors import max_rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def served():
    lens, nsx = synth.lensing("wide"), synth.nsx("v171019", seed=0)
    e = Engine(n_streams=3, memory_budget=2 << 30)
    e.load_lensing(lens)
    e.load_nsx(nsx)
    grids = {}
    for n in (128, 300):
        E = synth.energy_grid(n, 0.2, 12.0)
        g = e.add_energy_grid(E)
        grids[n] = (g, {ch: e.add_response(g, synth.response(ch, 1000, E, seed=0)) for ch in (300, 1500)})
    yield e, grids
    e.close()


def mixed_requests(grids, n, seed, n_sides=(16, 32, 48, 64), bins=(16, 32)):
    rng = np.random.default_rng(seed)
    out = []
    base, _ = synth.draw_prior(n, seed=seed, lens_u=(0.15, 0.55))
    for p in base:
        ne = int(rng.choice([128, 300]))
        g, rs = grids[ne]
        p.n_side = int(rng.choice(n_sides))
        p.n_bins = int(rng.choice(bins))
        p.n_fine = 6 * p.n_bins
        p.energy_grid = g
        p.response = rs[int(rng.choice([300, 1500]))]
        out.append(p)
    return out


def submit_all(e, reqs):
    bufs, tickets = [], []
    for p in reqs:
        (fs, cs) = e.sizes(p)
        flux, counts = np.zeros(fs), np.zeros(cs)
        bufs.append((flux, counts))
        tickets.append(e.submit(p, flux, counts))
    for t in tickets:
        assert e.wait(t, timeout_ms=120000).status == 0
        e.release(t)
    return bufs


def test_large_requests_mix_equals_alone(served):
    """Served requests at the serving workload's larger sizes (N_side 256 / 512,
    64 / 128 bins, both energy grids and responses) equal the profile alone."""
    e, grids = served
    reqs = mixed_requests(grids, 12, seed=21, n_sides=(256, 512), bins=(64, 128))
    bufs = submit_all(e, reqs)
    for p, (flux, counts) in zip(reqs, bufs):
        f1, c1, _ = e.profile(p)
        assert np.array_equal(flux, f1), (p.n_side, p.n_bins, max_rel(flux, f1))
        assert np.array_equal(counts, c1), (p.n_side, p.n_bins, max_rel(counts, c1))


def test_mix_equals_alone_and_latency_reported(served):
    e, grids = served
    reqs = mixed_requests(grids, 40, seed=5)
    bufs, tickets = [], []
    for p in reqs:
        (fs, cs) = e.sizes(p)
        flux, counts = np.zeros(fs), np.zeros(cs)
        bufs.append((flux, counts))
        tickets.append(e.submit(p, flux, counts))
    for t in tickets:
        info = e.wait(t, timeout_ms=120000)
        assert info.status == 0
        assert e.latency_us(t) > 0
        e.release(t)
        with pytest.raises(_abi.PpmError):  # a released ticket is unknown
            e.poll(t)
    for p, (flux, counts) in zip(reqs, bufs):
        f1, c1, _ = e.profile(p)
        assert np.array_equal(flux, f1), max_rel(flux, f1)
        assert np.array_equal(counts, c1), max_rel(counts, c1)


def test_invalid_request_rejected_at_submit(served):
    e, grids = served
    p = mixed_requests(grids, 1, seed=1)[0]
    p.n_gl = 9
    with pytest.raises(_abi.PpmError):
        e.submit(p, np.zeros(e.sizes(p)[0]), None)


def test_serve_trace_records_every_batch(served):
    e, grids = served
    before = e.serve_trace()
    reqs = mixed_requests(grids, 24, seed=9)
    bufs = [np.zeros(e.sizes(p)[1]) for p in reqs]
    tickets = [e.submit(p, None, b) for p, b in zip(reqs, bufs)]
    for t in tickets:
        assert e.wait(t, timeout_ms=120000).status == 0
        e.release(t)
    new = e.serve_trace()[len(before):]
    assert sum(b["n_requests"] for b in new) == len(reqs)
    for b in new:
        # the GPU may finish before the launch call returns, so finished is ordered only against admit and publish
        assert 0 <= b["t_admit"] <= b["t_launched"] <= b["t_published"]
        assert b["t_admit"] <= b["t_finished"] <= b["t_published"]
        assert b["n_requests"] >= 1 and b["staging_bytes"] >= 32 << 20
