"""Host-side helpers of bench.py: its error metric is the parity tests' metric,
the bench-workload parity check recovers a known error, and the CPU-baseline
sample respects its time budget."""
import types

import numpy as np

import bench
import oracle
from gpu_ppm_b200 import synth
from tests.errors import FLOOR, max_rel


def test_bench_metric_matches_parity_metric():
    rng = np.random.default_rng(3)
    ref = rng.random((300, 64)) * 10.0 ** rng.integers(-9, 1, size=(300, 64))
    a = ref * (1 + 1e-5 * rng.standard_normal(ref.shape))
    assert bench.REL_FLOOR == FLOOR
    assert bench.max_rel(a, ref) == max_rel(a, ref)
    assert bench.max_rel(np.zeros(4), np.zeros(4)) == 0.0


def test_parity_vs_oracle_recovers_a_planted_error():
    E = synth.energy_grid(300, 0.2, 12.0)
    rsp = synth.response(300, 1000, E, seed=0)
    plist = [types.SimpleNamespace(n_bins=b, exposure_s=1e6) for b in (32, 64, 128, 64, 32)]
    rng = np.random.default_rng(1)
    sample = np.array([3, 0, 2])
    ref_flux = [rng.random((plist[i].n_bins, 300)) for i in sample]
    off = np.cumsum([0] + [300 * p.n_bins for p in plist])
    counts = np.zeros(off[-1])
    for k, i in enumerate(sample):
        c = oracle.fold(rsp, ref_flux[k], 1e6) * (1 + (2e-6 if k == 1 else 0.0))
        counts[off[i]:off[i + 1]] = c.ravel()
    out = bench.parity_vs_oracle(sample, ref_flux, plist, counts, rsp)
    assert out["profiles"] == 3
    assert abs(out["max_rel_err"] - 2e-6) < 1e-12
    assert out["median_rel_err"] < 1e-12


def test_choose_sample_respects_budget_and_spreads():
    counts = np.arange(1, 4097) * 10
    order = np.argsort(counts)
    s = bench.choose_sample(order, counts, seconds=1.0, cores=4)
    budget = 1.0 * 4 * 1e9 / 60.0
    assert len(s) >= 1
    assert counts[s].sum() * 64 * 2 * 300 <= budget or len(s) == 1
    assert len(set(s.tolist())) == len(s)


def test_cpu_model_is_reported():
    assert isinstance(bench.cpu_model(), str) and bench.cpu_model()


def test_sustainable_rate_is_the_highest_rate_kept_up_with_under_the_bound():
    def run(rate, thr, p99):
        return {"offered_req_per_s": rate, "throughput_req_per_s": thr, "p50_ms": 1.0, "p99_ms": p99}

    curve = [run(100, 99, 5), run(500, 495, 12), run(1000, 980, 40), run(1500, 1200, 30), run(2000, 1190, 280)]
    assert bench.sustainable(curve, 50.0)["offered_req_per_s"] == 1000  # 1500 is not kept up with
    assert bench.sustainable(curve, 10.0)["offered_req_per_s"] == 100
    assert bench.sustainable(curve, 1.0) is None


def test_trace_summary_counts_only_the_batches_admitted_after_the_mark():
    def batch(admit, launched, finished, published, n):
        return {"t_admit": admit, "t_launched": launched, "t_finished": finished, "t_published": published,
                "n_requests": n, "stream_slot": 0, "staging_bytes": 0}

    trace = [batch(10, 20, 1020, 1030, 4), batch(2000, 2500, 4500, 4510, 8), batch(3000, 3100, 9100, 9300, 2)]
    s = bench.trace_summary(trace, 10)
    assert s["batches"] == 2 and s["batch_requests_max"] == 8 and s["batch_requests_mean"] == 5.0
    assert s["build_ms_max"] == 0.5 and s["gpu_ms_max"] == 6.0 and s["gpu_ms_p50"] == 4.0
    assert s["publish_ms_max"] == 0.2
    assert bench.trace_summary(trace, 5000) == {"batches": 0}
