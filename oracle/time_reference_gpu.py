"""Times the reference's OWN CUDA program (gpu/devarshi24st_gpu.cu, built unchanged
for sm_100a into oracle/_ref/ref_devarshi_gpu by oracle/Makefile) and the engine
on the same GPU, tables and scenarios, and prints one JSON line per scenario.

The reference program hard-codes its star (gpu/devarshi24st_gpu.cu:22-44: M = 1.4,
R_eq = 12 km, 300 Hz, inclination 2.391, 32 phase bins, logT = 6, D = 0.15 kpc), so
the scenarios are fixed-star ones: its four std stars at its own N_side
(:123-127, :520-524) and the two-spot ring/crescent at N_side 256, with 300
energies over 0.2-12 keV and a 300-channel response.

* reference: calc_one_star's own CUDA-event time of its kernel and cuBLAS fold
  (:452-483), read from its output; the first scenario is the program's warm-up.
* engine device: one plan + integrand + fold pass of a one-profile batch,
  CUDA events around each phase (ppm_batch_launch_timed); the phases
  (clear + plan, integrand, fold) are reported too.  The events between the
  phases add their own gaps, so the pass is also timed whole: the batch's
  captured graph (ppm_batch_launch) between two events, as the reference
  times its kernel (engine graph).
* engine plain: the synchronous ppm_profile call, host wall clock, counts
  downloaded to the host.

Also reports the largest relative difference between the two programs' counts
(floor 1e-6 of the maximum; informative: the reference's GPU lookups do not
clamp where its CPU does, and the engine follows the CPU).

--program os1 times the reference's blackbody program (gpu/os1_gpu.cu, built
unchanged into oracle/_ref/ref_os1_gpu) on its ten compile-time OS1 stars
(:54-63: N_side 256, 128 point-sampled phases, 1 keV) beside the engine's
blackbody path in FP32 (the reference's arithmetic) and FP64 (the engine's
parity default for this mode); the reference time is its kernel alone.
MEASUREMENT INFRASTRUCTURE ONLY; runs on a GPU with the reference programs
prebuilt.

    python oracle/time_reference_gpu.py [--repeats 3] [--program devarshi|os1|all]
    python oracle/time_reference_gpu.py --layout DIR [--only NAME]   # tables + scen.txt only (for a profiler)
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import re
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

PI = math.pi
# gpu/os1_gpu.cu:54-63: name, spin (Hz), spot colatitude (deg), inclination (deg), angular radius, beaming
OS1 = [
    ("os1a", 600, 90, 90, 0.01, "i"), ("os1b", 600, 90, 90, 1.0, "i"), ("os1c", 200, 90, 90, 0.01, "i"),
    ("os1d", 1, 90, 90, 1.0, "i"), ("os1e", 600, 60, 30, 1.0, "i"), ("os1f", 600, 20, 80, 1.0, "i"),
    ("os1g", 600, 60, 30, 1.0, "c"), ("os1h", 600, 60, 30, 1.0, "s"), ("os1i", 600, 20, 80, 1.0, "c"),
    ("os1j", 600, 20, 80, 1.0, "s"),
]
# name, N_side, N_fine, N_pts, setting, theta1, phi1, angrad1, theta2, phi2, angrad2
SCENARIOS = [
    ("Ring_Eq", 173, 192, 2, "std", 0.5 * PI, -0.2, 0.5, 0.5 * PI, 0.0, 0.25),
    ("Ring_Polar", 1708, 192, 2, "std", PI - 0.001, -0.02, 0.05, PI - 0.001, 0.0, 0.025),
    ("Crescent_Eq", 128, 192, 2, "std", 1.0, -1.0, 1.4, 0.5, 0.0, 0.5 * PI - 0.001),
    ("Crescent_Polar", 189, 192, 2, "std", 1.15, -0.1, 1.3, 1.75, 0.0, 0.5 * PI - 0.001),
    ("Cfg2_Ring", 256, 192, 2, "std", 30 * PI / 180, 0.0, 0.3, 30 * PI / 180, 0.0, 0.1),
    ("Cfg2_Crescent", 256, 192, 2, "std", 120 * PI / 180, 0.0, 0.35, 120 * PI / 180 - 0.1, 0.0, 0.2),
]


def max_rel(a, ref, floor=1e-6):
    scale = np.abs(ref).max()
    if scale == 0:
        return float(np.abs(a).max())
    denom = np.where(np.abs(ref) >= floor * scale, np.abs(ref), scale)
    return float((np.abs(a - ref) / denom).max())


def write_layout(d, lens, nsx, E, rsp, lines):
    """The reference program's working directory: tables, NSX file, output/ and scen.txt."""
    lens.write_dir(os.path.join(d, "tables", "lensing", "std"))
    nsx.write_file(os.path.join(d, "ext", "model_data", "nsx_H_v200804.out"))
    synth_mod().write_ism_inst(os.path.join(d, "tables", "ism_inst", "std"), E, rsp)
    os.makedirs(os.path.join(d, "output"), exist_ok=True)
    path = os.path.join(d, "scen.txt")
    with open(path, "w") as f:
        for ln in lines:
            f.write(" ".join(repr(x) if isinstance(x, float) else str(x) for x in ln) + "\n")
    return path


def synth_mod():
    from gpu_ppm_b200 import synth

    return synth


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--repeats", type=int, default=3)
    ap.add_argument("--layout", help="only write the reference program's working directory here and exit")
    ap.add_argument("--only", help="scenario name: for --layout, or the one star the engine runs (--program os1)")
    ap.add_argument("--program", default="all", choices=("devarshi", "os1", "all"))
    args = ap.parse_args()
    if args.layout:
        synth = synth_mod()
        E = synth.energy_grid(300, 0.2, 12.0)
        scen = [s for s in SCENARIOS if args.only in (None, s[0])]
        if not scen:
            raise SystemExit(f"unknown scenario {args.only}")
        write_layout(args.layout, synth.lensing("std"), synth.nsx("v200804", seed=0), E,
                     synth.response(300, 1000, E, seed=0), scen)
        return
    if args.program in ("devarshi", "all"):
        devarshi(args)
    if args.program in ("os1", "all"):
        os1(args)


def engine_times(eng, prm, repeats, want_counts):
    """Median device time of a one-profile batch pass and median wall time of the plain call, plus its output."""
    import torch

    from gpu_ppm_b200 import _abi

    stream = torch.cuda.Stream()
    batch = eng.batch([prm])
    ms3 = (ctypes.c_float * 3)()
    dev, phases = [], []
    for k in range(repeats + 1):
        _abi.check(_abi.lib().ppm_batch_launch_timed(eng.h, batch.h, ctypes.c_void_p(stream.cuda_stream), ms3))
        if k:
            dev.append(float(sum(ms3)))
            phases.append(list(ms3))
    engine_times.last_phases = [float(x) for x in np.median(np.array(phases), axis=0)]
    graph = []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for k in range(repeats + 1):
        e0.record(stream)
        _abi.check(_abi.lib().ppm_batch_launch(eng.h, batch.h, ctypes.c_void_p(stream.cuda_stream)))
        e1.record(stream)
        e1.synchronize()
        if k:
            graph.append(e0.elapsed_time(e1))
    engine_times.last_graph = float(np.median(graph))
    batch.close()
    plain = []
    for k in range(repeats + 1):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        flux, counts, info = eng.profile(prm, want_flux=not want_counts, want_counts=want_counts)
        if k:
            plain.append(1000.0 * (time.perf_counter() - t0))
    return float(np.median(dev)), float(np.median(plain)), (counts if want_counts else flux), info


def os1(args):
    prog = os.path.join(ROOT, "oracle", "_ref", "ref_os1_gpu")
    if not os.path.exists(prog):
        raise SystemExit(f"{prog} is missing: build it with `make -C oracle ref REF=<reference source tree>` where the reference sources are")
    from gpu_ppm_b200 import _abi, synth
    from gpu_ppm_b200.engine import Engine

    lens = synth.lensing("std")
    ref_ms, ref_flux = {}, {}
    with tempfile.TemporaryDirectory() as tmp:
        lens.write_dir(os.path.join(tmp, "tables", "lensing", "std"))
        os.makedirs(os.path.join(tmp, "output"))
        p = subprocess.run([prog, str(args.repeats)], cwd=tmp, capture_output=True, text=True, timeout=600)
        if p.returncode != 0:
            raise SystemExit(f"reference program failed ({p.returncode}): {p.stderr[-2000:]}")
        times = [float(m) for m in re.findall(r"Time taken: ([0-9.eE+-]+) ms", p.stdout)]
        assert len(times) == 1 + len(OS1) * args.repeats, len(times)
        for k, s in enumerate(OS1):
            ref_ms[s[0]] = float(np.median(times[1 + k * args.repeats: 1 + (k + 1) * args.repeats]))
            ref_flux[s[0]] = np.loadtxt(os.path.join(tmp, "output", f"{s[0]}_gpu.txt"))
    eng = Engine(device=0)
    eng.load_lensing(lens)
    g = eng.add_energy_grid(np.array([1.0]))
    for name, nu, th, inc, ar, beam in OS1:
        if args.only and name != args.only:
            continue
        row = {"scenario": name, "reference_gpu_ms": ref_ms[name], "repeats": args.repeats}
        for prec, tag in ((_abi.PREC_FP32, "fp32"), (_abi.PREC_FP64, "fp64")):
            kind = _abi.SPOT_POINT if ar < 0.1 else _abi.SPOT_HEALPIX
            beaming = {"i": _abi.BEAM_ISO, "s": _abi.BEAM_SIN2, "c": _abi.BEAM_COS2}[beam]
            prm = synth.params(mass_msun=1.4, r_eq_km=12.0, spin_hz=float(nu), inclination_rad=inc * PI / 180,
                               distance_kpc=0.2, spots=[synth.spot(th * PI / 180, 0.0, float(ar), kT_keV=0.35, kind=kind)],
                               atmosphere=_abi.ATM_BLACKBODY, beaming=beaming, n_side=256, n_bins=128, n_gl=0,
                               n_fine=384, energy_grid=g, precision=prec)
            dev, plain, flux, _ = engine_times(eng, prm, args.repeats, want_counts=False)
            row.update({f"engine_{tag}_device_ms": dev, f"engine_{tag}_plain_ms": plain,
                        f"engine_{tag}_graph_ms": engine_times.last_graph,
                        f"engine_{tag}_phases_ms": engine_times.last_phases,
                        f"speedup_{tag}_device": ref_ms[name] / dev,
                        f"max_rel_diff_{tag}": max_rel(np.asarray(flux).reshape(-1), ref_flux[name])})
        print(json.dumps(row), flush=True)
    eng.close()


def devarshi(args):
    prog = os.path.join(ROOT, "oracle", "_ref", "ref_devarshi_gpu")
    if not os.path.exists(prog):
        raise SystemExit(f"{prog} is missing: build it with `make -C oracle ref` where the reference sources are")

    from gpu_ppm_b200 import _abi, synth
    from gpu_ppm_b200.engine import Engine

    lens, nsx = synth.lensing("std"), synth.nsx("v200804", seed=0)
    E = synth.energy_grid(300, 0.2, 12.0)
    rsp = synth.response(300, 1000, E, seed=0)
    ref_ms, ref_counts = {}, {}
    with tempfile.TemporaryDirectory() as tmp:
        lines = [("Warmup",) + SCENARIOS[0][1:]] + [s for s in SCENARIOS for _ in range(args.repeats)]
        path = write_layout(tmp, lens, nsx, E, rsp, lines)
        p = subprocess.run([prog, path], cwd=tmp, capture_output=True, text=True, timeout=1200)
        if p.returncode != 0:
            raise SystemExit(f"reference program failed ({p.returncode}): {p.stderr[-2000:]}")
        times = [float(m) for m in re.findall(r"Time taken: ([0-9.eE+-]+) ms", p.stdout)]
        assert len(times) == len(lines), (len(times), len(lines))
        for (name, *_), t in zip(lines[1:], times[1:]):
            ref_ms.setdefault(name, []).append(t)
        for s in SCENARIOS:
            ref_counts[s[0]] = np.loadtxt(os.path.join(tmp, "output", f"{s[0]}_std_counts_gpu.txt"))

    eng = Engine(device=0)
    eng.load_lensing(lens)
    eng.load_nsx(nsx)
    g = eng.add_energy_grid(E)
    r = eng.add_response(g, rsp)
    for name, n_side, n_fine, n_pts, _set, t1, p1, a1, t2, p2, a2 in SCENARIOS:
        prm = synth.params(mass_msun=1.4, r_eq_km=12.0, spin_hz=300.0, inclination_rad=2.391, distance_kpc=0.15,
                           exposure_s=1e6, spots=[synth.spot(t1, p1, a1, t2, p2, a2, logT=6.0)],
                           atmosphere=_abi.ATM_NSX, interp=_abi.INTERP_2L2C_LE, n_side=n_side, n_bins=32,
                           n_gl=n_pts, n_fine=n_fine, energy_grid=g, response=r)
        dev, plain, counts, info = engine_times(eng, prm, args.repeats, want_counts=True)
        ref = float(np.median(ref_ms[name]))
        print(json.dumps({
            "scenario": name, "n_side": n_side, "energies": len(E), "channels": rsp.shape[0], "bins": 32,
            "reference_gpu_ms": ref, "engine_device_ms": dev, "engine_plain_ms": plain,
            "engine_graph_ms": engine_times.last_graph, "engine_phases_ms": engine_times.last_phases,
            "speedup_device": ref / dev, "speedup_plain": ref / plain,
            "max_rel_diff_counts": max_rel(counts.reshape(ref_counts[name].shape), ref_counts[name]),
            "repeats": args.repeats, "visible_points": int(info.n_points),
        }), flush=True)
    eng.close()


if __name__ == "__main__":
    main()
