"""Parameter sets reproducing the golden scenarios of tests/golden/make_golden.py
(the reference programs' hard-coded stars plus each scenario's spot/grid)."""
import math

import numpy as np

from gpu_ppm_b200 import _abi, synth

PI = math.pi


def ism_inst(meta):
    lo, hi, n = meta["ism_e"]
    e = synth.energy_grid(n, lo, hi)
    return e, synth.response(meta["ism_ch"], meta["ism_fine"], e, seed=0)


def devarshi_params(s, energy_grid=0, response=0):
    """cpu/devarshi24st_cpu.cpp:48-59: M=1.4, Re=12, nu=300, obs_theta=2.391, D=0.15 kpc,
    exposure 1e6 s, 32 bins, logT=6, NSX 2l2c_le."""
    name, n_side, n_fine, n_pts, _setting, t1, p1, a1, t2, p2, a2 = s
    return synth.params(mass_msun=1.4, r_eq_km=12.0, spin_hz=300.0, inclination_rad=2.391, distance_kpc=0.15,
                        exposure_s=1e6, spots=[synth.spot(t1, p1, a1, t2, p2, a2, logT=6.0)],
                        atmosphere=_abi.ATM_NSX, interp=_abi.INTERP_2L2C_LE, n_side=n_side, n_bins=32, n_gl=n_pts,
                        n_fine=n_fine, energy_grid=energy_grid, response=response)


def os1_params(s, energy_grid=0):
    """cpu/os1_cpu.cpp:30-52: M=1.4, Re=12, kT=0.35 keV, E=1 keV, D=0.2 kpc, N_side=256,
    128 phase points, 3x fine phases; point source when angular radius < 0.1."""
    name, nu, th, ot, ar, beam = s
    kind = _abi.SPOT_POINT if ar < 0.1 else _abi.SPOT_HEALPIX
    beaming = {"i": _abi.BEAM_ISO, "s": _abi.BEAM_SIN2, "c": _abi.BEAM_COS2}[beam]
    return synth.params(mass_msun=1.4, r_eq_km=12.0, spin_hz=float(nu), inclination_rad=ot * PI / 180,
                        distance_kpc=0.2, spots=[synth.spot(th * PI / 180, 0.0, float(ar), kT_keV=0.35, kind=kind)],
                        atmosphere=_abi.ATM_BLACKBODY, beaming=beaming, n_side=256, n_bins=128, n_gl=0,
                        n_fine=384, energy_grid=energy_grid, precision=_abi.PREC_FP64)


def tinterp_energies():
    # cpu/ut.hpp:8-16 linspace(0.1, 5, 1024): beg + i * step (no endpoint fix-up)
    step = (5.0 - 0.1) / (1024 - 1)
    return np.array([0.1 + i * step for i in range(1024)])


def tinterp_params(s, energy_grid=0):
    """cpu/t_interp.cpp:20-32: M=1.4, Re=12, nu=600, D=0.15 kpc, 256 bins, logT=6, point spot."""
    name, n_fine, n_pts, ot, th, ar, interp = s
    return synth.params(mass_msun=1.4, r_eq_km=12.0, spin_hz=600.0, inclination_rad=ot, distance_kpc=0.15,
                        spots=[synth.spot(th, 0.0, ar, logT=6.0, kind=_abi.SPOT_POINT)], atmosphere=_abi.ATM_NSX,
                        interp=interp, n_side=1, n_bins=256, n_gl=n_pts, n_fine=n_fine, energy_grid=energy_grid)
