"""Seeded synthetic inputs with the shapes of the reference's tables.

The reference's real inputs (NSX atmosphere grid, NICER RMF/ARF, ISM table)
live in an external archive that is not available, so every workload runs on
synthetic stand-ins of the same shape and value distribution:

* lensing tables: generated by the engine's restatement of c_lensing.py
  (``ppm_lensing_generate``), "std" grid = 256 u in [0.3, 0.5] x 512 cos psi in
  [-0.9, 1] x 512 cos alpha in [-0.2, 1] (c_lensing.py:8-27);
* NSX grid: the nsx_H_v171019 shape (cpu/nsx.hpp:39-51) — 35 logT x 11 logg x
  166 log(E/kT) x 67 mu — holding log10 of Planck x (1+2mu)/3 x (1 + 0.02 n),
  n a seeded sum of smooth sinusoids in all four axes;
* response: Gaussian redistribution (sigma = 0.05 sqrt(E) keV) times a smooth
  effective-area curve peaking at 1.5 keV on a fine energy grid, reduced to the
  integrand's log-spaced grid with the spline-integration map of
  c_ism_inst.py:72-96.

Files can be written in the reference's text layouts (tables/lensing/<setting>,
the 5-column NSX file, tables/ism_inst/<setting>).
"""
from __future__ import annotations

import ctypes
import hashlib
import math
import os

import numpy as np

from . import _abi

DATA_DIR = os.path.join(_abi.HERE, "_data")

# cgs constants for the synthetic NSX values: I_nu / T^3 = 2 k^3 x^3 / (h^2 c^2 (e^x - 1))
K_B_CGS = 1.380649e-16
H_CGS = 6.62607015e-27
C_CGS = 2.99792458e10
C_T3 = 2.0 * K_B_CGS**3 / (H_CGS**2 * C_CGS**2)

LENSING_SETTINGS = {
    # name: (u_min, u_max, n_u, n_cos_psi = n_cos_alpha)   c_lensing.py:8-27
    "std": (0.3, 0.5, 256, 512),
    "high": (0.3, 0.5, 256, 640),
    "ultra": (0.3, 0.5, 256, 1024),
    # wider u range for randomly drawn stars (same construction, lower u_min / higher u_max)
    "wide": (0.15, 0.55, 256, 512),
}

NSX_SHAPES = {
    # cpu/nsx.hpp:25-51
    "v171019": dict(n_logT=35, n_logg=11, n_logEkT=166, n_mu=67, logT=(5.10, 6.80), logg=(13.7, 14.7),
                    logEkT=(-1.30, 2.00)),
    "v200804": dict(n_logT=35, n_logg=14, n_logEkT=166, n_mu=67, logT=(5.10, 6.80), logg=(13.7, 15.0),
                    logEkT=(-1.30, 2.00)),
}


# --------------------------------------------------------------------------- lensing
class LensingTables:
    """Holds one set of lensing tables (arrays are float64, C-contiguous)."""

    def __init__(self, u, cos_psi, cos_alpha, ca, lf, cdt):
        self.u, self.cos_psi, self.cos_alpha = u, cos_psi, cos_alpha  # (min, max, n)
        self.ca = np.ascontiguousarray(ca, dtype=np.float64)
        self.lf = np.ascontiguousarray(lf, dtype=np.float64)
        self.cdt = np.ascontiguousarray(cdt, dtype=np.float64)

    def desc(self):
        d = _abi.LensingDesc()
        d.u_min, d.u_max, d.n_u = self.u
        d.cos_psi_min, d.cos_psi_max, d.n_cos_psi = self.cos_psi
        d.cos_alpha_min, d.cos_alpha_max, d.n_cos_alpha = self.cos_alpha
        d.cos_alpha_of_u_cos_psi = _abi.dptr(self.ca)
        d.lf_of_u_cos_psi = _abi.dptr(self.lf)
        d.cdt_over_R_of_u_cos_alpha = _abi.dptr(self.cdt)
        d._keep = self  # keep arrays alive with the struct
        return d

    def write_dir(self, folder):
        """Writes the tables/lensing/<setting> layout (c_lensing.py:35-44,109-110,155)."""
        os.makedirs(folder, exist_ok=True)
        for name, (lo, hi, n) in (("u", self.u), ("cos_psi", self.cos_psi), ("cos_alpha", self.cos_alpha)):
            with open(os.path.join(folder, f"{name}.txt"), "w") as f:
                f.write(f"{lo!r} {hi!r} {n}\n")
        np.savetxt(os.path.join(folder, "cos_alpha_of_u_cos_psi.txt"), self.ca, fmt="%.17g")
        np.savetxt(os.path.join(folder, "lf_of_u_cos_psi.txt"), self.lf, fmt="%.17g")
        np.savetxt(os.path.join(folder, "cdt_over_R_of_u_cos_alpha.txt"), self.cdt, fmt="%.17g")


def generate_lensing(u_min, u_max, n_u, n_cos_psi, n_cos_alpha=None, cos_psi=(-0.9, 1.0), cos_alpha=(-0.2, 1.0),
                     n_threads=0):
    n_cos_alpha = n_cos_alpha or n_cos_psi
    spec = _abi.LensingSpec(u_min, u_max, n_u, cos_psi[0], cos_psi[1], n_cos_psi, cos_alpha[0], cos_alpha[1],
                            n_cos_alpha, n_threads)
    ca = np.zeros((n_u, n_cos_psi))
    lf = np.zeros((n_u, n_cos_psi))
    cdt = np.zeros((n_u, n_cos_alpha))
    _abi.check(_abi.lib().ppm_lensing_generate(ctypes.byref(spec), _abi.dptr(ca), _abi.dptr(lf), _abi.dptr(cdt)))
    return LensingTables((u_min, u_max, n_u), (cos_psi[0], cos_psi[1], n_cos_psi),
                         (cos_alpha[0], cos_alpha[1], n_cos_alpha), ca, lf, cdt)


def lensing(setting="std", cache=True):
    """Lensing tables for a named setting, cached under gpu_ppm_b200/_data."""
    u_min, u_max, n_u, n = LENSING_SETTINGS[setting]
    key = f"lensing_{setting}_{u_min}_{u_max}_{n_u}_{n}"
    path = os.path.join(DATA_DIR, key + ".npz")
    if cache and os.path.exists(path):
        z = np.load(path)
        return LensingTables((u_min, u_max, n_u), (-0.9, 1.0, n), (-0.2, 1.0, n), z["ca"], z["lf"], z["cdt"])
    t = generate_lensing(u_min, u_max, n_u, n)
    if cache:
        os.makedirs(DATA_DIR, exist_ok=True)
        tmp = path + f".{os.getpid()}.tmp.npz"
        np.savez(tmp, ca=t.ca, lf=t.lf, cdt=t.cdt)
        os.replace(tmp, path)
    return t


def small_lensing(n_u=24, n=48, u=(0.3, 0.5)):
    """A coarse lensing table for quick CPU tests (same construction)."""
    return generate_lensing(u[0], u[1], n_u, n)


# --------------------------------------------------------------------------- NSX
class NsxTable:
    def __init__(self, n_logT, n_logg, n_logEkT, n_mu, logT, logg, logEkT, mu, log_I):
        self.n = (n_logT, n_logg, n_logEkT, n_mu)
        self.logT, self.logg, self.logEkT = logT, logg, logEkT  # (min, max)
        self.mu = np.ascontiguousarray(mu, dtype=np.float64)
        self.log_I = np.ascontiguousarray(log_I, dtype=np.float64).reshape(self.n)

    def axis(self, k):
        lo, hi = (self.logT, self.logg, self.logEkT)[k]
        n = self.n[k]
        # UniformHunt::operator[] (cpu/hunt.hpp:129): x_min + (x_max - x_min) * i / (n - 1)
        return np.array([lo + (hi - lo) * i / (n - 1) for i in range(n)])

    def desc(self):
        d = _abi.NsxDesc()
        d.n_logT, d.n_logg, d.n_logEkT, d.n_mu = self.n
        d.logT_min, d.logT_max = self.logT
        d.logg_min, d.logg_max = self.logg
        d.logEkT_min, d.logEkT_max = self.logEkT
        d.mu = _abi.dptr(self.mu)
        d.log_I_T3 = _abi.dptr(self.log_I.reshape(-1))
        d._keep = self
        return d

    def axes_desc(self):
        d = self.desc()
        d.mu = None
        d.log_I_T3 = None
        return d

    def write_file(self, path):
        """Five-column NSX text file (cpu/nsx.hpp:98-103): logEkT mu logInuT3 logT logg,
        loop order logT -> logg -> logEkT -> mu."""
        nT, ng, nE, nm = self.n
        T = self.axis(0)
        G = self.axis(1)
        E = self.axis(2)
        iT, ig, iE, im = np.meshgrid(np.arange(nT), np.arange(ng), np.arange(nE), np.arange(nm), indexing="ij")
        cols = np.stack([E[iE].ravel(), self.mu[im].ravel(), self.log_I.ravel(), T[iT].ravel(), G[ig].ravel()], 1)
        os.makedirs(os.path.dirname(os.path.abspath(path)), exist_ok=True)
        with open(path, "w") as f:
            # %.17g round-trips doubles exactly
            np.savetxt(f, cols, fmt="%.17g")


def mu_grid(n_mu):
    """Strictly descending emission-angle cosines 1 -> 0 (denser near mu = 1)."""
    mu = np.cos(np.linspace(0.0, 0.5 * np.pi, n_mu))
    mu[-1] = 0.0
    return mu


def nsx(shape="v171019", seed=0, n_mu=None, dims=None):
    """Synthetic NSX-shaped table: log10( x^3/expm1(x) C (1+2mu)/3 (1 + 0.02 n) ), x = 10^logEkT."""
    s = dict(NSX_SHAPES[shape])
    if dims is not None:
        s.update(dims)
    if n_mu is not None:
        s["n_mu"] = n_mu
    nT, ng, nE, nm = s["n_logT"], s["n_logg"], s["n_logEkT"], s["n_mu"]
    tab = NsxTable(nT, ng, nE, nm, s["logT"], s["logg"], s["logEkT"], mu_grid(nm), np.zeros((nT, ng, nE, nm)))
    T, G, E, mu = tab.axis(0), tab.axis(1), tab.axis(2), tab.mu
    rng = np.random.default_rng(seed)
    K = 6
    freqs = rng.choice([0.0, 0.5, 1.0, 1.5, 2.0], size=(K, 4))
    amps = rng.uniform(0.2, 1.0, size=K)
    amps /= amps.sum()
    phases = rng.uniform(0, 2 * np.pi, size=K)
    tT = (T - T[0]) / (T[-1] - T[0])
    tg = (G - G[0]) / (G[-1] - G[0]) if ng > 1 else np.zeros(ng)
    tE = (E - E[0]) / (E[-1] - E[0])
    arg = np.zeros((nT, ng, nE, nm))
    noise = np.zeros((nT, ng, nE, nm))
    for k in range(K):
        arg = (2 * np.pi * (freqs[k, 0] * tT[:, None, None, None] + freqs[k, 1] * tg[None, :, None, None]
                            + freqs[k, 2] * tE[None, None, :, None] + freqs[k, 3] * mu[None, None, None, :])
               + phases[k])
        noise += amps[k] * np.sin(arg)
    x = 10.0 ** E
    planck = x**3 / np.expm1(x)
    beaming = (1.0 + 2.0 * mu) / 3.0
    val = C_T3 * planck[None, None, :, None] * beaming[None, None, None, :] * (1.0 + 0.02 * noise)
    tab.log_I = np.log10(val)
    return tab


# --------------------------------------------------------------------------- energies / response
def energy_grid(n, lo, hi):
    """Log-spaced observed energies in keV (numpy.geomspace, c_ism_inst.py:72)."""
    return np.geomspace(lo, hi, n)


def effective_area(E, seed=0):
    """Smooth effective-area curve (cm^2) peaking at 1.5 keV."""
    rng = np.random.default_rng(seed + 1)
    a = rng.uniform(-1, 1, size=3)
    lnE = np.log(E / 1.5)
    wiggle = 1.0 + 0.05 * (a[0] * np.sin(1.3 * lnE) + a[1] * np.sin(2.1 * lnE + 0.4) + a[2] * np.cos(0.7 * lnE))
    return 1000.0 * np.exp(-lnE**2 / (2 * 0.6**2)) * wiggle


def response(n_ch, n_fine, e_obs, seed=0):
    """Response rsp[n_ch][len(e_obs)].

    Fine grid: n_fine equal bins over [e_obs[0], e_obs[-1]]; R_fine[ch][j] = A(E_j) x Gaussian
    redistribution of E_j into channel ch (sigma = 0.05 sqrt(E_j) keV, channel centres linear
    over the range).  Reduced to e_obs with C[j][i] = integral over fine bin j of the cubic
    spline through the i-th unit vector on e_obs (c_ism_inst.py:75-96), rsp = R_fine @ C.
    """
    from scipy.interpolate import CubicSpline

    lo, hi = float(e_obs[0]), float(e_obs[-1])
    edges = np.linspace(lo, hi, n_fine + 1)
    E_lo, E_hi = edges[:-1], edges[1:]
    E_mid = 0.5 * (E_lo + E_hi)
    ch_centres = np.linspace(lo, hi, n_ch)
    dch = (hi - lo) / n_ch
    sigma = 0.05 * np.sqrt(E_mid)
    gauss = np.exp(-((ch_centres[:, None] - E_mid[None, :]) ** 2) / (2 * sigma[None, :] ** 2)) / (
        sigma[None, :] * np.sqrt(2 * np.pi))
    R_fine = effective_area(E_mid, seed)[None, :] * gauss * dch
    cs = CubicSpline(e_obs, np.eye(len(e_obs)), axis=0)
    anti = cs.antiderivative()
    C = anti(E_hi) - anti(E_lo)  # [n_fine, n_e]
    rsp = R_fine @ C
    rsp[np.abs(rsp) < 1e-300] = 0.0
    return np.ascontiguousarray(rsp)


def write_ism_inst(folder, e_obs, rsp):
    """tables/ism_inst/<setting> layout: num.txt, E_obs.txt, rsp.txt (c_ism_inst.py:63-101)."""
    os.makedirs(folder, exist_ok=True)
    with open(os.path.join(folder, "num.txt"), "w") as f:
        f.write(f"{rsp.shape[0]} {rsp.shape[1]}\n")
    np.savetxt(os.path.join(folder, "E_obs.txt"), e_obs, fmt="%.17g")
    np.savetxt(os.path.join(folder, "rsp.txt"), rsp, fmt="%.17g")


# --------------------------------------------------------------------------- parameter sets
def spot(theta1, phi1, angrad1, theta2=0.0, phi2=0.0, angrad2=0.0, logT=6.0, kT_keV=0.0, kind=_abi.SPOT_HEALPIX):
    return dict(theta1=theta1, phi1=phi1, angrad1=angrad1, theta2=theta2, phi2=phi2, angrad2=angrad2, logT=logT,
                kT_keV=kT_keV, kind=kind)


def params(**kw):
    """Builds a ppm_params struct from keyword arguments (spots: list of dicts from `spot`)."""
    p = _abi.Params()
    defaults = dict(mass_msun=1.4, r_eq_km=12.0, spin_hz=300.0, inclination_rad=2.391, distance_kpc=0.15,
                    exposure_s=1e6, atmosphere=_abi.ATM_NSX, interp=_abi.INTERP_2L2C_LE, beaming=_abi.BEAM_ISO,
                    n_side=64, n_bins=32, n_gl=2, n_fine=None, energy_grid=0, response=-1,
                    precision=_abi.PREC_FP32, fold=_abi.FOLD_BF16X3)
    defaults.update(kw)
    spots = defaults.pop("spots")
    if defaults["n_fine"] is None:
        defaults["n_fine"] = 6 * defaults["n_bins"]  # cpu/devarshi24st_cpu.cpp:272
    for k, v in defaults.items():
        setattr(p, k, v)
    p.n_spots = len(spots)
    for i, s in enumerate(spots):
        for k, v in s.items():
            setattr(p.spots[i], k, v)
    return p


DEG = math.pi / 180.0


def config1_params(energy_grid=0):
    """Blackbody single disk, FP64 (the os1 workload with GL bins and an energy grid)."""
    return params(mass_msun=1.4, r_eq_km=12.0, spin_hz=300.0, inclination_rad=50 * DEG, distance_kpc=1.0,
                  spots=[spot(40 * DEG, 0.0, 0.25, kT_keV=0.3)], atmosphere=_abi.ATM_BLACKBODY, n_side=64,
                  n_bins=32, n_gl=2, energy_grid=energy_grid, response=-1, precision=_abi.PREC_FP64)


def config2_spots(logT=6.0):
    ring = spot(30 * DEG, 0.0, 0.3, 30 * DEG, 0.0, 0.1, logT=logT)
    crescent = spot(120 * DEG, 0.0, 0.35, 120 * DEG - 0.1, 0.0, 0.2, logT=logT)
    return [ring, crescent]


def config2_params(energy_grid=0, response=0, n_side=256, n_bins=64, fold=_abi.FOLD_BF16X3):
    """Ring + crescent, NSX 2l2c_le, Nside 256, 64 bins, 300 energies, 300-channel fold."""
    return params(mass_msun=1.6, r_eq_km=12.5, spin_hz=400.0, inclination_rad=60 * DEG, distance_kpc=0.15,
                  exposure_s=1e6, spots=config2_spots(), atmosphere=_abi.ATM_NSX, interp=_abi.INTERP_2L2C_LE,
                  n_side=n_side, n_bins=n_bins, n_gl=2, energy_grid=energy_grid, response=response,
                  precision=_abi.PREC_FP32, fold=fold)


def config3_params(energy_grid=0, response=0, fold=_abi.FOLD_BF16X3):
    return config2_params(energy_grid, response, n_side=512, n_bins=128, fold=fold)


def star_u_logg(mass, r_eq, spin):
    """Equatorial/polar compactness u = Rs/R and surface gravity log g for a star
    (cpu/devarshi24st_cpu.cpp:63-124 evaluated at the equator and the pole)."""
    Rs = mass * 2.9532501
    x = 0.5 * Rs / r_eq
    Ob = 2 * math.pi * spin * math.sqrt(r_eq**3 / mass) * 2.745011592867327e-6
    o2 = Ob * Ob * (-0.788 + 1.030 * x)
    out = []
    for c in (0.0, 1.0):
        R = r_eq * (1.0 + o2 * c * c)
        u = Rs / R
        ce, cp = -0.791 + 0.776 * x, 1.138 - 1.431 * x
        de, fe = -1.315 * x + 2.431 * x * x, -1.172 * x
        dp, fp = 0.653 * x - 2.864 * x * x, 0.975 * x
        d60 = 13.47 * x - 27.13 * x * x
        Ob2 = Ob * Ob
        Ob4, Ob6 = Ob2 * Ob2, Ob2 * Ob2 * Ob2
        g_g0 = 1 + (1 - c * c) * (ce * Ob2 + de * Ob4 + fe * Ob6) + c * c * (cp * Ob2 + dp * Ob4 + fp * Ob6 - d60 * Ob4) \
            + abs(c) * d60 * Ob4
        logg = math.log10(g_g0) + math.log10(mass / (r_eq * r_eq * math.sqrt(1 - Rs / r_eq))) \
            + math.log10(1.32712440041279419E16)
        out.append((u, logg))
    return out


def random_spot(rng, logT):
    """One spot drawn from the batching prior: colatitude U[0,180] deg, angular radius
    logU[0.01, 1.0] rad, morphology disk / ring / crescent / difference of disks."""
    th = rng.uniform(0.0, math.pi)
    ph = rng.uniform(0.0, 2 * math.pi)
    rho = math.exp(rng.uniform(math.log(0.01), math.log(1.0)))
    kind = int(rng.integers(0, 4))
    if kind == 0:  # disk
        return spot(th, ph, rho, logT=logT)
    if kind == 1:  # ring
        return spot(th, ph, rho, th, ph, rho * rng.uniform(0.2, 0.8), logT=logT)
    if kind == 2:  # crescent (offset along colatitude)
        d = rho * rng.uniform(0.2, 0.5)
        return spot(th, ph, rho, th - d, ph, rho * rng.uniform(0.5, 0.9), logT=logT)
    d = rho * rng.uniform(0.3, 0.9)  # difference of disks (offset in azimuth)
    return spot(th, ph, rho, th, ph + d, rho * rng.uniform(0.3, 1.0), logT=logT)


def draw_prior(n, seed=0, lens_u=(0.15, 0.55), nsx_logg=(13.7, 14.7), n_side=256, n_bins=64, energy_grid=0,
               response=0, fold=_abi.FOLD_BF16X3):
    """Draws n parameter sets from the batching prior; draws whose equatorial or polar u lies
    outside the lensing table, or whose log g leaves the NSX table, are rejected and redrawn.
    Returns (list of Params, rejection rate)."""
    rng = np.random.default_rng(seed)
    out = []
    tried = 0
    while len(out) < n:
        tried += 1
        M = rng.uniform(1.0, 2.2)
        R = rng.uniform(9.0, 15.0)
        nu = rng.uniform(100.0, 700.0)
        inc = rng.uniform(5.0, 90.0) * DEG
        logT = rng.uniform(5.8, 6.6)
        n_sp = int(rng.integers(1, 3))
        spots = [random_spot(rng, logT) for _ in range(n_sp)]
        (u_eq, g_eq), (u_po, g_po) = star_u_logg(M, R, nu)
        if not (lens_u[0] <= min(u_eq, u_po) and max(u_eq, u_po) <= lens_u[1]):
            continue
        if not (nsx_logg[0] <= min(g_eq, g_po) and max(g_eq, g_po) <= nsx_logg[1]):
            continue
        out.append(params(mass_msun=M, r_eq_km=R, spin_hz=nu, inclination_rad=inc, distance_kpc=0.15,
                          exposure_s=1e6, spots=spots, atmosphere=_abi.ATM_NSX, interp=_abi.INTERP_2L2C_LE,
                          n_side=n_side, n_bins=n_bins, n_gl=2, energy_grid=energy_grid, response=response,
                          precision=_abi.PREC_FP32, fold=fold))
    return out, 1.0 - n / tried


def params_key(p):
    return hashlib.sha1(bytes(p)).hexdigest()[:12]
