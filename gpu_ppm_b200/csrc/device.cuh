// Device-side data layout and the per-element physics shared by the planner
// and the integrand kernels.
//
// Everything that decides *which* elements, fine phases and phase points take
// part (spot masks, visibility, ring drop, phase-bin assignment) runs in FP64
// with the reference CPU's expressions (cpu/devarshi24st_cpu.cpp:90-241,
// cpu/grid.hpp:158-250); only the atmosphere interpolation and the per-energy
// accumulation run in FP32.
#pragma once

#include <cstdint>

namespace ppm {

constexpr int kMaxSpots = 2;
// doubles per fine phase k in DevProfile::fine: cos(2 pi k / n_fine), sin(2 pi k / n_fine), k / n_fine
constexpr int kFineStride = 3;
// per-profile counters: active (integrated rings), rings, dropped rings, points, clamped, active (dropped rings)
constexpr int kStats = 6;

// ---- resident tables -------------------------------------------------------
struct DevLens {
  double u_min, u_max, cp_min, cp_max, ca_min, ca_max;
  int n_u, n_cp, n_ca;
  const double* ca;   // [n_u][n_cp]  cos alpha(u, cos psi)
  const double* lf;   // [n_u][n_cp]  lensing factor
  const double* cdt;  // [n_u][n_ca]  c dt / R (u, cos alpha)
};

struct DevNsx {
  int nT, ng, nE, nmu;
  int slice_stride;  // floats between (logT, logg) slices, multiple of 4 (16-byte aligned)
  double T_min, T_max, g_min, g_max, E_min, E_max;
  double inv_dE;       // (nE - 1) / (E_max - E_min): t = (logEkT - E_min) * inv_dE
  const float* data;   // [nT][ng][slice_stride] with slice [nE][nmu], values 10^logInuT3 * 2^scale_exp
  const double* mu;    // [nmu] strictly descending
  const double* mu_den;  // [nmu - 3][4] reciprocals of the cubic Lagrange denominators per stencil start
  int scale_exp;       // power of two applied to the stored FP32 values
};

// An observed-energy grid, with the per-energy split of t_E = log10(E) * inv_dE
// into a relative cell index and a fraction (NSX) plus 1/E.
struct DevGrid {
  int n_e;
  int iE_min;  // min_e floor(t_E)
  int span;    // max_e floor(t_E) - iE_min + 1; a point needs span + 1 cells
  double tE_lo, tE_hi;  // min / max of t_E
  const double* E;
  const double* invE;
  const int* rE;    // floor(t_E) - iE_min
  const float* fE;  // t_E - floor(t_E)
  // energies grouped by home cell rE (ascending t_E): the energies of home cell r
  // are perm[cell_first[r] .. cell_first[r + 1]), their fractions fEs[same range]
  const int* perm;        // [n_e] energy index in t_E order
  const float* fEs;       // [n_e] fE in t_E order
  const int* cell_first;  // [span + 1]
  int maxe;               // most energies in one home cell
};

struct DevSpot {
  double s1, c1, ph1, cos_ar1;  // disk 1: sin/cos colatitude, azimuth, cos(angular radius)
  double s2, c2, ph2, cos_ar2;  // disk 2 (excluded)
  double cos_theta_pt, dOmega_pt;
  double kT;           // keV
  double l10kT;        // log10(kT)
  double out_scale;    // per-spot factor applied when partial sums are flushed
  int kind;            // PPM_SPOT_*
  int i_lo, i_hi;      // HEALPix ring range that can hold active elements
  int T_clamped;       // logT outside the NSX axis
  int nT_taps;         // 2 (linear logT) or 4 (cubic logT)
  int iT[4];
  double wT[4];
};

struct DevProfile {
  // star (cpu/devarshi24st_cpu.cpp:48-124)
  double Re, Rs, nu, o2, D2, cos_obs, sin_obs, dOmega_hp;
  double Ob2, Ob4, Ob6, ce, cp, de, fe, dp, fp, d60, logg_base;  // logg_base = logg0 + log10(GM)
  int n_side, n_bins, n_gl, n_fine, n_spots, atmosphere, interp, beaming, precision, n_e;
  long long flux_off;   // doubles into the flux pool
  const double* ring;   // [4 n_side] (z, cos(acos z), sin(acos z)) per ring index i (entry 0 unused)
  const double* fine;   // [n_fine][kFineStride] (cos 2 pi k/n, sin 2 pi k/n, k/n)
  DevGrid grid;
  unsigned long long* stats;  // [kStats]
  unsigned* ring_seen;        // [kMaxSpots][ring_words] bits: rings already counted in stats[1]
  int ring_words;
  DevSpot spot[kMaxSpots];
};

// One unit of work: candidate elements j in [j0, j1) of one ring of one spot,
// at the phase nodes u in [u0, u1) (u = bin * max(n_gl, 1) + GL point).
struct Tile {
  int profile;
  short spot;
  short first;  // 1 for the first chunk of a ring
  int ring;     // HEALPix ring index (1..4N-1), 0 for a point source
  int j0, j1;
  short u0, u1;
};

// Adds v to *a with a compensated (TwoSum) accumulation: the atomic returns the
// old value, so the rounding error of old + v is known exactly and is added to
// the compensation pool *c.  *a + *c is then the sum of every value added, to
// within a rounding of the compensation itself (about 1e-32 relative), in any
// order of the additions.  Without a pool (c == nullptr) a plain atomic add.
__device__ __forceinline__ void comp_add(double* a, double* c, double v) {
  if (!c) {
    atomicAdd(a, v);
    return;
  }
  const double old = atomicAdd(a, v);
  const double s = old + v;
  const double bb = s - old;
  const double err = (old - (s - bb)) + (v - bb);
  if (err != 0.0) atomicAdd(c, err);
}

struct WorkQueue {
  Tile* tiles;
  int capacity;
  int* n_tiles;    // written by the planner
  int* next;       // pulled by the persistent integrand
  int* overflow;   // set if the planner ran out of capacity
};

// ---- helpers ----------------------------------------------------------------
__host__ __device__ __forceinline__ int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// UniformHunt::operator() (cpu/hunt.hpp:98-121): clamps x to the grid.
__device__ __forceinline__ int uhunt(double& x, double lo, double hi, int n, double& a) {
  if (x <= lo) {
    a = 0.0;
    x = lo;
    return 0;
  }
  if (x >= hi) {
    a = 1.0;
    x = hi;
    return n - 2;
  }
  double t = (x - lo) / (hi - lo) * (n - 1);
  int i = (int)t;
  a = t - i;
  return i;
}

// VecHunt::operator() on a strictly monotone table (cpu/hunt.hpp:14-66):
// bracket with index clamped to [0, n-2] and extrapolated fraction.
__host__ __device__ __forceinline__ int vhunt(const double* xx, int n, double x, double& a) {
  bool ascnd = xx[n - 1] >= xx[0];
  int jl = -1, ju = n;
  while (ju - jl > 1) {
    int jm = (ju + jl) >> 1;
    if ((x >= xx[jm]) == ascnd)
      jl = jm;
    else
      ju = jm;
  }
  int i = clampi(jl, 0, n - 2);
  a = (x - xx[i]) / (xx[i + 1] - xx[i]);
  return i;
}

// Largest j in [-1, n-1] with xx[j] <= x for a non-decreasing xx (xx[-1] taken
// as -inf), searched from `jl`, a previous answer, by doubling steps and then
// bisection: the same index vhunt's bisection finds on such an array, in O(1)
// steps for successive nearby x.
__host__ __device__ __forceinline__ int hunt_from(const double* xx, int n, double x, int jl) {
  int lo, hi;  // xx[lo] <= x < xx[hi], with xx[-1] = -inf and xx[n] = +inf
  if (jl < 0 || x >= xx[jl]) {
    lo = jl;
    int step = 1;
    hi = lo + 1;
    while (hi < n && x >= xx[hi]) {
      lo = hi;
      step <<= 1;
      hi = lo + step;
    }
    if (hi > n) hi = n;
  } else {
    hi = jl;
    int step = 1;
    lo = hi - 1;
    while (lo >= 0 && x < xx[lo]) {
      hi = lo;
      step <<= 1;
      lo = hi - step;
    }
    if (lo < -1) lo = -1;
  }
  while (hi - lo > 1) {
    const int m = (lo + hi) >> 1;
    if (x >= xx[m])
      lo = m;
    else
      hi = m;
  }
  return lo;
}

// vhunt's clamped bracket on a non-decreasing xx (the largest i <= n - 2 with
// xx[i] <= x, or 0) by unit steps from any i in [0, n - 2]: a step or none
// when i is the bracket of a nearby x.
__host__ __device__ __forceinline__ int walk_bracket(const double* xx, int n, double x, int i) {
  while (i > 0 && x < xx[i]) --i;
  while (i < n - 2 && x >= xx[i + 1]) ++i;
  return i;
}

// cpu/nsx.hpp:159-168
__device__ __forceinline__ void cubic_lagrange(double w[4], double x, double x0, double x1, double x2, double x3) {
  w[0] = (x - x1) * (x - x2) * (x - x3) / ((x0 - x1) * (x0 - x2) * (x0 - x3));
  w[1] = (x - x0) * (x - x2) * (x - x3) / ((x1 - x0) * (x1 - x2) * (x1 - x3));
  w[2] = (x - x0) * (x - x1) * (x - x3) / ((x2 - x0) * (x2 - x1) * (x2 - x3));
  w[3] = (x - x0) * (x - x1) * (x - x2) / ((x3 - x0) * (x3 - x1) * (x3 - x2));
}

__device__ __forceinline__ double uhunt_at(double lo, double hi, int n, int i) { return lo + (hi - lo) * i / (n - 1); }

// HEALPix azimuth of element j in ring i, phi = dphi * (j - jofs)
// (cpu/grid.hpp:219-244, gpu/healpix.cuh:74-91): the per-ring factors, so that
// a loop over the elements of one ring evaluates the same expression.
struct RingPhi {
  double dphi, jofs;
};
__device__ __forceinline__ RingPhi healpix_ring_phi(int N, int i) {
  if (i > 2 * N) i = 4 * N - i;
  if (i < N) {
    double s = 1.;
    return RingPhi{3.14159265358979323846 / (2. * i), s / 2.};
  }
  double s = (i - N + 1) % 2;
  return RingPhi{3.14159265358979323846 / (2. * N), s / 2.};
}
__device__ __forceinline__ double healpix_phi(int N, int i, int j) {
  const RingPhi r = healpix_ring_phi(N, i);
  return r.dphi * (j - r.jofs);
}

__device__ __forceinline__ int healpix_jmax(int N, int i) {
  int m = i < 4 * N - i ? i : 4 * N - i;
  if (N < m) m = N;
  return 4 * m;
}

// DiskDifference (cpu/grid.hpp:158-190) with the ring's cos/sin of acos(z).
__device__ __forceinline__ bool in_spot(const DevSpot& s, double c2, double s2, double phi) {
  double cr1 = s.s1 * s2 * cos(phi - s.ph1) + s.c1 * c2;
  if (!(cr1 > s.cos_ar1)) return false;
  double cr2 = s.s2 * s2 * cos(phi - s.ph2) + s.c2 * c2;
  return !(cr2 > s.cos_ar2);
}

// Per-ring oblate geometry (cpu/devarshi24st_cpu.cpp:90-124).
struct RingGeom {
  double cos_t, sin_t, R, u, uu, dS, cos_tau, sin_tau, logg;
  double beta, gamma, dt2;  // the sweep's ring terms: surface speed / c, Lorentz factor, surface-to-R_eq delay
  int i_u;
  double a_u;
  bool u_clamped;
};

__device__ inline void ring_geometry(const DevProfile& p, const DevLens& L, double cos_t, double dOmega, bool need_logg,
                                     RingGeom& g) {
  g.cos_t = cos_t;
  g.sin_t = sqrt(1. - cos_t * cos_t);
  g.R = p.Re * (1. + p.o2 * cos_t * cos_t);
  double dRdtheta = -2. * p.Re * p.o2 * cos_t * g.sin_t;
  g.u = p.Rs / g.R;
  g.uu = sqrt(1. - g.u);
  double f = dRdtheta / (g.R * g.uu);
  double ff = sqrt(1. + f * f);
  g.dS = g.R * g.R * dOmega * ff;
  g.cos_tau = 1. / ff;
  g.sin_tau = f / ff;
  // the terms of every fine-phase sample that depend on the ring only (cpu/devarshi24st_cpu.cpp:153-154,
  // :162-170), computed once here with the sweep's own expressions
  {
    const double two_pi = 2. * 3.14159265358979323846;
    const double c_in_km_s = 299792458. / 1e3;
    g.beta = two_pi * p.nu * g.R * g.sin_t / g.uu / c_in_km_s;
    g.gamma = 1. / sqrt(1. - g.beta * g.beta);
    g.dt2 = (p.Re - g.R + p.Rs * log1p((p.Re - g.R) / (g.R - p.Rs))) / c_in_km_s;
  }
  double uc = g.u;
  g.u_clamped = (uc < L.u_min) || (uc > L.u_max);
  g.i_u = uhunt(uc, L.u_min, L.u_max, L.n_u, g.a_u);
  g.logg = 0.0;
  if (need_logg) {
    double sc2 = cos_t * cos_t, ss2 = g.sin_t * g.sin_t;
    double g_g0 = 1. + ss2 * (p.ce * p.Ob2 + p.de * p.Ob4 + p.fe * p.Ob6) +
                  sc2 * (p.cp * p.Ob2 + p.dp * p.Ob4 + p.fp * p.Ob6 - p.d60 * p.Ob4) + fabs(cos_t) * p.d60 * p.Ob4;
    g.logg = log10(g_g0) + p.logg_base;
  }
}

// Two rows (i_u, i_u + 1) of each lensing table; rows may live in shared or global memory.
struct LensRows {
  const double *ca0, *ca1, *lf0, *lf1, *cdt0, *cdt1;
};

__device__ __forceinline__ void lens_rows_global(const DevLens& L, int i_u, LensRows& r) {
  r.ca0 = L.ca + (size_t)i_u * L.n_cp;
  r.ca1 = r.ca0 + L.n_cp;
  r.lf0 = L.lf + (size_t)i_u * L.n_cp;
  r.lf1 = r.lf0 + L.n_cp;
  r.cdt0 = L.cdt + (size_t)i_u * L.n_ca;
  r.cdt1 = r.cdt0 + L.n_ca;
}

// One fine-phase sample of the sweep (cpu/devarshi24st_cpu.cpp:128-192).
// Writes flux/I without the 1/D^2 factor (applied at flush), the redshift
// factor, the observed phase and cos sigma'; returns false if invisible.
__device__ inline bool sweep_sample(const DevProfile& p, const DevLens& L, const RingGeom& g, const LensRows& rows,
                                    int i_phase, bool nsx, double& F, double& Z, double& P, double& MU) {
  const double two_pi = 2. * 3.14159265358979323846;
  const double c_in_km_s = 299792458. / 1e3;
  double phase = p.fine[kFineStride * i_phase + 2];  // 1. * i_phase / n_fine, divided on the host
  double cos_spot_phi = p.fine[kFineStride * i_phase];
  double sin_spot_phi = p.fine[kFineStride * i_phase + 1];
  double cos_psi = p.cos_obs * g.cos_t + p.sin_obs * g.sin_t * cos_spot_phi;
  if (cos_psi < L.cp_min) return false;
  double sin_psi = sqrt(1. - cos_psi * cos_psi);
  double a_u = g.a_u, b_u = 1. - a_u;
  double a_cp, xcp = cos_psi;
  int i_cp = uhunt(xcp, L.cp_min, L.cp_max, L.n_cp, a_cp);
  double b_cp = 1. - a_cp;
  double cos_alpha = b_u * b_cp * rows.ca0[i_cp] + a_u * b_cp * rows.ca1[i_cp] + b_u * a_cp * rows.ca0[i_cp + 1] +
                     a_u * a_cp * rows.ca1[i_cp + 1];
  double lf = b_u * b_cp * rows.lf0[i_cp] + a_u * b_cp * rows.lf1[i_cp] + b_u * a_cp * rows.lf0[i_cp + 1] +
              a_u * a_cp * rows.lf1[i_cp + 1];
  double sin_alpha = sqrt(1. - cos_alpha * cos_alpha);
  double saosp = cos_psi == 1. ? sqrt(lf) : sin_alpha / sin_psi;
  double cos_sigma = cos_alpha * g.cos_tau +
                     saosp * g.sin_tau * (p.cos_obs * g.sin_t - p.sin_obs * g.cos_t * cos_spot_phi);
  if (cos_sigma <= 0) return false;
  const double beta = g.beta, gamma = g.gamma;
  double cos_xi = -saosp * p.sin_obs * sin_spot_phi;
  double delta = 1. / (gamma * (1. - beta * cos_xi));
  double delta3 = delta * delta * delta;
  double a_ca, xca = cos_alpha;
  int i_ca = uhunt(xca, L.ca_min, L.ca_max, L.n_ca, a_ca);
  double b_ca = 1. - a_ca;
  double cdt_over_R = b_u * b_ca * rows.cdt0[i_ca] + a_u * b_ca * rows.cdt1[i_ca] + b_u * a_ca * rows.cdt0[i_ca + 1] +
                      a_u * a_ca * rows.cdt1[i_ca + 1];
  double dt1 = cdt_over_R * g.R / c_in_km_s;
  double Re = p.Re, Rs = p.Rs;
  double dt2 = g.dt2;
  if (!(cos_alpha >= 0)) {
    double tmp = (2. * sin_alpha) / sqrt(3. * (1. - g.u));
    double p_over_R = -tmp * cos((acos(3. * g.u / tmp) + 2. * 3.14159265358979323846) / 3.);
    double pp = p_over_R * g.R;
    double dt2p = (Re - pp + Rs * log1p((Re - pp) / (pp - Rs))) / c_in_km_s;
    dt2 = 2. * dt2p - dt2;
  }
  double delta_phase = (dt1 + dt2) * p.nu;
  double csp = cos_sigma * delta;
  double beaming = 1.0;
  if (!nsx) {
    if (p.beaming == 1)
      beaming = 1. - csp * csp;
    else if (p.beaming == 2)
      beaming = csp * csp;
  }
  F = g.uu * delta3 * csp * lf * (g.dS * gamma) * beaming;
  Z = 1. / (delta * g.uu);
  P = phase + delta_phase;
  MU = csp;
  return true;
}

// Gauss-Legendre nodes and weights on [-1, 1], N = 1..6 (cpu/gl.hpp:5-62).
__constant__ double c_gl_nodes[21] = {
    0.0,
    -0.5773502691896257645091488, 0.5773502691896257645091488,
    -0.7745966692414833770358531, 0.0, 0.7745966692414833770358531,
    -0.8611363115940525752239465, -0.3399810435848562648026658, 0.3399810435848562648026658,
    0.8611363115940525752239465,
    -0.9061798459386639927976269, -0.5384693101056830910363144, 0.0, 0.5384693101056830910363144,
    0.9061798459386639927976269,
    -0.9324695142031520278123016, -0.6612093864662645136613996, -0.2386191860831969086305017,
    0.2386191860831969086305017, 0.6612093864662645136613996, 0.9324695142031520278123016};
__constant__ double c_gl_weights[21] = {
    2.0,
    1.0, 1.0,
    0.5555555555555555555555556, 0.8888888888888888888888889, 0.5555555555555555555555556,
    0.3478548451374538573730639, 0.6521451548625461426269361, 0.6521451548625461426269361,
    0.3478548451374538573730639,
    0.2369268850561890875142640, 0.4786286704993664680412915, 0.5688888888888888888888889,
    0.4786286704993664680412915, 0.2369268850561890875142640,
    0.1713244923791703450402961, 0.3607615730481386075698335, 0.4679139345726910473898703,
    0.4679139345726910473898703, 0.3607615730481386075698335, 0.1713244923791703450402961};

}  // namespace ppm
