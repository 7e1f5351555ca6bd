// Lensing-table generator: Schwarzschild light-bending and time-delay
// integrals on the (u, cos psi) and (u, cos alpha) grids.
//
// Restates the algorithm of c_lensing.py (fizban007/gpu_ppm):
//   * psi(u, alpha) = 2 sin(a)/sqrt(1-u) * int_0^1 f dx          c_lensing.py:47-61
//     with the turning-point branch for alpha > pi/2              c_lensing.py:64-77
//   * march alpha from 0 by d_alpha = pi/(8 N_cos_psi) until psi
//     exceeds arccos(cos_psi_min)                                  c_lensing.py:32,84-93
//   * lensing factor = d cos(alpha) / d cos(psi) by numpy.gradient c_lensing.py:100
//   * PCHIP resampling onto the cos psi grid                       c_lensing.py:102-106
//   * c dt / R (u, alpha) = 2 sin^2/(1-u) * int_0^1 g dx            c_lensing.py:115-154
// scipy's QUADPACK is replaced by adaptive Gauss-Legendre bisection to a
// relative tolerance of 1e-12 (tables agree with the Python script to the
// script's own quadrature tolerance, 1.49e-8); numpy.gradient (edge_order=1,
// non-uniform spacing) and scipy's PchipInterpolator derivative rules are
// restated exactly.
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/ppm.h"
#include "common.h"

namespace {

constexpr double kPi = 3.14159265358979323846;

struct GaussLegendre {
  static constexpr int N = 10;
  double x[N], w[N];
  GaussLegendre() {
    // Newton iteration on P_N for the nodes on [-1, 1].
    for (int i = 0; i < N; ++i) {
      double z = std::cos(kPi * (i + 0.75) / (N + 0.5)), pp = 1.0;
      for (int it = 0; it < 64; ++it) {
        double p1 = 1.0, p2 = 0.0;
        for (int j = 1; j <= N; ++j) {
          double p3 = p2;
          p2 = p1;
          p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
        }
        pp = N * (z * p1 - p2) / (z * z - 1.0);
        double dz = p1 / pp;
        z -= dz;
        if (std::fabs(dz) < 1e-15) break;
      }
      double p1 = 1.0, p2 = 0.0;
      for (int j = 1; j <= N; ++j) {
        double p3 = p2;
        p2 = p1;
        p1 = ((2.0 * j - 1.0) * z * p2 - (j - 1.0) * p3) / j;
      }
      pp = N * (z * p1 - p2) / (z * z - 1.0);
      x[i] = z;
      w[i] = 2.0 / ((1.0 - z * z) * pp * pp);
    }
  }
};

const GaussLegendre& gl() {
  static GaussLegendre g;
  return g;
}

template <class F>
double gl_segment(F const& f, double a, double b) {
  const GaussLegendre& g = gl();
  double c = 0.5 * (a + b), h = 0.5 * (b - a), s = 0.0;
  for (int i = 0; i < GaussLegendre::N; ++i) s += g.w[i] * f(c + h * g.x[i]);
  return s * h;
}

// Bisection until the two halves agree with the whole to `tol` (halved per
// level) or to round-off of the segment (floor 4e-16 |segment|), whichever is
// looser; `budget` bounds the total number of segment pairs.
template <class F>
double adapt(F const& f, double a, double b, double whole, double tol, int depth, int* budget) {
  double m = 0.5 * (a + b);
  double l = gl_segment(f, a, m), r = gl_segment(f, m, b);
  double both = l + r;
  double floor_tol = 4e-16 * (std::fabs(l) + std::fabs(r));
  if (depth <= 0 || --*budget <= 0 || std::fabs(both - whole) <= (tol > floor_tol ? tol : floor_tol)) return both;
  return adapt(f, a, m, l, 0.5 * tol, depth - 1, budget) + adapt(f, m, b, r, 0.5 * tol, depth - 1, budget);
}

template <class F>
double integrate01(F const& f) {
  double whole = gl_segment(f, 0.0, 1.0);
  double tol = 1e-12 * std::fabs(whole) + 1e-300;
  int budget = 4096;
  return adapt(f, 0.0, 1.0, whole, tol, 40, &budget);
}

// c_lensing.py:47-54 (f) and 115-122 (g); s2 = sin^2(alpha), c2 = 1 - s2.
inline double qfac(double x, double u, double s2) {
  double x2 = x * x;
  double t = 1.0 - x2;
  return (2.0 - x2 - u * t * t / (1.0 - u)) * s2;
}

double psi1(double u, double alpha) {
  double s = std::sin(alpha);
  double s2 = s * s, c2 = 1.0 - s2;
  auto f = [&](double x) { return x / std::sqrt(c2 + x * x * qfac(x, u, s2)); };
  return 2.0 * s / std::sqrt(1.0 - u) * integrate01(f);
}

double turning_point_p_over_R(double u, double alpha) {
  double s = std::sin(alpha);
  double tmp = (2.0 * s) / std::sqrt(3.0 * (1.0 - u));
  return -tmp * std::cos((std::acos(3.0 * u / tmp) + 2.0 * kPi) / 3.0);
}

double psi_of(double u, double alpha) {
  if (alpha <= kPi / 2) return psi1(u, alpha);
  double p_over_R = turning_point_p_over_R(u, alpha);
  double psi_max = psi1(u / p_over_R, kPi / 2);
  return 2.0 * psi_max - psi1(u, kPi - alpha);
}

double cdt1(double u, double alpha) {
  double s = std::sin(alpha);
  double s2 = s * s, c2 = 1.0 - s2;
  auto g = [&](double x) {
    double t = std::sqrt(c2 + x * x * qfac(x, u, s2));
    return x / (t * (1.0 + t));
  };
  return 2.0 * s * s / (1.0 - u) * integrate01(g);
}

double cdt_of(double u, double alpha) {
  if (alpha <= kPi / 2) return cdt1(u, alpha);
  double p_over_R = turning_point_p_over_R(u, alpha);
  double dt_max = cdt1(u / p_over_R, kPi / 2);
  return 2.0 * dt_max - cdt1(u, kPi - alpha);
}

// numpy.gradient(f, x) with non-uniform x, edge_order=1.
void np_gradient(const std::vector<double>& f, const std::vector<double>& x, std::vector<double>& out) {
  size_t n = f.size();
  out.assign(n, 0.0);
  if (n < 2) return;
  for (size_t i = 1; i + 1 < n; ++i) {
    double dx1 = x[i] - x[i - 1], dx2 = x[i + 1] - x[i];
    double a = -dx2 / (dx1 * (dx1 + dx2));
    double b = (dx2 - dx1) / (dx1 * dx2);
    double c = dx1 / (dx2 * (dx1 + dx2));
    out[i] = a * f[i - 1] + b * f[i] + c * f[i + 1];
  }
  out[0] = (f[1] - f[0]) / (x[1] - x[0]);
  out[n - 1] = (f[n - 1] - f[n - 2]) / (x[n - 1] - x[n - 2]);
}

inline double sgn(double v) { return (v > 0) - (v < 0); }

// scipy.interpolate.PchipInterpolator endpoint rule.
double pchip_edge(double h0, double h1, double m0, double m1) {
  double d = ((2.0 * h0 + h1) * m0 - h0 * m1) / (h0 + h1);
  if (sgn(d) != sgn(m0)) return 0.0;
  if (sgn(m0) != sgn(m1) && std::fabs(d) > 3.0 * std::fabs(m0)) return 3.0 * m0;
  return d;
}

// PCHIP through (x, y), x strictly increasing, evaluated at xq.
void pchip_eval(const std::vector<double>& x, const std::vector<double>& y, const double* xq, int nq, double* out) {
  size_t n = x.size();
  std::vector<double> h(n - 1), m(n - 1), d(n, 0.0);
  for (size_t k = 0; k + 1 < n; ++k) {
    h[k] = x[k + 1] - x[k];
    m[k] = (y[k + 1] - y[k]) / h[k];
  }
  if (n == 2) {
    d[0] = d[1] = m[0];
  } else {
    for (size_t k = 1; k + 1 < n; ++k) {
      bool cond = (sgn(m[k]) != sgn(m[k - 1])) || m[k] == 0.0 || m[k - 1] == 0.0;
      if (cond) {
        d[k] = 0.0;
      } else {
        double w1 = 2.0 * h[k] + h[k - 1];
        double w2 = h[k] + 2.0 * h[k - 1];
        double whmean = (w1 / m[k - 1] + w2 / m[k]) / (w1 + w2);
        d[k] = 1.0 / whmean;
      }
    }
    d[0] = pchip_edge(h[0], h[1], m[0], m[1]);
    d[n - 1] = pchip_edge(h[n - 2], h[n - 3], m[n - 2], m[n - 3]);
  }
  for (int q = 0; q < nq; ++q) {
    double xv = xq[q];
    // interval k with x[k] <= xv < x[k+1]; clamp to the end intervals (extrapolate)
    size_t lo = 0, hi = n - 1;
    if (xv <= x[0]) {
      lo = 0;
    } else if (xv >= x[n - 1]) {
      lo = n - 2;
    } else {
      while (hi - lo > 1) {
        size_t mid = (lo + hi) / 2;
        if (x[mid] <= xv)
          lo = mid;
        else
          hi = mid;
      }
    }
    size_t k = lo;
    double t = (d[k] + d[k + 1] - 2.0 * m[k]) / h[k];
    double c0 = t / h[k];
    double c1 = (m[k] - d[k]) / h[k] - t;
    double c2 = d[k];
    double c3 = y[k];
    double s = xv - x[k];
    out[q] = ((c0 * s + c1) * s + c2) * s + c3;
  }
}

std::vector<double> linspace(double a, double b, int n) {
  std::vector<double> v(n);
  if (n == 1) {
    v[0] = a;
    return v;
  }
  // numpy.linspace: a + i*step, last element set to b exactly
  double step = (b - a) / (n - 1);
  for (int i = 0; i < n; ++i) v[i] = a + i * step;
  v[n - 1] = b;
  return v;
}

// One u-row of the (u, cos psi) tables; returns false on a non-finite march.
bool psi_row(double u, double d_alpha, double psi_stop, const std::vector<double>& out_cos_psi, double* ca_row,
             double* lf_row) {
  std::vector<double> alpha_grid, psi_grid;
  double alpha = 0.0;
  for (int guard = 0; guard < 1 << 22; ++guard) {
    double psi = psi_of(u, alpha);
    if (!std::isfinite(psi)) return false;
    alpha_grid.push_back(alpha);
    psi_grid.push_back(psi);
    alpha += d_alpha;
    if (psi > psi_stop) break;
    if (alpha > kPi) return false;
  }
  size_t n = alpha_grid.size();
  std::vector<double> cos_a(n), cos_p(n), lf;
  for (size_t i = 0; i < n; ++i) {
    cos_a[i] = std::cos(alpha_grid[i]);
    cos_p[i] = std::cos(psi_grid[i]);
  }
  np_gradient(cos_a, cos_p, lf);
  std::vector<double> xr(n), yr(n), lr(n);
  for (size_t i = 0; i < n; ++i) {
    xr[i] = cos_p[n - 1 - i];
    yr[i] = cos_a[n - 1 - i];
    lr[i] = lf[n - 1 - i];
  }
  pchip_eval(xr, yr, out_cos_psi.data(), (int)out_cos_psi.size(), ca_row);
  pchip_eval(xr, lr, out_cos_psi.data(), (int)out_cos_psi.size(), lf_row);
  return true;
}

}  // namespace

extern "C" int ppm_lensing_generate(const ppm_lensing_spec* spec, double* ca, double* lf, double* cdt) {
  if (!spec || !ca || !lf || !cdt) return ppm::set_error(PPM_E_INVALID, "ppm_lensing_generate: null argument");
  if (spec->n_u < 2 || spec->n_cos_psi < 2 || spec->n_cos_alpha < 2)
    return ppm::set_error(PPM_E_INVALID, "ppm_lensing_generate: every grid needs at least 2 points");
  if (!(spec->u_min > 0.0 && spec->u_max < 2.0 / 3.0 && spec->u_min < spec->u_max))
    return ppm::set_error(PPM_E_RANGE, "ppm_lensing_generate: u range must lie inside (0, 2/3)");
  if (!(spec->cos_psi_min > -1.0 && spec->cos_psi_max <= 1.0 && spec->cos_alpha_min > -1.0 &&
        spec->cos_alpha_max <= 1.0))
    return ppm::set_error(PPM_E_RANGE, "ppm_lensing_generate: cos ranges must lie inside (-1, 1]");

  const int nu = spec->n_u, np_ = spec->n_cos_psi, na = spec->n_cos_alpha;
  std::vector<double> u_grid = linspace(spec->u_min, spec->u_max, nu);
  std::vector<double> cpsi = linspace(spec->cos_psi_min, spec->cos_psi_max, np_);
  std::vector<double> calpha = linspace(spec->cos_alpha_min, spec->cos_alpha_max, na);
  const double d_alpha = kPi / (np_ * 8.0);
  const double psi_stop = std::acos(cpsi[0]);

  int nth = spec->n_threads > 0 ? spec->n_threads : (int)std::thread::hardware_concurrency();
  if (nth < 1) nth = 1;
  std::vector<int> bad(nu, 0);
  auto work = [&](int t) {
    for (int iu = t; iu < nu; iu += nth) {
      double u = u_grid[iu];
      if (!psi_row(u, d_alpha, psi_stop, cpsi, ca + (size_t)iu * np_, lf + (size_t)iu * np_)) bad[iu] = 1;
      for (int k = 0; k < na; ++k) {
        double v = cdt_of(u, std::acos(calpha[k]));
        if (!std::isfinite(v)) bad[iu] = 1;
        cdt[(size_t)iu * na + k] = v;
      }
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < nth; ++t) pool.emplace_back(work, t);
  work(0);
  for (auto& th : pool) th.join();
  for (int iu = 0; iu < nu; ++iu)
    if (bad[iu])
      return ppm::set_error(PPM_E_RANGE, "ppm_lensing_generate: non-finite ray integral at u=" +
                                             std::to_string(u_grid[iu]) +
                                             " (turning-point branch undefined; lower u_max or raise cos_alpha_min)");
  return PPM_OK;
}
