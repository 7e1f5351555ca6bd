// Instrument-response preparation (c_ism_inst.py): the RMF x ARF x ISM
// response on the instrument's fine energy bins, integrated over each fine bin
// against the cubic splines through the unit vectors of the observed-energy
// grid, so that rsp[ch][i] multiplies the flux at E_obs[i].
//
// The splines are the not-a-knot cubic splines of scipy.interpolate.CubicSpline
// (the reference's dependency, c_ism_inst.py:2): slopes from the tridiagonal
// system of the C1 and C2 continuity conditions with the not-a-knot end rows,
// a parabola for three knots and a line for two, the end pieces extrapolated.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/ppm.h"
#include "common.h"
#include "engine.h"

namespace ppm {
namespace {

// Piecewise cubic y = c3 t^3 + c2 t^2 + c1 t + c0, t = x - x[i] on [x[i], x[i+1]].
struct Spline {
  std::vector<double> x, c0, c1, c2, c3, F;  // F[i]: integral from x[0] to x[i]
};

Spline not_a_knot_spline(const std::vector<double>& x, const std::vector<double>& y) {
  const int n = (int)x.size();
  if (n < 2) throw Error(PPM_E_INVALID, "a cubic spline needs at least two knots");
  std::vector<double> dx(n - 1), slope(n - 1);
  for (int i = 0; i + 1 < n; ++i) {
    dx[i] = x[i + 1] - x[i];
    if (!(dx[i] > 0)) throw Error(PPM_E_INVALID, "spline knots must be strictly increasing");
    slope[i] = (y[i + 1] - y[i]) / dx[i];
  }
  std::vector<double> s(n);  // slopes at the knots
  if (n == 2) {
    s[0] = s[1] = slope[0];
  } else if (n == 3) {
    // the parabola through the three knots
    double A[3][3] = {{1, 1, 0}, {dx[1], 2 * (dx[0] + dx[1]), dx[0]}, {0, 1, 1}};
    double b[3] = {2 * slope[0], 3 * (dx[0] * slope[1] + dx[1] * slope[0]), 2 * slope[1]};
    for (int c = 0; c < 3; ++c) {  // Gaussian elimination with partial pivoting
      int piv = c;
      for (int r = c + 1; r < 3; ++r)
        if (std::fabs(A[r][c]) > std::fabs(A[piv][c])) piv = r;
      for (int k = 0; k < 3; ++k) std::swap(A[c][k], A[piv][k]);
      std::swap(b[c], b[piv]);
      for (int r = c + 1; r < 3; ++r) {
        const double f = A[r][c] / A[c][c];
        for (int k = c; k < 3; ++k) A[r][k] -= f * A[c][k];
        b[r] -= f * b[c];
      }
    }
    for (int r = 2; r >= 0; --r) {
      double v = b[r];
      for (int k = r + 1; k < 3; ++k) v -= A[r][k] * s[k];
      s[r] = v / A[r][r];
    }
  } else {
    // tridiagonal system: lower l, diagonal d, upper u, right-hand side b
    std::vector<double> l(n, 0), d(n, 0), u(n, 0), b(n, 0);
    for (int i = 1; i + 1 < n; ++i) {
      l[i] = dx[i];
      d[i] = 2 * (dx[i - 1] + dx[i]);
      u[i] = dx[i - 1];
      b[i] = 3 * (dx[i] * slope[i - 1] + dx[i - 1] * slope[i]);
    }
    {  // not-a-knot at the start: third derivative continuous at x[1]
      const double dd = x[2] - x[0];
      d[0] = dx[1];
      u[0] = dd;
      b[0] = ((dx[0] + 2 * dd) * dx[1] * slope[0] + dx[0] * dx[0] * slope[1]) / dd;
    }
    {  // and at the end, at x[n-2]
      const double dd = x[n - 1] - x[n - 3];
      d[n - 1] = dx[n - 3];
      l[n - 1] = dd;
      b[n - 1] = (dx[n - 2] * dx[n - 2] * slope[n - 3] + (2 * dd + dx[n - 2]) * dx[n - 3] * slope[n - 2]) / dd;
    }
    // Thomas algorithm
    for (int i = 1; i < n; ++i) {
      const double f = l[i] / d[i - 1];
      d[i] -= f * u[i - 1];
      b[i] -= f * b[i - 1];
    }
    s[n - 1] = b[n - 1] / d[n - 1];
    for (int i = n - 2; i >= 0; --i) s[i] = (b[i] - u[i] * s[i + 1]) / d[i];
  }
  Spline sp;
  sp.x = x;
  sp.c0.resize(n - 1);
  sp.c1.resize(n - 1);
  sp.c2.resize(n - 1);
  sp.c3.resize(n - 1);
  sp.F.assign(n, 0.0);
  for (int i = 0; i + 1 < n; ++i) {
    const double t = (s[i] + s[i + 1] - 2 * slope[i]) / dx[i];
    sp.c3[i] = t / dx[i];
    sp.c2[i] = (slope[i] - s[i]) / dx[i] - t;
    sp.c1[i] = s[i];
    sp.c0[i] = y[i];
  }
  for (int i = 0; i + 1 < n; ++i) {
    const double h = dx[i];
    sp.F[i + 1] = sp.F[i] + h * (sp.c0[i] + h * (sp.c1[i] / 2 + h * (sp.c2[i] / 3 + h * sp.c3[i] / 4)));
  }
  return sp;
}

// piece holding xq: the last knot <= xq, clipped to the first and last pieces
int piece(const Spline& sp, double xq) {
  const int n = (int)sp.x.size();
  const int i = (int)(std::upper_bound(sp.x.begin(), sp.x.end(), xq) - sp.x.begin()) - 1;
  return std::min(std::max(i, 0), n - 2);
}

double spline_value(const Spline& sp, double xq) {
  const int i = piece(sp, xq);
  const double t = xq - sp.x[i];
  return sp.c0[i] + t * (sp.c1[i] + t * (sp.c2[i] + t * sp.c3[i]));
}

// antiderivative from x[0]
double spline_primitive(const Spline& sp, double xq) {
  const int i = piece(sp, xq);
  const double t = xq - sp.x[i];
  return sp.F[i] + t * (sp.c0[i] + t * (sp.c1[i] / 2 + t * (sp.c2[i] / 3 + t * sp.c3[i] / 4)));
}

// rsp[ch][i] = sum_j rmf[ch][j] area[j] ism[j] C[j][i] (c_ism_inst.py:59, 76-96)
void prepare(int n_ch, int n_fine, const double* rmf, const double* area, const double* e_lo, const double* e_hi,
             const double* ism, int n_obs, const double* e_obs, double* rsp) {
  if (n_ch < 1 || n_fine < 1 || n_obs < 2) throw Error(PPM_E_INVALID, "response sizes must be positive (n_obs >= 2)");
  if (!rmf || !area || !e_lo || !e_hi || !e_obs || !rsp) throw Error(PPM_E_INVALID, "null response array");
  // C[j][i]: the integral over fine bin j of the spline through the unit vector e_i (c_ism_inst.py:76-86)
  const std::vector<double> xc(e_obs, e_obs + n_obs);
  std::vector<double> C((size_t)n_fine * n_obs);
  std::vector<double> unit(n_obs, 0.0);
  for (int i = 0; i < n_obs; ++i) {
    unit[i] = 1.0;
    const Spline sp = not_a_knot_spline(xc, unit);
    unit[i] = 0.0;
    for (int j = 0; j < n_fine; ++j) C[(size_t)j * n_obs + i] = spline_primitive(sp, e_hi[j]) - spline_primitive(sp, e_lo[j]);
  }
  std::vector<double> row(n_fine);
  for (int ch = 0; ch < n_ch; ++ch) {
    for (int j = 0; j < n_fine; ++j) row[j] = rmf[(size_t)ch * n_fine + j] * area[j] * (ism ? ism[j] : 1.0);
    for (int i = 0; i < n_obs; ++i) {
      double acc = 0;
      for (int j = 0; j < n_fine; ++j) acc += row[j] * C[(size_t)j * n_obs + i];
      rsp[(size_t)ch * n_obs + i] = acc;
    }
  }
}

// numpy.loadtxt of the numeric lines after `skip` lines: rows of whitespace-separated values
std::vector<std::vector<double>> load_table(const std::string& path, int skip) {
  std::ifstream f(path);
  if (!f) throw Error(PPM_E_IO, "cannot open " + path);
  std::string line;
  for (int k = 0; k < skip && std::getline(f, line); ++k) {
  }
  std::vector<std::vector<double>> rows;
  while (std::getline(f, line)) {
    const size_t hash = line.find('#');
    if (hash != std::string::npos) line.resize(hash);
    std::istringstream ss(line);
    std::vector<double> r;
    double v;
    while (ss >> v) r.push_back(v);
    if (!ss.eof()) throw Error(PPM_E_IO, "non-numeric value in " + path);
    if (!r.empty()) rows.push_back(std::move(r));
  }
  if (rows.empty()) throw Error(PPM_E_IO, "no data rows in " + path);
  return rows;
}

void write_rows(const std::string& path, const double* v, size_t rows, size_t cols) {
  FILE* f = std::fopen(path.c_str(), "w");
  if (!f) throw Error(PPM_E_IO, "cannot write " + path);
  for (size_t r = 0; r < rows; ++r)
    for (size_t c = 0; c < cols; ++c) std::fprintf(f, "%.18e%c", v[r * cols + c], c + 1 == cols ? '\n' : ' ');
  if (std::fclose(f) != 0) throw Error(PPM_E_IO, "error writing " + path);
}

// c_ism_inst.py:30-101 with runtime settings
void prepare_files(const char* rmf_path, const char* arf_path, const char* ism_path, int i_e_min, int i_e_max,
                   int i_ch_min, int i_ch_max, int n_e_obs, const char* out_dir) {
  if (!rmf_path || !arf_path || !out_dir) throw Error(PPM_E_INVALID, "null path");
  if (n_e_obs < 2) throw Error(PPM_E_INVALID, "n_e_obs must be at least 2");
  // ARF: E_lo E_hi area per fine bin after 3 header lines; RMF: last column, energy-major
  const auto arf = load_table(arf_path, 3);
  const auto rmf_rows = load_table(rmf_path, 3);
  const size_t n_e_all = arf.size();
  if (rmf_rows.size() % n_e_all) throw Error(PPM_E_IO, "RMF size is not a multiple of the ARF's energy count");
  const size_t n_ch_all = rmf_rows.size() / n_e_all;
  if (i_e_min < 0 || i_e_max > (int)n_e_all || i_e_min >= i_e_max || i_ch_min < 0 || i_ch_max > (int)n_ch_all ||
      i_ch_min >= i_ch_max)
    throw Error(PPM_E_RANGE, "trim ranges outside the RMF / ARF (" + std::to_string(n_ch_all) + " channels, " +
                                 std::to_string(n_e_all) + " energies)");
  const int n_e = i_e_max - i_e_min, n_ch = i_ch_max - i_ch_min;
  std::vector<double> e_lo(n_e), e_hi(n_e), area(n_e), rmf((size_t)n_ch * n_e), ism(n_e, 1.0);
  for (int j = 0; j < n_e; ++j) {
    const auto& r = arf[(size_t)(i_e_min + j)];
    if (r.size() < 3) throw Error(PPM_E_IO, "ARF rows need E_lo, E_hi and area");
    e_lo[j] = r[0];
    e_hi[j] = r[1];
    area[j] = r[2];
  }
  for (int ch = 0; ch < n_ch; ++ch)
    for (int j = 0; j < n_e; ++j) rmf[(size_t)ch * n_e + j] = rmf_rows[(size_t)(i_e_min + j) * n_ch_all + i_ch_min + ch].back();
  // ISM transmission: spline through (column 0, column 2), at the bin middles, to the 5th power (c_ism_inst.py:88-93)
  if (ism_path) {
    const auto t = load_table(ism_path, 0);
    std::vector<double> xe, fr;
    for (const auto& r : t) {
      if (r.size() < 3) throw Error(PPM_E_IO, "ISM rows need at least three columns");
      xe.push_back(r[0]);
      fr.push_back(r[2]);
    }
    const Spline sp = not_a_knot_spline(xe, fr);
    for (int j = 0; j < n_e; ++j) ism[j] = std::pow(spline_value(sp, 0.5 * (e_lo[j] + e_hi[j])), 5);
  }
  // E_obs = geomspace(E_edges[0], E_edges[-1], n) (c_ism_inst.py:61)
  const double a = e_lo[0], b = e_hi[n_e - 1];
  std::vector<double> e_obs(n_e_obs);
  const double la = std::log10(a), lb = std::log10(b), step = (lb - la) / (n_e_obs - 1);
  for (int i = 0; i < n_e_obs; ++i) e_obs[i] = std::pow(10.0, i * step + la);
  e_obs[0] = a;
  e_obs[n_e_obs - 1] = b;
  std::vector<double> rsp((size_t)n_ch * n_e_obs);
  prepare(n_ch, n_e, rmf.data(), area.data(), e_lo.data(), e_hi.data(), ism_path ? ism.data() : nullptr, n_e_obs,
          e_obs.data(), rsp.data());
  for (double& v : rsp)
    if (std::fabs(v) < 1e-300) v = 0.0;  // c_ism_inst.py:99
  const std::string d(out_dir);
  {
    FILE* f = std::fopen((d + "/num.txt").c_str(), "w");
    if (!f) throw Error(PPM_E_IO, "cannot write " + d + "/num.txt");
    std::fprintf(f, "%d %d\n", n_ch, n_e_obs);
    std::fclose(f);
  }
  write_rows(d + "/E_obs.txt", e_obs.data(), (size_t)n_e_obs, 1);
  write_rows(d + "/rsp.txt", rsp.data(), (size_t)n_ch, (size_t)n_e_obs);
}

template <class F>
int guarded_host(F&& f) {
  try {
    clear_error();
    f();
    return PPM_OK;
  } catch (const Error& e) {
    return set_error(e.code, e.what());
  } catch (const std::bad_alloc&) {
    return set_error(PPM_E_OOM, "host allocation failed");
  } catch (const std::exception& e) {
    return set_error(PPM_E_INVALID, e.what());
  }
}

}  // namespace
}  // namespace ppm

extern "C" {

int ppm_response_prepare(int32_t n_ch, int32_t n_fine, const double* rmf, const double* area, const double* e_lo,
                         const double* e_hi, const double* ism, int32_t n_obs, const double* e_obs, double* rsp) {
  return ppm::guarded_host([&] { ppm::prepare(n_ch, n_fine, rmf, area, e_lo, e_hi, ism, n_obs, e_obs, rsp); });
}

int ppm_ism_inst_prepare(const char* rmf_path, const char* arf_path, const char* ism_path, int32_t i_e_min,
                         int32_t i_e_max, int32_t i_ch_min, int32_t i_ch_max, int32_t n_e_obs, const char* out_dir) {
  return ppm::guarded_host([&] {
    ppm::prepare_files(rmf_path, arf_path, ism_path, i_e_min, i_e_max, i_ch_min, i_ch_max, n_e_obs, out_dir);
  });
}

}  // extern "C"
