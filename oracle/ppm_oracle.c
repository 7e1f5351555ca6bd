/*
 * ppm_oracle.c — FP64 CPU restatement of the fizban007/gpu_ppm pulse-profile
 * path.  TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and the
 * CPU-baseline leg of bench.py use it as the checker.  The engine never links,
 * loads or calls it.
 *
 * It restates, with runtime parameters instead of the reference's constexpr
 * scenario constants:
 *   GenerateHealpixGrid + DiskDifference     cpu/grid.hpp:158-250
 *   PointSource                              cpu/grid.hpp:18-27
 *   calc_one_star (oblate geometry, fine-phase sweep, gap fill, GL deposit)
 *                                            cpu/devarshi24st_cpu.cpp:25-242
 *   blackbody + beaming variant              cpu/os1_cpu.cpp:39-183, cpu/unit.hpp:28-31
 *   response fold                            cpu/devarshi24st_cpu.cpp:249-258
 *   Lensing bilinear lookups                 cpu/lensing.hpp:44-72
 *   UniformHunt / VecHunt                    cpu/hunt.hpp:8-131
 *   NSX interpolators 4c, 4c_le, 2l2c_le, 4l cpu/nsx.hpp:159-321
 *   Gauss-Legendre nodes/weights             cpu/gl.hpp:1-70
 * Expressions keep the reference's operation order so that, compiled with
 * -ffp-contract=off, results match the reference CPU build bit for bit where
 * the same libm is used.  Out-of-range lookups are clamped as the reference
 * CPU does and counted instead of printed.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/ppm.h"

/* cpu/unit.hpp:5-25 */
static const double schwarzschild_radius_of_sun_in_km = 2.9532501;
static const double sqrt_km3_over_s2_GMsun = 2.745011592867327e-6;
static const double pi = 3.14159265358979323846;
#define two_pi (2. * pi)
static const double h_in_keV_s = 4.135668e-18;
#define c_in_m_s 299792458.
#define c_in_km_s (c_in_m_s / 1e3)
#define c_in_cm_s (c_in_m_s * 1e2)
#define Ibb_constant (2. / (h_in_keV_s * h_in_keV_s * h_in_keV_s * c_in_cm_s * c_in_cm_s))
static const double kpc_in_km = 3.08567758e+16;
static const double planck = 6.62607015E-27;

/* cpu/gl.hpp:5-62 — published Gauss-Legendre nodes/weights on [-1,1], N = 1..6 */
static const double GLNodes_raw[] = {
    0.0,
    -0.5773502691896257645091488, 0.5773502691896257645091488,
    -0.7745966692414833770358531, 0.0, 0.7745966692414833770358531,
    -0.8611363115940525752239465, -0.3399810435848562648026658, 0.3399810435848562648026658,
    0.8611363115940525752239465,
    -0.9061798459386639927976269, -0.5384693101056830910363144, 0.0, 0.5384693101056830910363144,
    0.9061798459386639927976269,
    -0.9324695142031520278123016, -0.6612093864662645136613996, -0.2386191860831969086305017,
    0.2386191860831969086305017, 0.6612093864662645136613996, 0.9324695142031520278123016};
static const double GLWeights_raw[] = {
    2.0,
    1.0, 1.0,
    0.5555555555555555555555556, 0.8888888888888888888888889, 0.5555555555555555555555556,
    0.3478548451374538573730639, 0.6521451548625461426269361, 0.6521451548625461426269361,
    0.3478548451374538573730639,
    0.2369268850561890875142640, 0.4786286704993664680412915, 0.5688888888888888888888889,
    0.4786286704993664680412915, 0.2369268850561890875142640,
    0.1713244923791703450402961, 0.3607615730481386075698335, 0.4679139345726910473898703,
    0.4679139345726910473898703, 0.3607615730481386075698335, 0.1713244923791703450402961};

/* cpu/gl.hpp:64-70 */
static double GLNodes(int N, int i, double a, double b) {
  return 0.5 * (a + b + GLNodes_raw[N * (N - 1) / 2 + i] * (b - a));
}
static double GLWeights(int N, int i, double dx) { return 0.5 * dx * GLWeights_raw[N * (N - 1) / 2 + i]; }

/* ---- hunts (cpu/hunt.hpp) ------------------------------------------------ */
typedef struct {
  double x_min, x_max;
  int n;
} uhunt;

/* cpu/hunt.hpp:98-121: clamps *x to the grid and returns (i, a). */
static int uhunt_find(const uhunt* h, double* x, double* a, int64_t* nclamp) {
  if (*x <= h->x_min) {
    if (*x < h->x_min && nclamp) ++*nclamp;
    *a = 0;
    *x = h->x_min;
    return 0;
  }
  if (*x >= h->x_max) {
    if (*x > h->x_max && nclamp) ++*nclamp;
    *a = 1;
    *x = h->x_max;
    return h->n - 2;
  }
  double t = (*x - h->x_min) / (h->x_max - h->x_min) * (h->n - 1);
  int i = (int)t;
  *a = t - i;
  return i;
}
/* cpu/hunt.hpp:123-130 */
static double uhunt_at(const uhunt* h, int i) { return h->x_min + (h->x_max - h->x_min) * i / (h->n - 1); }

/* cpu/hunt.hpp:14-66 for a strictly monotone table: the bracket jl with
 * xx[jl] <= x < xx[jl+1] (ascending) or xx[jl] > x >= xx[jl+1] (descending),
 * index clamped to [0, n-2], fraction extrapolated.  The reference's saved
 * starting index (jsav) only changes where the search starts, not the bracket. */
static int vhunt_find(const double* xx, int n, double x, double* a) {
  int ascnd = (xx[n - 1] >= xx[0]);
  int jl = -1, ju = n; /* invariant: jl < answer bracket <= ju */
  while (ju - jl > 1) {
    int jm = (ju + jl) >> 1;
    if ((x >= xx[jm]) == ascnd)
      jl = jm;
    else
      ju = jm;
  }
  int i = jl < 0 ? 0 : (jl > n - 2 ? n - 2 : jl);
  *a = (x - xx[i]) / (xx[i + 1] - xx[i]);
  return i;
}

static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

/* cpu/nsx.hpp:159-168 */
static void cubic_lagrange(double w[4], double x, double x0, double x1, double x2, double x3) {
  w[0] = (x - x1) * (x - x2) * (x - x3) / ((x0 - x1) * (x0 - x2) * (x0 - x3));
  w[1] = (x - x0) * (x - x2) * (x - x3) / ((x1 - x0) * (x1 - x2) * (x1 - x3));
  w[2] = (x - x0) * (x - x1) * (x - x3) / ((x2 - x0) * (x2 - x1) * (x2 - x3));
  w[3] = (x - x0) * (x - x1) * (x - x2) / ((x3 - x0) * (x3 - x1) * (x3 - x2));
}

/* ---- tables ----------------------------------------------------------------- */
typedef struct oracle_ctx {
  /* lensing (cpu/lensing.hpp:9-41) */
  uhunt cos_psi, u, cos_alpha;
  double *ca, *lf, *cdt;
  /* NSX (cpu/nsx.hpp:55-148), values stored as 10^logInuT3 */
  int has_nsx;
  int nT, ng, nE, nmu;
  uhunt logT_h, logg_h, logEkT_h;
  double* mu_vec;
  double* data;
} oracle_ctx;

static double nsx_at(const oracle_ctx* c, int iT, int ig, int iE, int im) {
  return c->data[(((size_t)iT * c->ng + ig) * c->nE + iE) * c->nmu + im];
}

/* cpu/lensing.hpp:44-61 */
static void lens_ca_lf(const oracle_ctx* c, double u_, double cos_psi_, double* ca, double* lf, int64_t* ncl) {
  double a_u, a_cp;
  int i_u = uhunt_find(&c->u, &u_, &a_u, ncl);
  int i_cp = uhunt_find(&c->cos_psi, &cos_psi_, &a_cp, ncl);
  double b_u = 1. - a_u, b_cp = 1. - a_cp;
  int n = c->cos_psi.n;
  const double* T = c->ca;
  *ca = b_u * b_cp * T[i_u * n + i_cp] + a_u * b_cp * T[(i_u + 1) * n + i_cp] + b_u * a_cp * T[i_u * n + i_cp + 1] +
        a_u * a_cp * T[(i_u + 1) * n + i_cp + 1];
  T = c->lf;
  *lf = b_u * b_cp * T[i_u * n + i_cp] + a_u * b_cp * T[(i_u + 1) * n + i_cp] + b_u * a_cp * T[i_u * n + i_cp + 1] +
        a_u * a_cp * T[(i_u + 1) * n + i_cp + 1];
}

/* cpu/lensing.hpp:63-72 */
static double lens_cdt(const oracle_ctx* c, double u_, double cos_alpha_, int64_t* ncl) {
  double a_u, a_ca;
  int i_u = uhunt_find(&c->u, &u_, &a_u, ncl);
  int i_ca = uhunt_find(&c->cos_alpha, &cos_alpha_, &a_ca, ncl);
  double b_u = 1. - a_u, b_ca = 1. - a_ca;
  int n = c->cos_alpha.n;
  const double* T = c->cdt;
  return b_u * b_ca * T[i_u * n + i_ca] + a_u * b_ca * T[(i_u + 1) * n + i_ca] + b_u * a_ca * T[i_u * n + i_ca + 1] +
         a_u * a_ca * T[(i_u + 1) * n + i_ca + 1];
}

/* ---- NSX interpolators (cpu/nsx.hpp:172-321) ----------------------------------- */
static double interp_4c(const oracle_ctx* c, double logT, double logg, double logEkT, double mu, int use_sg,
                        int64_t* ncl) {
  double aT, ag, aE, am;
  int iT = uhunt_find(&c->logT_h, &logT, &aT, ncl);
  int ig = uhunt_find(&c->logg_h, &logg, &ag, ncl);
  int iE = uhunt_find(&c->logEkT_h, &logEkT, &aE, ncl);
  int im = vhunt_find(c->mu_vec, c->nmu, mu, &am);
  iT = clampi(iT - 1, 0, c->nT - 4);
  ig = clampi(ig - 1, 0, c->ng - 4);
  iE = clampi(iE - 1, 0, c->nE - 4);
  im = clampi(im - 1, 0, c->nmu - 4);
  double wT[4], wg[4], wE[4], wm[4];
  cubic_lagrange(wT, logT, uhunt_at(&c->logT_h, iT), uhunt_at(&c->logT_h, iT + 1), uhunt_at(&c->logT_h, iT + 2),
                 uhunt_at(&c->logT_h, iT + 3));
  cubic_lagrange(wg, logg, uhunt_at(&c->logg_h, ig), uhunt_at(&c->logg_h, ig + 1), uhunt_at(&c->logg_h, ig + 2),
                 uhunt_at(&c->logg_h, ig + 3));
  cubic_lagrange(wE, logEkT, uhunt_at(&c->logEkT_h, iE), uhunt_at(&c->logEkT_h, iE + 1),
                 uhunt_at(&c->logEkT_h, iE + 2), uhunt_at(&c->logEkT_h, iE + 3));
  cubic_lagrange(wm, mu, c->mu_vec[im], c->mu_vec[im + 1], c->mu_vec[im + 2], c->mu_vec[im + 3]);
  double ret = 0;
  for (int jT = 0; jT <= 3; ++jT)
    for (int jg = 0; jg <= 3; ++jg)
      for (int jE = 0; jE <= 3; ++jE)
        for (int jm = 0; jm <= 3; ++jm) {
          double v = nsx_at(c, iT + jT, ig + jg, iE + jE, im + jm);
          double weight = wT[jT] * wg[jg] * wE[jE] * wm[jm];
          ret += v * weight;
        }
  if (use_sg && ret < 0) ret = 0;
  return ret;
}

static double interp_4c_le(const oracle_ctx* c, double logT, double logg, double logEkT, double mu, int64_t* ncl) {
  double aT, ag, aE, am;
  int iT = uhunt_find(&c->logT_h, &logT, &aT, ncl);
  int ig = uhunt_find(&c->logg_h, &logg, &ag, ncl);
  int iE = uhunt_find(&c->logEkT_h, &logEkT, &aE, ncl);
  int im = vhunt_find(c->mu_vec, c->nmu, mu, &am);
  iT = clampi(iT - 1, 0, c->nT - 4);
  ig = clampi(ig - 1, 0, c->ng - 4);
  iE = clampi(iE - 1, 0, c->nE - 4);
  double wT[4], wg[4], wE[4], wm[4];
  cubic_lagrange(wT, logT, uhunt_at(&c->logT_h, iT), uhunt_at(&c->logT_h, iT + 1), uhunt_at(&c->logT_h, iT + 2),
                 uhunt_at(&c->logT_h, iT + 3));
  cubic_lagrange(wg, logg, uhunt_at(&c->logg_h, ig), uhunt_at(&c->logg_h, ig + 1), uhunt_at(&c->logg_h, ig + 2),
                 uhunt_at(&c->logg_h, ig + 3));
  cubic_lagrange(wE, logEkT, uhunt_at(&c->logEkT_h, iE), uhunt_at(&c->logEkT_h, iE + 1),
                 uhunt_at(&c->logEkT_h, iE + 2), uhunt_at(&c->logEkT_h, iE + 3));
  int jm_max;
  if (im >= c->nmu - 5) {
    jm_max = 1;
    wm[0] = 1 - am;
    wm[1] = am;
  } else {
    jm_max = 3;
    im = clampi(im - 1, 0, c->nmu - 4);
    cubic_lagrange(wm, mu, c->mu_vec[im], c->mu_vec[im + 1], c->mu_vec[im + 2], c->mu_vec[im + 3]);
  }
  double ret = 0;
  for (int jT = 0; jT <= 3; ++jT)
    for (int jg = 0; jg <= 3; ++jg)
      for (int jE = 0; jE <= 3; ++jE)
        for (int jm = 0; jm <= jm_max; ++jm) {
          double v = nsx_at(c, iT + jT, ig + jg, iE + jE, im + jm);
          double weight = wT[jT] * wg[jg] * wE[jE] * wm[jm];
          ret += v * weight;
        }
  return ret;
}

static double interp_2l2c_le(const oracle_ctx* c, double logT, double logg, double logEkT, double mu, int64_t* ncl) {
  double aT, ag, aE, am;
  int iT = uhunt_find(&c->logT_h, &logT, &aT, ncl);
  int ig = uhunt_find(&c->logg_h, &logg, &ag, ncl);
  int iE = uhunt_find(&c->logEkT_h, &logEkT, &aE, ncl);
  int im = vhunt_find(c->mu_vec, c->nmu, mu, &am);
  iE = clampi(iE - 1, 0, c->nE - 4);
  double wE[4], wm[4];
  cubic_lagrange(wE, logEkT, uhunt_at(&c->logEkT_h, iE), uhunt_at(&c->logEkT_h, iE + 1),
                 uhunt_at(&c->logEkT_h, iE + 2), uhunt_at(&c->logEkT_h, iE + 3));
  int jm_max;
  if (im >= c->nmu - 5) {
    jm_max = 1;
    wm[0] = 1 - am;
    wm[1] = am;
  } else {
    jm_max = 3;
    im = clampi(im - 1, 0, c->nmu - 4);
    cubic_lagrange(wm, mu, c->mu_vec[im], c->mu_vec[im + 1], c->mu_vec[im + 2], c->mu_vec[im + 3]);
  }
  double ret = 0;
  for (int jT = 0; jT <= 1; ++jT)
    for (int jg = 0; jg <= 1; ++jg)
      for (int jE = 0; jE <= 3; ++jE)
        for (int jm = 0; jm <= jm_max; ++jm) {
          double v = nsx_at(c, iT + jT, ig + jg, iE + jE, im + jm);
          double weight = (jT * aT + (1 - jT) * (1 - aT)) * (jg * ag + (1 - jg) * (1 - ag)) * wE[jE] * wm[jm];
          ret += v * weight;
        }
  return ret;
}

static double interp_4l(const oracle_ctx* c, double logT, double logg, double logEkT, double mu, int64_t* ncl) {
  double aT, ag, aE, am;
  int iT = uhunt_find(&c->logT_h, &logT, &aT, ncl);
  int ig = uhunt_find(&c->logg_h, &logg, &ag, ncl);
  int iE = uhunt_find(&c->logEkT_h, &logEkT, &aE, ncl);
  int im = vhunt_find(c->mu_vec, c->nmu, mu, &am);
  double ret = 0;
  for (int jT = 0; jT <= 1; ++jT)
    for (int jg = 0; jg <= 1; ++jg)
      for (int jE = 0; jE <= 1; ++jE)
        for (int jm = 0; jm <= 1; ++jm) {
          double v = nsx_at(c, iT + jT, ig + jg, iE + jE, im + jm);
          double weight = (jT * aT + (1 - jT) * (1 - aT)) * (jg * ag + (1 - jg) * (1 - ag)) *
                          (jE * aE + (1 - jE) * (1 - aE)) * (jm * am + (1 - jm) * (1 - am));
          ret += v * weight;
        }
  return ret;
}

static double interp_any(const oracle_ctx* c, int mode, double logT, double logg, double logEkT, double mu,
                         int64_t* ncl) {
  switch (mode) {
    case PPM_INTERP_4C: return interp_4c(c, logT, logg, logEkT, mu, 0, ncl);
    case PPM_INTERP_4C_SG: return interp_4c(c, logT, logg, logEkT, mu, 1, ncl);
    case PPM_INTERP_4C_LE: return interp_4c_le(c, logT, logg, logEkT, mu, ncl);
    case PPM_INTERP_4L: return interp_4l(c, logT, logg, logEkT, mu, ncl);
    default: return interp_2l2c_le(c, logT, logg, logEkT, mu, ncl);
  }
}

/* ---- context ------------------------------------------------------------------- */
void oracle_destroy(oracle_ctx* c) {
  if (!c) return;
  free(c->ca);
  free(c->lf);
  free(c->cdt);
  free(c->mu_vec);
  free(c->data);
  free(c);
}

oracle_ctx* oracle_create(const ppm_lensing_desc* L, const ppm_nsx_desc* N) {
  if (!L) return NULL;
  oracle_ctx* c = (oracle_ctx*)calloc(1, sizeof(oracle_ctx));
  c->u = (uhunt){L->u_min, L->u_max, L->n_u};
  c->cos_psi = (uhunt){L->cos_psi_min, L->cos_psi_max, L->n_cos_psi};
  c->cos_alpha = (uhunt){L->cos_alpha_min, L->cos_alpha_max, L->n_cos_alpha};
  size_t np_ = (size_t)L->n_u * L->n_cos_psi, na = (size_t)L->n_u * L->n_cos_alpha;
  c->ca = (double*)malloc(np_ * sizeof(double));
  c->lf = (double*)malloc(np_ * sizeof(double));
  c->cdt = (double*)malloc(na * sizeof(double));
  memcpy(c->ca, L->cos_alpha_of_u_cos_psi, np_ * sizeof(double));
  memcpy(c->lf, L->lf_of_u_cos_psi, np_ * sizeof(double));
  memcpy(c->cdt, L->cdt_over_R_of_u_cos_alpha, na * sizeof(double));
  if (N) {
    c->has_nsx = 1;
    c->nT = N->n_logT;
    c->ng = N->n_logg;
    c->nE = N->n_logEkT;
    c->nmu = N->n_mu;
    c->logT_h = (uhunt){N->logT_min, N->logT_max, N->n_logT};
    c->logg_h = (uhunt){N->logg_min, N->logg_max, N->n_logg};
    c->logEkT_h = (uhunt){N->logEkT_min, N->logEkT_max, N->n_logEkT};
    c->mu_vec = (double*)malloc(sizeof(double) * N->n_mu);
    memcpy(c->mu_vec, N->mu, sizeof(double) * N->n_mu);
    size_t n = (size_t)N->n_logT * N->n_logg * N->n_logEkT * N->n_mu;
    c->data = (double*)malloc(n * sizeof(double));
    /* cpu/nsx.hpp:134 stores std::pow(10, logInuT3) */
    for (size_t k = 0; k < n; ++k) c->data[k] = pow(10, N->log_I_T3[k]);
  }
  return c;
}

/* Direct interpolator access (cpu/t_interp.cpp:420-428). */
double oracle_interp(const oracle_ctx* c, int mode, double logT, double logg, double logEkT, double mu) {
  return interp_any(c, mode, logT, logg, logEkT, mu, NULL);
}

/* ---- surface grid (cpu/grid.hpp) ------------------------------------------------- */
/* cpu/grid.hpp:219-244 cal_z_phi; returns 0 when (i, j) is on the grid. */
static int healpix_z_phi(int N_side, int i, int j, double* z, double* phi) {
  int mirror = 0;
  if (i > 2 * N_side) {
    i = 4 * N_side - i;
    mirror = 1;
  }
  if (1 <= i && i < N_side && 1 <= j && j <= 4 * i) {
    *z = 1. - 1. * i * i / (3. * N_side * N_side);
    double s = 1.;
    *phi = pi / (2. * i) * (j - s / 2.);
  } else if (N_side <= i && i <= 2 * N_side && 1 <= j && j <= 4 * N_side) {
    *z = 4. / 3. - 2. * i / (3. * N_side);
    double s = (i - N_side + 1) % 2;
    *phi = pi / (2. * N_side) * (j - s / 2.);
  } else {
    return -1;
  }
  if (mirror) *z = -*z;
  return 0;
}

/* cpu/grid.hpp:158-167 IsInside */
static int is_inside(double patch_theta, double patch_phi, double th, double ph, double ar) {
  double s1 = sin(th);
  double c1 = cos(th);
  double c2 = cos(patch_theta);
  double s2 = sin(patch_theta);
  double cos_rho = s1 * s2 * cos(patch_phi - ph) + c1 * c2;
  return cos_rho > cos(ar);
}

/* cpu/grid.hpp:184-189 DiskDifference::operator() */
static int in_spot(const ppm_spot* s, double theta, double phi) {
  return is_inside(theta, phi, s->theta1, s->phi1, s->angrad1) && !is_inside(theta, phi, s->theta2, s->phi2, s->angrad2);
}

typedef struct {
  double cos_theta, dOmega;
  int n_active;
  double* phi;
} oring;

/* GenerateHealpixGrid (cpu/grid.hpp:194-250) or PointSource (cpu/grid.hpp:18-27),
 * restricted to rings ring_begin <= i < ring_end (a point source is ring 0). */
static int build_grid(const ppm_spot* s, int N_side, int ring_begin, int ring_end, oring** out, int* n_rings,
                      int64_t* n_active) {
  *n_active = 0;
  if (s->kind == PPM_SPOT_POINT && !(ring_begin <= 0 && 0 < ring_end)) {
    *out = NULL;
    *n_rings = 0;
    return 0;
  }
  if (s->kind == PPM_SPOT_POINT) {
    oring* r = (oring*)calloc(1, sizeof(oring));
    double sin_half_ar = sin(0.5 * s->angrad1);
    r->cos_theta = cos(s->theta1);
    r->dOmega = two_pi * 2. * sin_half_ar * sin_half_ar;
    r->n_active = 1;
    r->phi = (double*)calloc(1, sizeof(double));
    *out = r;
    *n_rings = 1;
    *n_active = 1;
    return 0;
  }
  double dOmega = pi / (3. * N_side * N_side);
  int cap = 4 * N_side - 1;
  oring* rings = (oring*)calloc(cap, sizeof(oring));
  double* buf = (double*)malloc(sizeof(double) * 4 * N_side);
  int nr = 0;
  for (int i = 1; i <= 4 * N_side - 1; ++i) {
    if (i < ring_begin || i >= ring_end) continue;
    int m = i < 4 * N_side - i ? i : 4 * N_side - i;
    if (N_side < m) m = N_side;
    int jmax = 4 * m;
    double cos_theta = -999, z, phi;
    int na = 0;
    for (int j = 1; j <= jmax; ++j) {
      healpix_z_phi(N_side, i, j, &z, &phi);
      cos_theta = z;
      if (in_spot(s, acos(cos_theta), phi)) buf[na++] = phi;
    }
    if (na > 0) {
      rings[nr].cos_theta = cos_theta;
      rings[nr].dOmega = dOmega;
      rings[nr].n_active = na;
      rings[nr].phi = (double*)malloc(sizeof(double) * na);
      memcpy(rings[nr].phi, buf, sizeof(double) * na);
      *n_active += na;
      ++nr;
    }
  }
  free(buf);
  *out = rings;
  *n_rings = nr;
  return 0;
}

int64_t oracle_count_active(const ppm_spot* s, int N_side) {
  oring* rings;
  int nr;
  int64_t na;
  build_grid(s, N_side, 0, 4 * N_side, &rings, &nr, &na);
  for (int r = 0; r < nr; ++r) free(rings[r].phi);
  free(rings);
  return na;
}

/* ---- one profile ------------------------------------------------------------------ */
/* flux[n_bins][n_e] accumulates the reference's total_flux(i_phase_bin, i_E), over
 * the HEALPix rings ring_begin <= i < ring_end only (a point source is ring 0). */
int oracle_profile_rings(const oracle_ctx* c, const ppm_params* p, int ring_begin, int ring_end, int n_e,
                         const double* E_obs, double* flux, ppm_result_info* info) {
  if (!c || !p || !E_obs || !flux) return PPM_E_INVALID;
  const int nsx = p->atmosphere == PPM_ATM_NSX;
  if (nsx && !c->has_nsx) return PPM_E_STATE;
  const int N_fine_phase = p->n_fine;
  const int N_bins = p->n_bins;
  const int N_pts = p->n_gl;
  ppm_result_info inf;
  memset(&inf, 0, sizeof(inf));
  memset(flux, 0, sizeof(double) * (size_t)N_bins * n_e);

  /* cpu/devarshi24st_cpu.cpp:48-74 with runtime values */
  const double M = p->mass_msun, Re = p->r_eq_km, frequency_nu = p->spin_hz, obs_theta = p->inclination_rad;
  const double D = p->distance_kpc * kpc_in_km;
  const double phase_bin_width = 1. / N_bins;
  double Rs = M * schwarzschild_radius_of_sun_in_km;
  double ue = Rs / Re;
  double uue = sqrt(1. - ue);
  double logg0 = log10(M / (Re * Re * uue));
  double logGMsun_s2_km2cm = log10(1.32712440041279419E16);
  double Omega_bar = two_pi * frequency_nu * sqrt(Re * Re * Re / M) * sqrt_km3_over_s2_GMsun;
  double x = 0.5 * Rs / Re;
  double o2 = Omega_bar * Omega_bar * (-0.788 + 1.030 * x);
  double D2 = D * D;
  double cos_obs_theta = cos(obs_theta);
  double sin_obs_theta = sin(obs_theta);

  double* F = (double*)malloc(sizeof(double) * (N_fine_phase + 1));
  double* Z = (double*)malloc(sizeof(double) * (N_fine_phase + 1));
  double* P = (double*)malloc(sizeof(double) * (N_fine_phase + 1));
  double* MU = (double*)malloc(sizeof(double) * (N_fine_phase + 1));

  for (int sp = 0; sp < p->n_spots; ++sp) {
    const ppm_spot* s = &p->spots[sp];
    double logT = s->logT;
    double T_in_kelvin = pow(10, logT);
    double kT_in_keV = nsx ? T_in_kelvin * 8.617333262E-8 : s->kT_keV;
    double IT3_to_I = pow(10, 3 * logT) / planck; /* applied as IT3 * pow(10, 3 logT) / planck */
    (void)IT3_to_I;
    oring* grid;
    int n_rings;
    int64_t n_act;
    build_grid(s, p->n_side, ring_begin, ring_end, &grid, &n_rings, &n_act);
    inf.n_active += n_act;
    inf.n_rings += n_rings;

    for (int r = 0; r < n_rings; ++r) {
      const oring* ring = &grid[r];
      /* cpu/devarshi24st_cpu.cpp:90-124 */
      double cos_spot_theta = ring->cos_theta;
      double sin_spot_theta = sqrt(1. - cos_spot_theta * cos_spot_theta);
      double R = Re * (1. + o2 * cos_spot_theta * cos_spot_theta);
      double dRdtheta = -2. * Re * o2 * cos_spot_theta * sin_spot_theta;
      double u = Rs / R;
      double uu = sqrt(1. - u);
      double f = dRdtheta / (R * uu);
      double ff = sqrt(1. + f * f);
      double dS = R * R * ring->dOmega * ff;
      double cos_tau = 1. / ff;
      double sin_tau = f / ff;
      if (u < c->u.x_min || u > c->u.x_max) ++inf.n_clamped;

      const double c0e = -0.791, c1e = 0.776, c0p = 1.138, c1p = -1.431, d1e = -1.315, d2e = 2.431, f1e = -1.172,
                   d1p = 0.653, d2p = -2.864, f1p = 0.975, d160 = 13.47, d260 = -27.13;
      double ce = c0e + c1e * x;
      double cp = c0p + c1p * x;
      double de = d1e * x + d2e * x * x;
      double fe = f1e * x;
      double dp = d1p * x + d2p * x * x;
      double fp = f1p * x;
      double d60 = d160 * x + d260 * x * x;
      double Ob2 = Omega_bar * Omega_bar;
      double Ob4 = Ob2 * Ob2;
      double Ob6 = Ob4 * Ob2;
      double sc = cos_spot_theta;
      double sc2 = cos_spot_theta * cos_spot_theta;
      double ss2 = sin_spot_theta * sin_spot_theta;
      double g_g0 = 1. + ss2 * (ce * Ob2 + de * Ob4 + fe * Ob6) + sc2 * (cp * Ob2 + dp * Ob4 + fp * Ob6 - d60 * Ob4) +
                    fabs(sc) * d60 * Ob4;
      double logg_g0 = log10(g_g0);
      double logg = logg_g0 + logg0 + logGMsun_s2_km2cm;

      /* fine-phase sweep, cpu/devarshi24st_cpu.cpp:126-193 */
      int inv_min = N_fine_phase + 1, inv_max = -1;
      for (int i_phase = 0; i_phase < N_fine_phase; ++i_phase) {
        int is_visible = 1;
        do {
          double phase = 1. * i_phase / N_fine_phase;
          double spot_phi = two_pi * phase;
          double cos_spot_phi = cos(spot_phi);
          double sin_spot_phi = sin(spot_phi);
          double cos_psi = cos_obs_theta * cos_spot_theta + sin_obs_theta * sin_spot_theta * cos_spot_phi;
          if (cos_psi < c->cos_psi.x_min) {
            is_visible = 0;
            break;
          }
          double sin_psi = sqrt(1. - cos_psi * cos_psi);
          double cos_alpha, lf;
          lens_ca_lf(c, u, cos_psi, &cos_alpha, &lf, NULL);
          double sin_alpha = sqrt(1. - cos_alpha * cos_alpha);
          double sin_alpha_over_sin_psi = cos_psi == 1. ? sqrt(lf) : sin_alpha / sin_psi;
          double cos_sigma = cos_alpha * cos_tau + sin_alpha_over_sin_psi * sin_tau *
                                                       (cos_obs_theta * sin_spot_theta -
                                                        sin_obs_theta * cos_spot_theta * cos_spot_phi);
          if (cos_sigma <= 0) {
            is_visible = 0;
            break;
          }
          double beta = two_pi * frequency_nu * R * sin_spot_theta / uu / c_in_km_s;
          double gamma = 1. / sqrt(1. - beta * beta);
          double cos_xi = -sin_alpha_over_sin_psi * sin_obs_theta * sin_spot_phi;
          double delta = 1. / (gamma * (1. - beta * cos_xi));
          double delta3 = delta * delta * delta;
          double cdt_over_R = lens_cdt(c, u, cos_alpha, NULL);
          double dt1 = cdt_over_R * R / c_in_km_s;
          double dt2;
          {
            double RR = R;
            double lg = log1p((Re - RR) / (RR - Rs));
            double cdt = Re - RR + Rs * lg;
            dt2 = cdt / c_in_km_s;
          }
          if (!(cos_alpha >= 0)) {
            double tmp = (2. * sin_alpha) / sqrt(3. * (1. - u));
            double p_over_R = -tmp * cos((acos(3. * u / tmp) + 2. * pi) / 3.);
            double pp = p_over_R * R;
            double lg = log1p((Re - pp) / (pp - Rs));
            double cdt = Re - pp + Rs * lg;
            double dt2p = cdt / c_in_km_s;
            dt2 = 2. * dt2p - dt2;
          }
          double delta_phase = (dt1 + dt2) * frequency_nu;
          double cos_sigma_prime = cos_sigma * delta;
          double beaming_factor = 1.0;
          if (!nsx) {
            if (p->beaming == PPM_BEAM_SIN2)
              beaming_factor = 1. - cos_sigma_prime * cos_sigma_prime;
            else if (p->beaming == PPM_BEAM_COS2)
              beaming_factor = cos_sigma_prime * cos_sigma_prime;
          }
          F[i_phase] = uu * delta3 * cos_sigma_prime * lf * (dS * gamma) / D2 * beaming_factor;
          Z[i_phase] = 1. / (delta * uu);
          P[i_phase] = phase + delta_phase;
          MU[i_phase] = cos_sigma_prime;
        } while (0);
        if (!is_visible) {
          F[i_phase] = 0;
          Z[i_phase] = -1;
          P[i_phase] = -1;
          MU[i_phase] = 0;
          if (i_phase < inv_min) inv_min = i_phase;
          if (i_phase > inv_max) inv_max = i_phase;
        }
      }
      /* cpu/devarshi24st_cpu.cpp:195-212 */
      if (inv_min == 0 || inv_max == N_fine_phase - 1) {
        ++inf.n_dropped_rings;
        continue;
      }
      if (inv_min <= inv_max) {
        int beg = inv_min - 1;
        int end = inv_max + 1;
        double phase0 = P[beg], phase1 = P[end];
        double rf0 = Z[beg], rf1 = Z[end];
        for (int i_phase = inv_min; i_phase <= inv_max; ++i_phase) {
          P[i_phase] = phase0 + (phase1 - phase0) * ((double)(i_phase - beg) / (end - beg));
          Z[i_phase] = rf0 + (rf1 - rf0) * ((double)(i_phase - beg) / (end - beg));
        }
      }
      F[N_fine_phase] = F[0];
      Z[N_fine_phase] = Z[0];
      P[N_fine_phase] = 1.0 + P[0];
      MU[N_fine_phase] = MU[0];

      /* deposit, cpu/devarshi24st_cpu.cpp:214-241 (GL bins) and cpu/os1_cpu.cpp:169-182 (points) */
      int n_pp = N_pts > 0 ? N_bins * N_pts : N_bins;
      for (int i_pp = 0; i_pp < n_pp; ++i_pp) {
        int i_bin = N_pts > 0 ? i_pp / N_pts : i_pp;
        int j_in_bin = N_pts > 0 ? i_pp % N_pts : 0;
        for (int k = 0; k < ring->n_active; ++k) {
          double phi = ring->phi[k];
          double phase_shift = phi / two_pi;
          double phase_point;
          if (N_pts > 0) {
            double phase_lb = i_bin * phase_bin_width;
            double phase_ub = (i_bin + 1) * phase_bin_width;
            phase_point = GLNodes(N_pts, j_in_bin, phase_lb, phase_ub);
          } else {
            phase_point = i_bin * (1.0 / N_bins);
          }
          double patch_phase = fmod(phase_point + phase_shift + 1., 1.);
          if (patch_phase < P[0]) patch_phase += 1.;
          double a;
          int i = vhunt_find(P, N_fine_phase + 1, patch_phase, &a);
          double flux_over_I = (1 - a) * F[i] + a * F[i + 1];
          if (flux_over_I == 0) continue;
          ++inf.n_points;
          double redshift_factor = (1 - a) * Z[i] + a * Z[i + 1];
          double w = N_pts > 0 ? GLWeights(N_pts, j_in_bin, 1) : 1.0;
          double* row = flux + (size_t)i_bin * n_e;
          if (nsx) {
            double mu = (1 - a) * MU[i] + a * MU[i + 1];
            if (mu < c->mu_vec[c->nmu - 1]) mu = c->mu_vec[c->nmu - 1];
            int clamped = 0;
            for (int i_E = 0; i_E < n_e; ++i_E) {
              double E_obs_in_keV = E_obs[i_E];
              double E_emit_in_keV = E_obs_in_keV * redshift_factor;
              double logEkT = log10(E_emit_in_keV / kT_in_keV);
              int64_t ncl = 0;
              double IT3 = interp_any(c, p->interp, logT, logg, logEkT, mu, &ncl);
              if (ncl) clamped = 1;
              double I = IT3 * pow(10, 3 * logT) / planck;
              if (N_pts > 0)
                row[i_E] += flux_over_I * I / E_obs_in_keV * w;
              else
                row[i_E] += flux_over_I * I / E_obs_in_keV;
            }
            inf.n_clamped += clamped;
          } else {
            for (int i_E = 0; i_E < n_e; ++i_E) {
              double E_obs_in_keV = E_obs[i_E];
              double E_emit = E_obs_in_keV * redshift_factor;
              double I = Ibb_constant * (E_emit * E_emit * E_emit) / expm1(E_emit / kT_in_keV);
              if (N_pts > 0)
                row[i_E] += flux_over_I * I / E_obs_in_keV * w;
              else
                row[i_E] += flux_over_I * I / E_obs_in_keV;
            }
          }
        }
      }
    }
    for (int r = 0; r < n_rings; ++r) free(grid[r].phi);
    free(grid);
  }
  free(F);
  free(Z);
  free(P);
  free(MU);
  if (info) *info = inf;
  return PPM_OK;
}

int oracle_profile(const oracle_ctx* c, const ppm_params* p, int n_e, const double* E_obs, double* flux,
                   ppm_result_info* info) {
  return oracle_profile_rings(c, p, 0, 1 << 30, n_e, E_obs, flux, info);
}

/* cpu/devarshi24st_cpu.cpp:249-258: counts[ch][b] = sum_E flux[b][E] rsp[ch][E] * exposure * bin width */
void oracle_fold(int n_ch, int n_e, int n_bins, const double* rsp, const double* flux, double exposure_time,
                 double* counts) {
  double phase_bin_width = 1. / n_bins;
  for (int i_ch = 0; i_ch < n_ch; ++i_ch)
    for (int b = 0; b < n_bins; ++b) {
      double sum = 0;
      for (int i_E = 0; i_E < n_e; ++i_E) sum += flux[(size_t)b * n_e + i_E] * rsp[(size_t)i_ch * n_e + i_E];
      counts[(size_t)i_ch * n_bins + b] = sum * exposure_time * phase_bin_width;
    }
}

/* ---- many profiles on host threads (CPU baseline) ---------------------------------- */
typedef struct {
  const oracle_ctx* c;
  const ppm_params* p;
  int n_e;
  const double* E;
  double* flux;
  size_t stride;
  int n;
  int* next; /* shared work counter: profiles are handed out one at a time */
  ppm_result_info* info;
} batch_job;

static void* batch_worker(void* arg) {
  batch_job* j = (batch_job*)arg;
  for (;;) {
    int k = __atomic_fetch_add(j->next, 1, __ATOMIC_RELAXED);
    if (k >= j->n) break;
    oracle_profile(j->c, &j->p[k], j->n_e, j->E, j->flux + (size_t)k * j->stride, j->info ? &j->info[k] : NULL);
  }
  return NULL;
}

/* Runs n profiles (same energy grid and n_bins) on n_threads host threads. */
int oracle_profile_batch(const oracle_ctx* c, int n, const ppm_params* p, int n_e, const double* E, double* flux,
                         ppm_result_info* info, int n_threads) {
  if (n_threads < 1) n_threads = 1;
  if (n_threads > 256) n_threads = 256;
  size_t stride = (size_t)p[0].n_bins * n_e;
  pthread_t th[256];
  batch_job jobs[256];
  int next = 0;
  for (int t = 0; t < n_threads; ++t) {
    jobs[t] = (batch_job){c, p, n_e, E, flux, stride, n, &next, info};
    pthread_create(&th[t], NULL, batch_worker, &jobs[t]);
  }
  for (int t = 0; t < n_threads; ++t) pthread_join(th[t], NULL);
  return PPM_OK;
}
