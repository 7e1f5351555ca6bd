// extern "C" entry points of include/ppm.h and the reference text-table readers.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <limits>
#include <string>
#include <vector>

#include "../../include/ppm.h"
#include "common.h"
#include "engine.h"

using ppm::Engine;
using ppm::Error;

struct ppm_engine {
  Engine* impl;
};

namespace {

template <class F>
int guarded(F&& f) {
  try {
    ppm::clear_error();
    f();
    return PPM_OK;
  } catch (const Error& e) {
    return ppm::set_error(e.code, e.what());
  } catch (const std::bad_alloc&) {
    return ppm::set_error(PPM_E_OOM, "host allocation failed");
  } catch (const std::exception& e) {
    return ppm::set_error(PPM_E_INVALID, e.what());
  }
}

Engine& eng(ppm_engine* e) {
  if (!e || !e->impl) throw Error(PPM_E_INVALID, "null engine");
  return *e->impl;
}

// read3 (gpu/read_file.cuh:23-35): "min max n"
void read3(const std::string& path, double& lo, double& hi, int& n) {
  std::ifstream f(path);
  if (!f) throw Error(PPM_E_IO, "cannot open " + path);
  if (!(f >> lo >> hi >> n)) throw Error(PPM_E_IO, "cannot read 3 values from " + path);
  if (n < 2) throw Error(PPM_E_IO, path + ": n must be at least 2 (cpu/hunt.hpp:91)");
}

void read_matrix(const std::string& path, size_t rows, size_t cols, std::vector<double>& m) {
  std::ifstream f(path);
  if (!f) throw Error(PPM_E_IO, "cannot open " + path);
  m.resize(rows * cols);
  for (size_t k = 0; k < m.size(); ++k)
    if (!(f >> m[k])) throw Error(PPM_E_IO, "error reading matrix from " + path);
}

// NSX::IsClose (cpu/nsx.hpp:150-156)
bool is_close(double a, double b) {
  const double atol = 10 * std::numeric_limits<double>::epsilon();
  const double rtol = 1e-8;
  double bigger = std::max(std::fabs(a), std::fabs(b));
  return std::fabs(a - b) <= atol + rtol * bigger;
}

}  // namespace

extern "C" {

int ppm_engine_create(const ppm_engine_config* cfg, ppm_engine** out) {
  return guarded([&] {
    if (!out) throw Error(PPM_E_INVALID, "null output handle");
    *out = nullptr;
    ppm_engine_config c{};
    if (cfg) c = *cfg;
    ppm_engine* h = new ppm_engine{new Engine(c)};
    *out = h;
  });
}

void ppm_engine_destroy(ppm_engine* e) {
  if (!e) return;
  delete e->impl;
  delete e;
}

int ppm_engine_load_lensing(ppm_engine* e, const ppm_lensing_desc* d) {
  return guarded([&] {
    if (!d) throw Error(PPM_E_INVALID, "null lensing description");
    eng(e).load_lensing(*d);
  });
}

// Lensing(setting) (cpu/lensing.hpp:33-41): u.txt, cos_psi.txt, cos_alpha.txt and three matrices.
int ppm_engine_load_lensing_dir(ppm_engine* e, const char* dir) {
  return guarded([&] {
    if (!dir) throw Error(PPM_E_INVALID, "null directory");
    std::string d(dir);
    ppm_lensing_desc L{};
    int nu, ncp, nca;
    read3(d + "/u.txt", L.u_min, L.u_max, nu);
    read3(d + "/cos_psi.txt", L.cos_psi_min, L.cos_psi_max, ncp);
    read3(d + "/cos_alpha.txt", L.cos_alpha_min, L.cos_alpha_max, nca);
    L.n_u = nu;
    L.n_cos_psi = ncp;
    L.n_cos_alpha = nca;
    std::vector<double> ca, lf, cdt;
    read_matrix(d + "/cos_alpha_of_u_cos_psi.txt", nu, ncp, ca);
    read_matrix(d + "/lf_of_u_cos_psi.txt", nu, ncp, lf);
    read_matrix(d + "/cdt_over_R_of_u_cos_alpha.txt", nu, nca, cdt);
    L.cos_alpha_of_u_cos_psi = ca.data();
    L.lf_of_u_cos_psi = lf.data();
    L.cdt_over_R_of_u_cos_alpha = cdt.data();
    eng(e).load_lensing(L);
  });
}

int ppm_engine_load_nsx(ppm_engine* e, const ppm_nsx_desc* d) {
  return guarded([&] {
    if (!d) throw Error(PPM_E_INVALID, "null NSX description");
    eng(e).load_nsx(*d);
  });
}

// NSX() (cpu/nsx.hpp:83-148): 5 columns logEkT mu logInuT3 logT logg, loop
// order logT -> logg -> logEkT -> mu, axes checked against the uniform grids.
int ppm_engine_load_nsx_file(ppm_engine* e, const char* path, const ppm_nsx_desc* axes) {
  return guarded([&] {
    if (!path || !axes) throw Error(PPM_E_INVALID, "null path or axes");
    const ppm_nsx_desc& a = *axes;
    if (a.n_logT < 2 || a.n_logg < 2 || a.n_logEkT < 2 || a.n_mu < 2) throw Error(PPM_E_INVALID, "NSX axes too short");
    std::ifstream f(path);
    if (!f) throw Error(PPM_E_IO, std::string("could not open NSX file: ") + path);
    const size_t n = (size_t)a.n_logT * a.n_logg * a.n_logEkT * a.n_mu;
    std::vector<double> logI(n), mu(a.n_mu, 0.0);
    std::vector<char> mu_set(a.n_mu, 0);
    auto node = [](double lo, double hi, int cnt, int i) { return lo + (hi - lo) * i / (cnt - 1); };
    size_t k = 0;
    for (int iT = 0; iT < a.n_logT; ++iT)
      for (int ig = 0; ig < a.n_logg; ++ig)
        for (int iE = 0; iE < a.n_logEkT; ++iE)
          for (int im = 0; im < a.n_mu; ++im, ++k) {
            double logEkT, m, logInuT3, logT, logg;
            if (!(f >> logEkT >> m >> logInuT3 >> logT >> logg))
              throw Error(PPM_E_IO, "error reading NSX data at indices " + std::to_string(iT) + "," +
                                        std::to_string(ig) + "," + std::to_string(iE) + "," + std::to_string(im));
            if (!mu_set[im]) {
              mu[im] = m;
              mu_set[im] = 1;
            } else if (!is_close(mu[im], m)) {
              throw Error(PPM_E_IO, "inconsistent mu value at index " + std::to_string(im));
            }
            if (!is_close(node(a.logEkT_min, a.logEkT_max, a.n_logEkT, iE), logEkT))
              throw Error(PPM_E_IO, "inconsistent logEkT value at index " + std::to_string(iE));
            if (!is_close(node(a.logT_min, a.logT_max, a.n_logT, iT), logT))
              throw Error(PPM_E_IO, "inconsistent logT value at index " + std::to_string(iT));
            if (!is_close(node(a.logg_min, a.logg_max, a.n_logg, ig), logg))
              throw Error(PPM_E_IO, "inconsistent logg value at index " + std::to_string(ig));
            logI[k] = logInuT3;
          }
    for (int i = 0; i + 1 < a.n_mu; ++i)
      if (mu[i] < mu[i + 1]) throw Error(PPM_E_IO, "mu is not monotonically decreasing at index " + std::to_string(i));
    ppm_nsx_desc d = a;
    d.mu = mu.data();
    d.log_I_T3 = logI.data();
    eng(e).load_nsx(d);
  });
}

int ppm_engine_add_energy_grid(ppm_engine* e, int32_t n_e, const double* E, int32_t* id) {
  return guarded([&] {
    int g = eng(e).add_grid(n_e, E);
    if (id) *id = g;
  });
}

int ppm_engine_add_response(ppm_engine* e, int32_t grid, int32_t n_ch, const double* rsp, int32_t* id) {
  return guarded([&] {
    int r = eng(e).add_response(grid, n_ch, rsp);
    if (id) *id = r;
  });
}

// IsmInst(setting) (cpu/ism_inst.hpp:65-69): num.txt (N_CH N_E_obs), E_obs.txt, rsp.txt.
int ppm_engine_load_ism_inst_dir(ppm_engine* e, const char* dir, int32_t* grid_id, int32_t* rsp_id) {
  return guarded([&] {
    if (!dir) throw Error(PPM_E_INVALID, "null directory");
    std::string d(dir);
    std::ifstream fn(d + "/num.txt");
    int n_ch, n_e;
    if (!fn) throw Error(PPM_E_IO, "could not open file: " + d + "/num.txt");
    if (!(fn >> n_ch >> n_e)) throw Error(PPM_E_IO, "error reading 2 values from " + d + "/num.txt");
    std::vector<double> E, rsp;
    read_matrix(d + "/E_obs.txt", 1, n_e, E);
    read_matrix(d + "/rsp.txt", n_ch, n_e, rsp);
    int g = eng(e).add_grid(n_e, E.data());
    int r = eng(e).add_response(g, n_ch, rsp.data());
    if (grid_id) *grid_id = g;
    if (rsp_id) *rsp_id = r;
  });
}

int ppm_profile(ppm_engine* e, const ppm_params* p, double* flux, double* counts, ppm_result_info* info) {
  return guarded([&] {
    if (!p) throw Error(PPM_E_INVALID, "null params");
    eng(e).profile(*p, flux, counts, info);
  });
}

int ppm_profile_batch(ppm_engine* e, int32_t n, const ppm_params* p, double* flux, double* counts,
                      ppm_result_info* info) {
  return guarded([&] {
    if (!p) throw Error(PPM_E_INVALID, "null params");
    eng(e).profile_batch(n, p, flux, counts, info);
  });
}

int ppm_batch_create(ppm_engine* e, int32_t n, const ppm_params* p, ppm_batch** out) {
  return guarded([&] {
    if (!p || !out) throw Error(PPM_E_INVALID, "null params or output handle");
    *out = nullptr;
    ppm::BatchImpl* b = new ppm::BatchImpl();
    try {
      eng(e).batch_build(*b, n, p);
    } catch (...) {
      delete b;
      throw;
    }
    *out = reinterpret_cast<ppm_batch*>(b);
  });
}

int ppm_batch_launch(ppm_engine* e, ppm_batch* b, void* stream) {
  return guarded([&] {
    if (!b) throw Error(PPM_E_INVALID, "null batch");
    eng(e).batch_launch(*reinterpret_cast<ppm::BatchImpl*>(b), (cudaStream_t)stream);
  });
}

int ppm_batch_device_outputs(ppm_batch* b, double** flux, int64_t* n_flux, double** counts, int64_t* n_counts) {
  return guarded([&] {
    if (!b) throw Error(PPM_E_INVALID, "null batch");
    auto* B = reinterpret_cast<ppm::BatchImpl*>(b);
    if (flux) *flux = B->d_flux;
    if (n_flux) *n_flux = B->flux_off[B->n];
    if (counts) *counts = B->d_counts;
    if (n_counts) *n_counts = B->counts_off[B->n];
  });
}

int ppm_batch_create_rings(ppm_engine* e, int32_t n, const ppm_params* p, int32_t ring_begin, int32_t ring_end,
                           ppm_batch** out) {
  return guarded([&] {
    if (!p || !out) throw Error(PPM_E_INVALID, "null params or output handle");
    *out = nullptr;
    ppm::BatchImpl* b = new ppm::BatchImpl();
    try {
      eng(e).batch_build(*b, n, p, nullptr, ring_begin, ring_end);
    } catch (...) {
      delete b;
      throw;
    }
    *out = reinterpret_cast<ppm_batch*>(b);
  });
}

int ppm_profile_rings(ppm_engine* e, const ppm_params* p, int32_t ring_begin, int32_t ring_end, double* flux,
                      double* counts, ppm_result_info* info) {
  return guarded([&] {
    if (!p) throw Error(PPM_E_INVALID, "null params");
    eng(e).profile_rings(*p, ring_begin, ring_end, flux, counts, info);
  });
}

int ppm_batch_collect(ppm_engine* e, ppm_batch* b, double* flux, double* counts, ppm_result_info* info) {
  return guarded([&] {
    if (!b) throw Error(PPM_E_INVALID, "null batch");
    eng(e).batch_collect(*reinterpret_cast<ppm::BatchImpl*>(b), flux, counts, info, nullptr);
  });
}

int ppm_batch_launch_timed(ppm_engine* e, ppm_batch* b, void* stream, float* ms) {
  return guarded([&] {
    if (!b || !ms) throw Error(PPM_E_INVALID, "null batch or output");
    eng(e).batch_launch_timed(*reinterpret_cast<ppm::BatchImpl*>(b), (cudaStream_t)stream, ms);
  });
}

int ppm_batch_kernel_count(ppm_engine* e, ppm_batch* b, int32_t* n) {
  return guarded([&] {
    if (!b || !n) throw Error(PPM_E_INVALID, "null batch or output");
    *n = eng(e).kernels_per_pass(*reinterpret_cast<ppm::BatchImpl*>(b));
  });
}

void ppm_batch_destroy(ppm_engine* e, ppm_batch* b) {
  if (!b) return;
  if (e && e->impl) cudaSetDevice(e->impl->cfg.device);
  delete reinterpret_cast<ppm::BatchImpl*>(b);
}

int ppm_engine_add_observed(ppm_engine* e, int32_t response, int32_t n_bins, const double* counts, int32_t* observed_id) {
  return guarded([&] {
    if (!observed_id) throw Error(PPM_E_INVALID, "null output");
    *observed_id = eng(e).add_observed(response, n_bins, counts);
  });
}

int ppm_batch_fit(ppm_engine* e, ppm_batch* b, int32_t observed_id, ppm_fit* out, void* stream) {
  return guarded([&] {
    if (!b) throw Error(PPM_E_INVALID, "null batch");
    eng(e).batch_fit(*reinterpret_cast<ppm::BatchImpl*>(b), observed_id, out, (cudaStream_t)stream);
  });
}

int ppm_profile_fit(ppm_engine* e, const ppm_params* p, int32_t observed_id, ppm_fit* out, ppm_result_info* info) {
  return guarded([&] {
    if (!p || !out) throw Error(PPM_E_INVALID, "null params or output");
    eng(e).profile_fit(*p, observed_id, out, info);
  });
}

int ppm_profile_noalloc(ppm_engine* e, const ppm_params* p, double* flux_device, double* counts_device, void* stream) {
  return guarded([&] {
    if (!p) throw Error(PPM_E_INVALID, "null params");
    eng(e).profile_noalloc(*p, flux_device, counts_device, (cudaStream_t)stream);
  });
}

int ppm_profile_noalloc_result(ppm_engine* e, void* stream, ppm_result_info* info) {
  int code = PPM_OK;
  const int rc = guarded([&] { code = eng(e).profile_noalloc_result((cudaStream_t)stream, info); });
  if (rc != PPM_OK) return rc;
  if (code == PPM_E_RANGE) return ppm::set_error(code, "ppm_profile_noalloc: the work queue overflowed");
  if (code == PPM_E_TIMEOUT)
    return ppm::set_error(code, "ppm_profile_noalloc: a bounded wait in the tensor-core fold ran out");
  return PPM_OK;
}

int ppm_engine_autotune(ppm_engine* e, int32_t n, const ppm_params* sample, char* report, int32_t report_len) {
  return guarded([&] {
    if (!sample || n < 1) throw Error(PPM_E_INVALID, "autotune needs sample profiles");
    std::string r = eng(e).autotune(n, sample);
    if (report && report_len > 0) {
      size_t k = std::min((size_t)report_len - 1, r.size());
      std::memcpy(report, r.data(), k);
      report[k] = 0;
    }
  });
}

int ppm_fold(ppm_engine* e, int32_t response, int32_t fold, int32_t n_profiles, int32_t n_bins, const double* alpha,
             const double* flux, double* counts) {
  return guarded([&] { eng(e).fold(response, fold, n_profiles, n_bins, alpha, flux, counts, false, nullptr); });
}

int ppm_fold_device(ppm_engine* e, int32_t response, int32_t fold, int32_t n_profiles, int32_t n_bins,
                    const double* alpha, const double* flux_device, double* counts_device, void* stream) {
  return guarded([&] {
    eng(e).fold(response, fold, n_profiles, n_bins, alpha, flux_device, counts_device, true, (cudaStream_t)stream);
  });
}

int ppm_output_sizes(ppm_engine* e, const ppm_params* p, int64_t* n_flux, int64_t* n_counts) {
  return guarded([&] {
    if (!p) throw Error(PPM_E_INVALID, "null params");
    eng(e).output_sizes(*p, n_flux, n_counts);
  });
}

int ppm_submit(ppm_engine* e, const ppm_params* p, double* flux, double* counts, uint64_t* ticket) {
  return guarded([&] {
    if (!p || !ticket) throw Error(PPM_E_INVALID, "null params or ticket");
    *ticket = eng(e).submit(*p, flux, counts);
  });
}

int ppm_poll(ppm_engine* e, uint64_t ticket, int32_t* done) {
  return guarded([&] {
    int d = eng(e).poll(ticket);
    if (done) *done = d;
  });
}

int ppm_wait(ppm_engine* e, uint64_t ticket, int32_t timeout_ms, ppm_result_info* info) {
  int st = PPM_OK;
  int rc = guarded([&] { st = eng(e).wait(ticket, timeout_ms, info); });
  if (rc != PPM_OK) return rc;
  return st;
}

int ppm_ticket_latency_us(ppm_engine* e, uint64_t ticket, double* us) {
  return guarded([&] {
    double v = eng(e).latency_us(ticket);
    if (us) *us = v;
  });
}

int ppm_ticket_release(ppm_engine* e, uint64_t ticket) {
  return guarded([&] { eng(e).release_ticket(ticket); });
}

int ppm_serve_trace(ppm_engine* e, ppm_serve_batch_trace* out, int32_t cap, int32_t* n_out) {
  return guarded([&] {
    if (cap < 0 || (cap > 0 && !out)) throw Error(PPM_E_INVALID, "trace buffer");
    const int n = eng(e).serve_trace(out, cap);
    if (n_out) *n_out = n;
  });
}

}  // extern "C"
