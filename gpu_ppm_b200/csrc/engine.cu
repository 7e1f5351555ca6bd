// Host side of the engine: resident tables, parameter conversion, workspace,
// and the plain / batched profile paths behind the C ABI of include/ppm.h.
//
// Replaces the reference's table constructors (gpu/lensing.cuh:27-54,
// gpu/nsx.cuh:83-128, gpu/ism_inst.cuh:18-32) and calc_one_star
// (gpu/devarshi24st_gpu.cu:432-511, gpu/os1_gpu.cu:304-349).  All device
// memory is owned by the engine; every error becomes a status code.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ppm.h"
#include "common.h"
#include "engine.h"
#include "kernels.cuh"

namespace ppm {

using namespace units;

#define PPM_CUDA(call)                                                                          \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess)                                                                      \
      throw Error(PPM_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));              \
  } while (0)

template <class T>
static T* dev_alloc(size_t n) {
  void* p = nullptr;
  if (n == 0) n = 1;
  cudaError_t e = cudaMalloc(&p, n * sizeof(T));
  if (e != cudaSuccess) throw Error(PPM_E_OOM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  return (T*)p;
}

template <class T>
static T* dev_upload(const T* h, size_t n) {
  T* d = dev_alloc<T>(n);
  cudaError_t e = cudaMemcpy(d, h, n * sizeof(T), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) throw Error(PPM_E_CUDA, std::string("cudaMemcpy: ") + cudaGetErrorString(e));
  return d;
}

void DeviceBuffer::reserve(size_t bytes) {
  if (bytes <= cap) return;
  size_t want = std::max(bytes, cap + cap / 2);
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  cap = 0;
  cudaError_t e = cudaMalloc(&ptr, want);
  if (e != cudaSuccess) throw Error(PPM_E_OOM, std::string("cudaMalloc workspace: ") + cudaGetErrorString(e));
  cap = want;
}
void* BlockCache::get(size_t bytes, size_t* got) {
  std::lock_guard<std::mutex> lk(m_);
  auto it = free_.lower_bound(bytes);
  if (it == free_.end() || it->first > 2 * bytes + (1u << 20)) return nullptr;
  void* p = it->second;
  *got = it->first;
  held_ -= it->first;
  free_.erase(it);
  return p;
}
void BlockCache::put(void* p, size_t bytes) {
  {
    std::lock_guard<std::mutex> lk(m_);
    if (held_ + bytes <= limit_) {
      free_.emplace(bytes, p);
      held_ += bytes;
      return;
    }
  }
  cudaFree(p);
}
void BlockCache::trim() {
  std::lock_guard<std::mutex> lk(m_);
  for (auto& kv : free_) cudaFree(kv.second);
  free_.clear();
  held_ = 0;
}

void* DeviceArena::alloc(size_t bytes) {
  void* p = nullptr;
  size_t sz = std::max<size_t>(bytes, 16);
  if (cache && !stream) {
    // 64 KiB granules, so that blocks of batches of similar size fit one another
    sz = (sz + 65535) / 65536 * 65536;
    size_t got = 0;
    p = cache->get(sz, &got);
    if (p) sz = got;
  }
  if (!p) {
    cudaError_t e = stream ? cudaMallocAsync(&p, sz, stream) : cudaMalloc(&p, sz);
    if (e != cudaSuccess && cache && !stream) {  // give the cached blocks back and retry once
      cudaGetLastError();
      cache->trim();
      e = cudaMalloc(&p, sz);
    }
    if (e != cudaSuccess) throw Error(PPM_E_OOM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  }
  ptrs.push_back(p);
  sizes.push_back(sz);
  bytes_held += bytes;
  return p;
}
DeviceArena::~DeviceArena() {
  for (size_t k = 0; k < ptrs.size(); ++k) {
    if (stream)
      cudaFreeAsync(ptrs[k], stream);
    else if (cache)
      cache->put(ptrs[k], sizes[k]);
    else
      cudaFree(ptrs[k]);
  }
}
BatchImpl::~BatchImpl() {
  if (graph) cudaGraphExecDestroy(graph);
  // cached blocks are handed to the next batch at once: the last launch must be done with them
  if (mem.cache && !mem.stream && last_stream) cudaStreamSynchronize(last_stream);
}

void DeviceBuffer::release() {
  if (ptr) cudaFree(ptr);
  ptr = nullptr;
  cap = 0;
}
void HostBuffer::reserve(size_t bytes) {
  if (bytes <= cap) return;
  if (ptr) cudaFreeHost(ptr);
  ptr = nullptr;
  cap = 0;
  cudaError_t e = cudaMallocHost(&ptr, bytes);
  if (e != cudaSuccess) throw Error(PPM_E_OOM, std::string("cudaMallocHost: ") + cudaGetErrorString(e));
  cap = bytes;
}
void HostBuffer::release() {
  if (ptr) cudaFreeHost(ptr);
  ptr = nullptr;
  cap = 0;
}

Engine::Engine(const ppm_engine_config& c) : cfg(c) {
  if (cfg.memory_budget <= 0) cfg.memory_budget = 64ll << 30;
  if (cfg.n_streams <= 0) cfg.n_streams = 3;
  if (cfg.max_batch <= 0) cfg.max_batch = 1 << 16;
  block_cache.set_limit((size_t)cfg.memory_budget);
  int n_dev = 0;
  PPM_CUDA(cudaGetDeviceCount(&n_dev));
  if (cfg.device < 0 || cfg.device >= n_dev) throw Error(PPM_E_INVALID, "no such CUDA device");
  PPM_CUDA(cudaSetDevice(cfg.device));
  PPM_CUDA(cudaDeviceGetAttribute(&sm_count, cudaDevAttrMultiProcessorCount, cfg.device));
  PPM_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  // launch-shape overrides for experiments: PPM_PB, PPM_CHUNK, PPM_SMALL_CHUNK, PPM_NE_T, PPM_MINB, PPM_KERNEL,
  // PPM_SETS, PPM_CPL, PPM_SPLITS, PPM_BB_NT
  if (const char* v = std::getenv("PPM_PB")) tune.pb = std::max(1, std::atoi(v));
  if (const char* v = std::getenv("PPM_CHUNK")) tune.chunk = std::max(32, std::atoi(v));
  if (const char* v = std::getenv("PPM_SMALL_CHUNK")) tune.small_chunk = std::max(32, std::atoi(v));
  if (const char* v = std::getenv("PPM_NE_T")) tune.ne_t = std::atoi(v);
  if (const char* v = std::getenv("PPM_MINB")) tune.minb = std::max(1, std::min(2, std::atoi(v)));
  if (const char* v = std::getenv("PPM_KERNEL")) tune.kernel = std::atoi(v) ? 1 : 0;
  if (const char* v = std::getenv("PPM_SETS")) tune.sets = std::max(0, std::atoi(v));
  if (const char* v = std::getenv("PPM_CPL")) tune.cpl = std::max(0, std::min(3, std::atoi(v)));
  if (const char* v = std::getenv("PPM_SPLITS")) tune.splits = std::max(0, std::atoi(v));
  if (const char* v = std::getenv("PPM_BB_NT")) tune.bb_nt = std::atoi(v) >= 512 ? 512 : (std::atoi(v) > 0 ? 256 : 0);
  for (int k = 0; k < 4; ++k) PPM_CUDA(cudaEventCreate(&ev[k]));
  PPM_CUDA(cudaMalloc(&d_err, sizeof(int)));
  PPM_CUDA(cudaMemset(d_err, 0, sizeof(int)));
}

Engine::~Engine() {
  cudaSetDevice(cfg.device);
  serve_shutdown();
  cudaStreamSynchronize(stream);
  block_cache.trim();
  if (d_err) cudaFree(d_err);
  for (void* p : owned) cudaFree(p);
  for (auto& kv : ring_tabs) cudaFree(kv.second);
  for (auto& kv : fine_tabs) cudaFree(kv.second);
  for (const Grid& g : grids)
    for (void* q : {(void*)g.drE, (void*)g.dfE, (void*)g.dperm, (void*)g.dfEs, (void*)g.dcell_first})
      if (q) cudaFree(q);
  for (int k = 0; k < 4; ++k) cudaEventDestroy(ev[k]);
  cudaStreamDestroy(stream);
}

void Engine::track(void* p) { owned.push_back(p); }

// ---- tables ------------------------------------------------------------------
void Engine::load_lensing(const ppm_lensing_desc& d) {
  if (d.n_u < 2 || d.n_cos_psi < 2 || d.n_cos_alpha < 2 || !d.cos_alpha_of_u_cos_psi || !d.lf_of_u_cos_psi ||
      !d.cdt_over_R_of_u_cos_alpha)
    throw Error(PPM_E_INVALID, "lensing table: need >= 2 points per axis and all three matrices");
  if (!(d.u_min < d.u_max && d.cos_psi_min < d.cos_psi_max && d.cos_alpha_min < d.cos_alpha_max))
    throw Error(PPM_E_INVALID, "lensing table: axis min must be below max");
  if (d.n_cos_psi > 4096 || d.n_cos_alpha > 4096) throw Error(PPM_E_RANGE, "lensing table: at most 4096 points per angle axis");
  PPM_CUDA(cudaSetDevice(cfg.device));
  PPM_CUDA(cudaStreamSynchronize(stream));
  DevLens L{};
  L.u_min = d.u_min;
  L.u_max = d.u_max;
  L.cp_min = d.cos_psi_min;
  L.cp_max = d.cos_psi_max;
  L.ca_min = d.cos_alpha_min;
  L.ca_max = d.cos_alpha_max;
  L.n_u = d.n_u;
  L.n_cp = d.n_cos_psi;
  L.n_ca = d.n_cos_alpha;
  double* ca = dev_upload(d.cos_alpha_of_u_cos_psi, (size_t)d.n_u * d.n_cos_psi);
  double* lf = dev_upload(d.lf_of_u_cos_psi, (size_t)d.n_u * d.n_cos_psi);
  double* cdt = dev_upload(d.cdt_over_R_of_u_cos_alpha, (size_t)d.n_u * d.n_cos_alpha);
  track(ca);
  track(lf);
  track(cdt);
  L.ca = ca;
  L.lf = lf;
  L.cdt = cdt;
  lens = L;
  has_lens = true;
}

void Engine::load_nsx(const ppm_nsx_desc& d) {
  if (d.n_logT < 2 || d.n_logg < 2 || d.n_logEkT < 4 || d.n_mu < 4 || !d.mu || !d.log_I_T3)
    throw Error(PPM_E_INVALID, "NSX table: need >= 2 logT/logg points, >= 4 logEkT/mu points and data");
  for (int i = 0; i + 1 < d.n_mu; ++i)
    if (!(d.mu[i] > d.mu[i + 1])) throw Error(PPM_E_INVALID, "NSX table: mu must be strictly descending (cpu/nsx.hpp:142-147)");
  PPM_CUDA(cudaSetDevice(cfg.device));
  PPM_CUDA(cudaStreamSynchronize(stream));
  const size_t slice = (size_t)d.n_logEkT * d.n_mu;
  const size_t stride = (slice + 3) / 4 * 4;
  const size_t n_sl = (size_t)d.n_logT * d.n_logg;
  // values 10^logInuT3 (cpu/nsx.hpp:134) scaled by a power of two so the largest is O(1) in FP32
  std::vector<double> lin(slice * n_sl);
  double vmax = 0.0;
  for (size_t k = 0; k < lin.size(); ++k) {
    lin[k] = std::pow(10, d.log_I_T3[k]);
    if (std::isfinite(lin[k])) vmax = std::max(vmax, std::fabs(lin[k]));
  }
  int e2 = 0;
  if (vmax > 0) std::frexp(vmax, &e2);
  const int scale_exp = -e2;
  std::vector<float> h(stride * n_sl, 0.0f);
  for (size_t sl = 0; sl < n_sl; ++sl)
    for (size_t k = 0; k < slice; ++k) h[sl * stride + k] = (float)std::ldexp(lin[sl * slice + k], scale_exp);
  float* data = dev_upload(h.data(), h.size());
  double* mu = dev_upload(d.mu, (size_t)d.n_mu);
  // 1 / ((x_j - x_k)(x_j - x_l)(x_j - x_m)) of each 4-node mu stencil (cpu/nsx.hpp:159-168)
  std::vector<double> den(4 * (size_t)(d.n_mu - 3));
  for (int st = 0; st + 3 < d.n_mu; ++st) {
    const double* x = d.mu + st;
    den[4 * st + 0] = 1.0 / ((x[0] - x[1]) * (x[0] - x[2]) * (x[0] - x[3]));
    den[4 * st + 1] = 1.0 / ((x[1] - x[0]) * (x[1] - x[2]) * (x[1] - x[3]));
    den[4 * st + 2] = 1.0 / ((x[2] - x[0]) * (x[2] - x[1]) * (x[2] - x[3]));
    den[4 * st + 3] = 1.0 / ((x[3] - x[0]) * (x[3] - x[1]) * (x[3] - x[2]));
  }
  double* mu_den = dev_upload(den.data(), den.size());
  track(data);
  track(mu);
  track(mu_den);
  DevNsx X{};
  X.nT = d.n_logT;
  X.ng = d.n_logg;
  X.nE = d.n_logEkT;
  X.nmu = d.n_mu;
  X.slice_stride = (int)stride;
  X.T_min = d.logT_min;
  X.T_max = d.logT_max;
  X.g_min = d.logg_min;
  X.g_max = d.logg_max;
  X.E_min = d.logEkT_min;
  X.E_max = d.logEkT_max;
  X.inv_dE = (d.n_logEkT - 1) / (d.logEkT_max - d.logEkT_min);
  X.data = data;
  X.mu = mu;
  X.mu_den = mu_den;
  X.scale_exp = scale_exp;
  nsx = X;
  nsx_mu.assign(d.mu, d.mu + d.n_mu);
  has_nsx = true;
  ++nsx_version;
}

int Engine::add_grid(int n_e, const double* E) {
  if (n_e < 1 || !E) throw Error(PPM_E_INVALID, "energy grid: need at least one energy");
  if (n_e > 2048) throw Error(PPM_E_RANGE, "energy grid: at most 2048 energies");
  for (int i = 0; i < n_e; ++i)
    if (!(E[i] > 0) || !std::isfinite(E[i])) throw Error(PPM_E_INVALID, "energy grid: energies must be positive");
  Grid g;
  g.E.assign(E, E + n_e);
  PPM_CUDA(cudaSetDevice(cfg.device));
  g.dE = dev_upload(E, n_e);
  std::vector<double> inv(n_e);
  for (int i = 0; i < n_e; ++i) inv[i] = 1.0 / E[i];
  g.dinvE = dev_upload(inv.data(), n_e);
  track(g.dE);
  track(g.dinvE);
  grids.push_back(std::move(g));
  return (int)grids.size() - 1;
}

void split_grid(const std::vector<double>& E, double inv_dE, GridSplit& o) {
  const int n = (int)E.size();
  std::vector<int> iE(n);
  o.rE.assign(n, 0);
  o.fE.assign(n, 0.0f);
  double lo = 1e300, hi = -1e300;
  int imin = 1 << 30, imax = -(1 << 30);
  for (int i = 0; i < n; ++i) {
    double t = std::log10(E[i]) * inv_dE;
    double fl = std::floor(t);
    iE[i] = (int)fl;
    o.fE[i] = (float)(t - fl);
    if (o.fE[i] >= 1.0f) {  // rounding of the fraction up to 1
      o.fE[i] = 0.0f;
      iE[i] += 1;
    }
    lo = std::min(lo, t);
    hi = std::max(hi, t);
    imin = std::min(imin, iE[i]);
    imax = std::max(imax, iE[i]);
  }
  for (int i = 0; i < n; ++i) o.rE[i] = iE[i] - imin;
  o.iE_min = imin;
  o.span = imax - imin + 1;
  o.lo = lo;
  o.hi = hi;
  // energies grouped by home cell, ascending fraction inside a cell
  o.perm.resize(n);
  for (int i = 0; i < n; ++i) o.perm[i] = i;
  std::stable_sort(o.perm.begin(), o.perm.end(), [&](int a, int b) {
    return o.rE[a] != o.rE[b] ? o.rE[a] < o.rE[b] : o.fE[a] < o.fE[b];
  });
  o.fEs.resize(n);
  for (int i = 0; i < n; ++i) o.fEs[i] = o.fE[o.perm[i]];
  o.cell_first.assign(o.span + 1, 0);
  for (int i = 0; i < n; ++i) o.cell_first[o.rE[i] + 1] += 1;
  o.maxe = 0;
  for (int r = 0; r < o.span; ++r) {
    o.maxe = std::max(o.maxe, o.cell_first[r + 1]);
    o.cell_first[r + 1] += o.cell_first[r];
  }
}

// Per-energy split of t_E = log10(E) (n_E - 1)/(logEkT_max - logEkT_min) for the loaded NSX axis.
void Engine::prepare_grid(int id) {
  Grid& g = grids[id];
  if (!has_nsx) return;
  if (g.nsx_version == nsx_version) return;
  GridSplit sp;
  split_grid(g.E, nsx.inv_dE, sp);
  const int n = (int)g.E.size();
  for (void* q : {(void*)g.drE, (void*)g.dfE, (void*)g.dperm, (void*)g.dfEs, (void*)g.dcell_first})
    if (q) cudaFree(q);
  g.drE = dev_upload(sp.rE.data(), n);
  g.dfE = dev_upload(sp.fE.data(), n);
  g.dperm = dev_upload(sp.perm.data(), n);
  g.dfEs = dev_upload(sp.fEs.data(), n);
  g.dcell_first = dev_upload(sp.cell_first.data(), sp.cell_first.size());
  g.maxe = sp.maxe;
  g.iE_min = sp.iE_min;
  g.span = sp.span;
  g.tE_lo = sp.lo;
  g.tE_hi = sp.hi;
  g.nsx_version = nsx_version;
}

DevGrid Engine::dev_grid(int id) {
  Grid& g = grids[id];
  DevGrid d{};
  d.n_e = (int)g.E.size();
  d.iE_min = g.iE_min;
  d.span = g.span;
  d.tE_lo = g.tE_lo;
  d.tE_hi = g.tE_hi;
  d.E = g.dE;
  d.invE = g.dinvE;
  d.rE = g.drE;
  d.fE = g.dfE;
  d.perm = g.dperm;
  d.fEs = g.dfEs;
  d.cell_first = g.dcell_first;
  d.maxe = g.maxe;
  return d;
}

int Engine::add_response(int grid, int n_ch, const double* rsp) {
  if (grid < 0 || grid >= (int)grids.size()) throw Error(PPM_E_INVALID, "response: unknown energy grid");
  if (n_ch < 1 || !rsp) throw Error(PPM_E_INVALID, "response: need channels and a matrix");
  if (n_ch > 8192) throw Error(PPM_E_RANGE, "response: at most 8192 channels");
  PPM_CUDA(cudaSetDevice(cfg.device));
  Resp r;
  r.grid = grid;
  r.n_ch = n_ch;
  r.n_e = (int)grids[grid].E.size();
  r.d_rsp = dev_upload(rsp, (size_t)n_ch * r.n_e);
  track(r.d_rsp);
  r.h_rsp.assign(rsp, rsp + (size_t)n_ch * r.n_e);
  fold_tc_prepare(r);
  resps.push_back(std::move(r));
  return (int)resps.size() - 1;
}

// (z, cos(acos z), sin(acos z)) of every ring, computed with the host libm as
// the reference's GenerateHealpixGrid does (cpu/grid.hpp:219-244,254).
void compute_ring_rows(int N, std::vector<double>& h) {
  h.assign(3 * (size_t)4 * N, 0.0);
  for (int i = 1; i <= 4 * N - 1; ++i) {
    int ii = i > 2 * N ? 4 * N - i : i;
    double z = ii < N ? 1. - 1. * ii * ii / (3. * N * N) : 4. / 3. - 2. * ii / (3. * N);
    if (i > 2 * N) z = -z;
    double th = std::acos(z);
    h[3 * i] = z;
    h[3 * i + 1] = std::cos(th);
    h[3 * i + 2] = std::sin(th);
  }
}

void compute_fine_rows(int nf, std::vector<double>& h) {
  h.resize(kFineStride * (size_t)nf);
  for (int k = 0; k < nf; ++k) {
    double phase = 1. * k / nf;
    double spot_phi = two_pi * phase;
    h[kFineStride * k] = std::cos(spot_phi);
    h[kFineStride * k + 1] = std::sin(spot_phi);
    h[kFineStride * k + 2] = phase;  // the sweep's phase, the same IEEE division as on the device
  }
}

const double* Engine::ring_table(int N) {
  auto it = ring_tabs.find(N);
  if (it != ring_tabs.end()) return it->second;
  std::vector<double> h;
  compute_ring_rows(N, h);
  host_rings[N] = h;
  double* d = dev_upload(h.data(), h.size());
  ring_tabs[N] = d;
  return d;
}

// (cos, sin) of 2 pi k / n_fine and k / n_fine (cpu/devarshi24st_cpu.cpp:131-134).
const double* Engine::fine_table(int nf) {
  auto it = fine_tabs.find(nf);
  if (it != fine_tabs.end()) return it->second;
  std::vector<double> h;
  compute_fine_rows(nf, h);
  double* d = dev_upload(h.data(), h.size());
  fine_tabs[nf] = d;
  return d;
}

// ---- parameters -----------------------------------------------------------------
void Engine::validate(const ppm_params& p) const {
  if (!has_lens) throw Error(PPM_E_STATE, "lensing tables not loaded");
  if (p.n_spots < 1 || p.n_spots > 2) throw Error(PPM_E_INVALID, "n_spots must be 1 or 2");
  if (p.atmosphere != PPM_ATM_NSX && p.atmosphere != PPM_ATM_BLACKBODY) throw Error(PPM_E_INVALID, "unknown atmosphere");
  if (p.atmosphere == PPM_ATM_NSX && !has_nsx) throw Error(PPM_E_STATE, "NSX table not loaded");
  if (p.atmosphere == PPM_ATM_NSX && p.precision != PPM_PREC_FP32)
    throw Error(PPM_E_INVALID, "the NSX integrand runs in FP32 (precision must be PPM_PREC_FP32)");
  if (p.interp < 0 || p.interp > 4) throw Error(PPM_E_INVALID, "unknown NSX interpolator");
  if (p.atmosphere == PPM_ATM_NSX && (p.interp <= 2) && (nsx.nT < 4 || nsx.ng < 4))
    throw Error(PPM_E_RANGE, "cubic logT/logg interpolation needs >= 4 points on both axes");
  if (p.beaming < 0 || p.beaming > 2) throw Error(PPM_E_INVALID, "unknown beaming");
  if (p.precision != PPM_PREC_FP32 && p.precision != PPM_PREC_FP64) throw Error(PPM_E_INVALID, "unknown precision");
  if (p.fold < 0 || p.fold > 2) throw Error(PPM_E_INVALID, "unknown fold");
  if (p.n_side < 1 || p.n_side > 8192) throw Error(PPM_E_RANGE, "n_side must be in [1, 8192]");
  if (p.n_bins < 1 || p.n_bins > 4096) throw Error(PPM_E_RANGE, "n_bins must be in [1, 4096]");
  if (p.n_gl < 0 || p.n_gl > 6) throw Error(PPM_E_RANGE, "n_gl must be in [0, 6] (cpu/gl.hpp)");
  if (p.n_fine < 2 || p.n_fine > 4096) throw Error(PPM_E_RANGE, "n_fine must be in [2, 4096]");
  if (p.energy_grid < 0 || p.energy_grid >= (int)grids.size()) throw Error(PPM_E_INVALID, "unknown energy grid");
  if (p.response >= (int)resps.size() || p.response < -1) throw Error(PPM_E_INVALID, "unknown response");
  if (p.response >= 0 && resps[p.response].grid != p.energy_grid)
    throw Error(PPM_E_INVALID, "response is defined on another energy grid");
  if (!(p.mass_msun > 0) || !(p.r_eq_km > 0) || !(p.spin_hz >= 0) || !(p.distance_kpc > 0))
    throw Error(PPM_E_INVALID, "mass, radius and distance must be positive");
  if (!(p.mass_msun * schwarzschild_radius_of_sun_in_km < p.r_eq_km))
    throw Error(PPM_E_RANGE, "star inside its Schwarzschild radius");
  for (int s = 0; s < p.n_spots; ++s) {
    const ppm_spot& sp = p.spots[s];
    if (sp.kind != PPM_SPOT_HEALPIX && sp.kind != PPM_SPOT_POINT) throw Error(PPM_E_INVALID, "unknown spot kind");
    if (p.atmosphere == PPM_ATM_BLACKBODY && !(sp.kT_keV > 0)) throw Error(PPM_E_INVALID, "blackbody spot needs kT_keV > 0");
    if (!std::isfinite(sp.theta1) || !std::isfinite(sp.angrad1) || !std::isfinite(sp.logT))
      throw Error(PPM_E_INVALID, "non-finite spot parameter");
  }
}

void Engine::to_device(const ppm_params& p, DevProfile& d, long long flux_off, unsigned long long* stats) {
  const double* ring = ring_table(p.n_side);
  const double* fine = fine_table(p.n_fine);
  prepare_grid(p.energy_grid);
  fill_profile(p, d, flux_off, stats, ring, fine, dev_grid(p.energy_grid), host_rings[p.n_side]);
}

// Everything of to_device that needs no device allocation: the ring / fine
// tables and the energy grid are passed in.
void Engine::fill_profile(const ppm_params& p, DevProfile& d, long long flux_off, unsigned long long* stats,
                          const double* ring, const double* fine, const DevGrid& grid, const std::vector<double>& rt) {
  std::memset(&d, 0, sizeof(d));
  // cpu/devarshi24st_cpu.cpp:48-74
  const double M = p.mass_msun, Re = p.r_eq_km, frequency_nu = p.spin_hz;
  const double D = p.distance_kpc * kpc_in_km;
  double Rs = M * schwarzschild_radius_of_sun_in_km;
  double ue = Rs / Re;
  double uue = std::sqrt(1. - ue);
  double logg0 = std::log10(M / (Re * Re * uue));
  double logGMsun_s2_km2cm = std::log10(1.32712440041279419E16);
  double Omega_bar = two_pi * frequency_nu * std::sqrt(Re * Re * Re / M) * sqrt_km3_over_s2_GMsun;
  double x = 0.5 * Rs / Re;
  double o2 = Omega_bar * Omega_bar * (-0.788 + 1.030 * x);
  d.Re = Re;
  d.Rs = Rs;
  d.nu = frequency_nu;
  d.o2 = o2;
  d.D2 = D * D;
  d.cos_obs = std::cos(p.inclination_rad);
  d.sin_obs = std::sin(p.inclination_rad);
  d.dOmega_hp = pi / (3. * p.n_side * p.n_side);
  const double c0e = -0.791, c1e = 0.776, c0p = 1.138, c1p = -1.431, d1e = -1.315, d2e = 2.431, f1e = -1.172,
               d1p = 0.653, d2p = -2.864, f1p = 0.975, d160 = 13.47, d260 = -27.13;
  d.ce = c0e + c1e * x;
  d.cp = c0p + c1p * x;
  d.de = d1e * x + d2e * x * x;
  d.fe = f1e * x;
  d.dp = d1p * x + d2p * x * x;
  d.fp = f1p * x;
  d.d60 = d160 * x + d260 * x * x;
  d.Ob2 = Omega_bar * Omega_bar;
  d.Ob4 = d.Ob2 * d.Ob2;
  d.Ob6 = d.Ob4 * d.Ob2;
  d.logg_base = logg0 + logGMsun_s2_km2cm;
  d.n_side = p.n_side;
  d.n_bins = p.n_bins;
  d.n_gl = p.n_gl;
  d.n_fine = p.n_fine;
  d.n_spots = p.n_spots;
  d.atmosphere = p.atmosphere;
  d.interp = p.interp;
  d.beaming = p.beaming;
  d.precision = p.precision;
  d.flux_off = flux_off;
  d.ring = ring;
  d.fine = fine;
  d.grid = grid;
  d.n_e = d.grid.n_e;
  d.stats = stats;
  const bool nsx_atm = p.atmosphere == PPM_ATM_NSX;
  for (int s = 0; s < p.n_spots; ++s) {
    const ppm_spot& sp = p.spots[s];
    DevSpot& o = d.spot[s];
    o.kind = sp.kind;
    // IsInside (cpu/grid.hpp:158-167) evaluates these with the host libm
    o.s1 = std::sin(sp.theta1);
    o.c1 = std::cos(sp.theta1);
    o.ph1 = sp.phi1;
    o.cos_ar1 = std::cos(sp.angrad1);
    o.s2 = std::sin(sp.theta2);
    o.c2 = std::cos(sp.theta2);
    o.ph2 = sp.phi2;
    o.cos_ar2 = std::cos(sp.angrad2);
    double sin_half_ar = std::sin(0.5 * sp.angrad1);
    o.cos_theta_pt = std::cos(sp.theta1);
    o.dOmega_pt = two_pi * 2. * sin_half_ar * sin_half_ar;  // cpu/grid.hpp:19-22
    double logT = sp.logT;
    o.kT = nsx_atm ? std::pow(10, logT) * 8.617333262E-8 : sp.kT_keV;
    o.l10kT = std::log10(o.kT);
    if (nsx_atm)
      o.out_scale = (1.0 / d.D2) * (std::pow(10, 3 * logT) / planck) * std::ldexp(1.0, -nsx.scale_exp);
    else
      o.out_scale = Ibb_constant / d.D2;
    // ring range that can hold elements of disk 1
    if (sp.kind == PPM_SPOT_HEALPIX) {
      // disk 1 lies within |theta - theta1| <= angrad1; one ring of margin on each side
      const int N = p.n_side, nr = 4 * N - 1;
      const double t1 = sp.theta1, r1 = std::fabs(sp.angrad1);
      const bool all = !(t1 >= 0 && t1 <= pi) || r1 >= pi;
      const double zhi = (all || t1 - r1 <= 0) ? 2.0 : std::cos(t1 - r1) + 1e-9;
      const double zlo = (all || t1 + r1 >= pi) ? -2.0 : std::cos(t1 + r1) - 1e-9;
      int ilo = nr + 1, ihi = 0;
      for (int i = 1; i <= nr; ++i) {
        const double z = rt[3 * i];
        if (z <= zhi && z >= zlo) {
          ilo = std::min(ilo, i);
          ihi = std::max(ihi, i);
        }
      }
      if (ilo > ihi) {
        o.i_lo = 1;
        o.i_hi = 0;
      } else {
        o.i_lo = std::max(1, ilo - 1);
        o.i_hi = std::min(nr, ihi + 1);
      }
    }
    if (nsx_atm) {
      // logT taps (cpu/nsx.hpp:174-187 cubic, 250-285 linear)
      double xT = logT, aT;
      int iT;
      o.T_clamped = (xT < nsx.T_min || xT > nsx.T_max) ? 1 : 0;
      if (xT <= nsx.T_min) {
        aT = 0;
        xT = nsx.T_min;
        iT = 0;
      } else if (xT >= nsx.T_max) {
        aT = 1;
        xT = nsx.T_max;
        iT = nsx.nT - 2;
      } else {
        double t = (xT - nsx.T_min) / (nsx.T_max - nsx.T_min) * (nsx.nT - 1);
        iT = (int)t;
        aT = t - iT;
      }
      const bool cubic = p.interp <= 2;
      if (cubic) {
        int i0 = std::min(std::max(iT - 1, 0), nsx.nT - 4);
        auto node = [&](int i) { return nsx.T_min + (nsx.T_max - nsx.T_min) * i / (nsx.nT - 1); };
        double x0 = node(i0), x1 = node(i0 + 1), x2 = node(i0 + 2), x3 = node(i0 + 3);
        o.wT[0] = (xT - x1) * (xT - x2) * (xT - x3) / ((x0 - x1) * (x0 - x2) * (x0 - x3));
        o.wT[1] = (xT - x0) * (xT - x2) * (xT - x3) / ((x1 - x0) * (x1 - x2) * (x1 - x3));
        o.wT[2] = (xT - x0) * (xT - x1) * (xT - x3) / ((x2 - x0) * (x2 - x1) * (x2 - x3));
        o.wT[3] = (xT - x0) * (xT - x1) * (xT - x2) / ((x3 - x0) * (x3 - x1) * (x3 - x2));
        for (int k = 0; k < 4; ++k) o.iT[k] = i0 + k;
        o.nT_taps = 4;
      } else {
        o.iT[0] = iT;
        o.iT[1] = iT + 1;
        o.wT[0] = 1 - aT;
        o.wT[1] = aT;
        o.nT_taps = 2;
      }
    }
  }
}

// ---- batches ----------------------------------------------------------------------
// Converts and uploads n profiles, sizes the work queue and output pools, and
// records the launch shapes; the batch owns all of its device memory.
void Engine::batch_build(BatchImpl& B, int n, const ppm_params* ps, cudaStream_t copy_stream, int ring_begin,
                         int ring_end, int chunk_override) {
  NvtxRange range("batch build");
  if (n < 1) throw Error(PPM_E_INVALID, "empty batch");
  if (ring_begin > ring_end) throw Error(PPM_E_INVALID, "ring window with begin > end");
  if (!B.mem.stream) B.mem.cache = &block_cache;
  if (n > cfg.max_batch) throw Error(PPM_E_RANGE, "batch larger than max_batch");
  PPM_CUDA(cudaSetDevice(cfg.device));
  B.n = n;
  B.params.assign(ps, ps + n);
  B.flux_off.assign(n + 1, 0);
  B.counts_off.assign(n + 1, 0);
  for (int i = 0; i < n; ++i) {
    validate(ps[i]);
    ring_table(ps[i].n_side);
    const long long ne = (long long)grids[ps[i].energy_grid].E.size();
    B.flux_off[i + 1] = B.flux_off[i] + (long long)ps[i].n_bins * ne;
    const long long nc = ps[i].response >= 0 ? (long long)resps[ps[i].response].n_ch * ps[i].n_bins : 0;
    B.counts_off[i + 1] = B.counts_off[i] + nc;
  }
  // kernel variants, one group and integrand launch each: 0 = NSX home-cell kernel, 1 = blackbody FP64,
  // 2 = blackbody FP32, 3 = NSX pooled-polynomial kernel (grids the home-cell kernel does not take), 4 = NSX
  // home-cell kernel for grids with at most two energies in an NSX cell (half the energy slots of variant 0)
  std::map<int, bool> cell_ok;  // per energy grid
  auto variant = [&](const ppm_params& p) -> int {
    if (p.atmosphere != PPM_ATM_NSX) return p.precision == PPM_PREC_FP64 ? 1 : 2;
    auto it = cell_ok.find(p.energy_grid);
    if (it == cell_ok.end()) it = cell_ok.emplace(p.energy_grid, cell_kernel_takes(p.energy_grid)).first;
    if (!it->second) return 3;
    return grids[p.energy_grid].maxe <= 2 ? 4 : 0;
  };
  constexpr int NV = 5;
  std::vector<int> order, vof(n);
  order.reserve(n);
  for (int i = 0; i < n; ++i) vof[i] = variant(ps[i]);
  for (int v = 0; v < NV; ++v)
    for (int i = 0; i < n; ++i)
      if (vof[i] == v) order.push_back(i);
  // ring bits per profile and spot (rings 0 .. 4 N_side - 1)
  std::vector<long long> ring_off(n + 1, 0);
  for (int i = 0; i < n; ++i) ring_off[i + 1] = ring_off[i] + (long long)kMaxSpots * (4ll * ps[i].n_side / 32 + 1);
  B.ring_words = ring_off[n];
  // the counters, the ring bits and the queue control words in one block (cleared by one memset per pass)
  const size_t stats_bytes = sizeof(unsigned long long) * kStats * (size_t)n;
  const size_t ring_bytes = (sizeof(unsigned) * (size_t)B.ring_words + 63) / 64 * 64;
  B.small_bytes = stats_bytes + ring_bytes + sizeof(int) * 16;
  unsigned char* small = (unsigned char*)B.mem.alloc(B.small_bytes);
  B.d_stats = (unsigned long long*)small;
  B.d_ring_seen = (unsigned*)(small + stats_bytes);
  B.d_ctrl = (int*)(small + stats_bytes + ring_bytes);
  std::vector<DevProfile> hp(n);
  GroupWork gw[NV];
  for (int k = 0; k < n; ++k) {
    const int i = order[k];
    to_device(ps[i], hp[k], B.flux_off[i], B.d_stats + (size_t)kStats * i);
    hp[k].ring_seen = B.d_ring_seen + ring_off[i];
    hp[k].ring_words = (int)(4ll * ps[i].n_side / 32 + 1);
    for (int s = 0; s < ps[i].n_spots; ++s) {  // ring window (a point source is ring 0)
      DevSpot& sp = hp[k].spot[s];
      if (sp.kind == PPM_SPOT_POINT) {
        if (!(ring_begin <= 0 && 0 < ring_end)) {
          sp.i_lo = 1;
          sp.i_hi = 0;
        }
      } else {
        sp.i_lo = std::max(sp.i_lo, ring_begin);
        sp.i_hi = std::min(sp.i_hi, ring_end - 1);
      }
    }
    gw[vof[i]].add(ps[i], hp[k]);
  }
  int chunk[NV], npt[NV];
  for (int v = 0; v < NV; ++v) group_tiling(v == 3, gw[v], chunk_override, &chunk[v], &npt[v]);
  B.chunk = chunk[0];
  long long cap[NV] = {0, 0, 0, 0, 0};
  int start[NV + 1] = {0, 0, 0, 0, 0, 0};
  for (int k = 0; k < n; ++k) {
    const int i = order[k];
    const int v = vof[i];
    cap[v] += tile_bound(ps[i], hp[k], chunk[v], npt[v]);
    start[v + 1] = k + 1;
  }
  for (int v = 1; v <= NV; ++v) start[v] = std::max(start[v], start[v - 1]);
  long long cap_total = 0;
  for (int v = 0; v < NV; ++v) cap_total += cap[v];
  if (cap_total > (1ll << 31) - 1) throw Error(PPM_E_RANGE, "batch too large for one work queue");
  B.d_prof = (DevProfile*)B.mem.alloc(sizeof(DevProfile) * (size_t)n);
  // the flux pool and its compensation pool in one block (cleared by one memset per pass)
  B.d_flux = (double*)B.mem.alloc(2 * sizeof(double) * (size_t)std::max(1ll, B.flux_off[n]));
  B.d_comp = B.d_flux + std::max(1ll, B.flux_off[n]);
  B.d_counts = (double*)B.mem.alloc(sizeof(double) * (size_t)std::max(1ll, B.counts_off[n]));
  Tile* tiles = (Tile*)B.mem.alloc(sizeof(Tile) * (size_t)std::max(1ll, cap_total));
  // uploads: from the caller's pinned area when it has room (asynchronous), else from the pageable source (the
  // copy returns once the source is staged, ordered on the batch's stream), else synchronous
  size_t staged = 0;
  auto upload = [&](void* dst, const void* src, size_t bytes) {
    if (copy_stream && B.h_upload && staged + bytes <= B.h_upload_cap) {
      unsigned char* h = (unsigned char*)B.h_upload + staged;
      std::memcpy(h, src, bytes);
      staged += (bytes + 255) & ~(size_t)255;
      PPM_CUDA(cudaMemcpyAsync(dst, h, bytes, cudaMemcpyHostToDevice, copy_stream));
    } else if (copy_stream) {
      PPM_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, copy_stream));
    } else {
      PPM_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
    }
  };
  upload(B.d_prof, hp.data(), sizeof(DevProfile) * (size_t)n);
  B.h2d_bytes = sizeof(DevProfile) * (size_t)n;
  long long base = 0;
  B.groups.clear();
  for (int v = 0; v < NV; ++v) {
    const int g0 = start[v], g1 = start[v + 1];
    if (g1 <= g0) continue;
    BatchImpl::Group G;
    G.g0 = g0;
    G.g1 = g1;
    G.chunk = chunk[v];
    G.npt = npt[v];
    WorkQueue& q = G.args.queue;
    q.tiles = tiles + base;
    q.capacity = (int)cap[v];
    q.n_tiles = B.d_ctrl + 3 * v;
    q.next = B.d_ctrl + 3 * v + 1;
    q.overflow = B.d_ctrl + 3 * v + 2;
    base += cap[v];
    int ne_max = 1, nf_max = 2, cells_max = 2, maxe_max = 0, bins_max = 0;
    for (int k = g0; k < g1; ++k) {
      ne_max = std::max(ne_max, hp[k].n_e);
      nf_max = std::max(nf_max, hp[k].n_fine);
      cells_max = std::max(cells_max, hp[k].grid.span + 1);
      maxe_max = std::max(maxe_max, hp[k].grid.maxe);
      bins_max = std::max(bins_max, hp[k].n_bins);
    }
    G.args.profiles = B.d_prof + g0;
    G.args.lens = lens;
    G.args.nsx = nsx;
    G.args.flux = B.d_flux;
    G.args.comp = B.d_comp;
    G.args.shape =
        choose_shape(v == 0 || v == 3 || v == 4, v == 1, ne_max, nf_max, cells_max, maxe_max, bins_max,
                     v == 0 || v == 4, gw[v].rings);
    if ((v == 0 || v == 4) && !G.args.shape.cellk)
      throw Error(PPM_E_STATE, "home-cell NSX kernel expected for the grid");
    PPM_CUDA(configure_integrand_smem(G.args.shape));
    const int occ = max_active_ctas(G.args.shape);
    if (occ < 1)
      throw Error(PPM_E_RANGE, "integrand launch shape does not fit on an SM (" + std::to_string(G.args.shape.total) +
                                   " bytes of shared memory)");
    G.grid = (int)std::min<long long>((long long)sm_count * occ, std::max(1ll, cap[v]));
    B.groups.push_back(G);
  }
  // fused point-source mode: one blackbody group, every spot a point source taking the phase-major walk,
  // at most two flux additions per (bin, energy), so that plain additions give the compensated sum's bits
  B.fused_points = B.groups.size() == 1 && (vof[0] == 1 || vof[0] == 2);
  for (int i = 0; i < n && B.fused_points; ++i) {
    const ppm_params& q = ps[i];
    bool points = q.n_spots >= 1;
    for (int k = 0; k < q.n_spots; ++k) points &= q.spots[k].kind == PPM_SPOT_POINT;
    B.fused_points = points && (long long)grids[q.energy_grid].E.size() <= 4 && q.n_spots * std::max(1, q.n_gl) <= 2;
  }
  if (B.fused_points) {
    BatchImpl::Group& G = B.groups[0];
    G.args.n_fused = n;
    G.args.comp = nullptr;
    G.grid = n;
    // the queue control words are never written by a fused pass: zero once, for the collect's overflow check
    // (a synchronous copy when there is no copy stream, complete before the batch is launched on any stream)
    const int zeros[16] = {0};
    upload(B.d_ctrl, zeros, sizeof(zeros));
  }
  // folds grouped by (response, n_bins, arithmetic)
  std::map<std::tuple<int, int, int>, std::vector<FoldJob>> folds;
  for (int i = 0; i < n; ++i) {
    if (ps[i].response < 0) continue;
    FoldJob j{B.flux_off[i], B.counts_off[i], ps[i].exposure_s * (1. / ps[i].n_bins)};
    folds[std::make_tuple(ps[i].response, ps[i].n_bins, ps[i].fold)].push_back(j);
  }
  std::vector<FoldJob> jobs;
  B.folds.clear();
  for (auto& kv : folds) {
    BatchImpl::Fold f{std::get<0>(kv.first), std::get<1>(kv.first), std::get<2>(kv.first), (int)jobs.size(),
                      (int)kv.second.size()};
    B.folds.push_back(f);
    jobs.insert(jobs.end(), kv.second.begin(), kv.second.end());
  }
  if (!jobs.empty()) {
    B.d_jobs = (FoldJob*)B.mem.alloc(sizeof(FoldJob) * jobs.size());
    upload(B.d_jobs, jobs.data(), sizeof(FoldJob) * jobs.size());
    B.h2d_bytes += sizeof(FoldJob) * jobs.size();
  }
}

// One pass: clear outputs and queue, plan, integrate, fold.  With `events`,
// records events[0..3] around the phases.
void Engine::batch_enqueue(BatchImpl& B, cudaStream_t st, cudaEvent_t* events) {
  const int n = B.n;
  if (events) PPM_CUDA(cudaEventRecord(events[0], st));
  if (!B.fused_points) {
    NvtxRange range("clear + plan");
    PPM_CUDA(cudaMemsetAsync(B.d_flux, 0, 2 * sizeof(double) * (size_t)std::max(1ll, B.flux_off[n]), st));
    PPM_CUDA(cudaMemsetAsync(B.d_stats, 0, B.small_bytes, st));
    for (const auto& G : B.groups)
      PPM_CUDA(launch_plan(B.d_prof + G.g0, G.g1 - G.g0, lens, G.args.queue, G.chunk, G.npt, st));
  }
  if (events) PPM_CUDA(cudaEventRecord(events[1], st));
  {
    NvtxRange range("integrand");
    for (const auto& G : B.groups) PPM_CUDA(launch_integrand(G.args, G.grid, st));
    // the compensation pool's rounding errors back into the flux pool (a fused pass adds plainly)
    if (!B.fused_points) PPM_CUDA(launch_add_comp(B.d_flux, B.d_comp, B.flux_off[n], sm_count, st));
  }
  if (events) PPM_CUDA(cudaEventRecord(events[2], st));
  NvtxRange fold_range("fold");
  for (const auto& f : B.folds) {
    const Resp& r = resps[f.resp];
    const FoldJob* jobs = B.d_jobs + f.job0;
    if (f.mode == PPM_FOLD_BF16X3 && r.tc_ok)
      PPM_CUDA(fold_tc_launch(r, jobs, f.n_jobs, f.n_bins, B.d_flux, B.d_counts, st));
    else
      PPM_CUDA(launch_fold_simt(jobs, f.n_jobs, r.d_rsp, r.n_ch, r.n_e, f.n_bins, B.d_flux, B.d_counts,
                                f.mode != PPM_FOLD_FP32, st));
  }
  if (events) PPM_CUDA(cudaEventRecord(events[3], st));
}

void Engine::batch_launch_timed(BatchImpl& B, cudaStream_t st, float* ms) {
  std::lock_guard<std::mutex> lk(mu);
  PPM_CUDA(cudaSetDevice(cfg.device));
  if (!st) st = stream;
  batch_enqueue(B, st, ev);
  B.last_stream = st;
  PPM_CUDA(cudaEventSynchronize(ev[3]));
  for (int k = 0; k < 3; ++k) PPM_CUDA(cudaEventElapsedTime(&ms[k], ev[k], ev[k + 1]));
}

int Engine::kernels_per_pass(const BatchImpl& B) const {
  if (B.fused_points) return 1 + (int)B.folds.size();          // the fused integrand, folds
  return 2 * (int)B.groups.size() + 1 + (int)B.folds.size();  // plan + integrand per group, add_comp, folds
}

void Engine::batch_capture(BatchImpl& B) {
  cudaStream_t cs;
  PPM_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    try {
      batch_enqueue(B, cs, nullptr);
    } catch (...) {
      cudaStreamEndCapture(cs, &g);
      if (g) cudaGraphDestroy(g);
      cudaStreamDestroy(cs);
      throw;
    }
    e = cudaStreamEndCapture(cs, &g);
  }
  cudaStreamDestroy(cs);
  if (e != cudaSuccess) throw Error(PPM_E_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
  e = cudaGraphInstantiate(&B.graph, g, 0);
  cudaGraphDestroy(g);
  if (e != cudaSuccess) throw Error(PPM_E_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
}

void Engine::batch_launch(BatchImpl& B, cudaStream_t st) {
  PPM_CUDA(cudaSetDevice(cfg.device));
  if (!st) st = stream;
  if (!B.graph) batch_capture(B);
  PPM_CUDA(cudaGraphLaunch(B.graph, st));
  B.last_stream = st;
}

void Engine::batch_collect(BatchImpl& B, double* flux, double* counts, ppm_result_info* info, cudaStream_t st) {
  NvtxRange range("collect");
  PPM_CUDA(cudaSetDevice(cfg.device));
  if (!st) st = B.last_stream ? B.last_stream : stream;
  const int n = B.n;
  std::vector<unsigned long long> stats((size_t)kStats * n);
  int ctrl[16];
  if (flux)
    PPM_CUDA(cudaMemcpyAsync(flux, B.d_flux, sizeof(double) * (size_t)B.flux_off[n], cudaMemcpyDeviceToHost, st));
  if (counts && B.counts_off[n] > 0)
    PPM_CUDA(cudaMemcpyAsync(counts, B.d_counts, sizeof(double) * (size_t)B.counts_off[n], cudaMemcpyDeviceToHost, st));
  PPM_CUDA(cudaMemcpyAsync(stats.data(), B.d_stats, sizeof(unsigned long long) * stats.size(), cudaMemcpyDeviceToHost,
                           st));
  PPM_CUDA(cudaMemcpyAsync(ctrl, B.d_ctrl, sizeof(ctrl), cudaMemcpyDeviceToHost, st));
  PPM_CUDA(cudaStreamSynchronize(st));
  PPM_CUDA(cudaGetLastError());
  if (ctrl[2] || ctrl[5] || ctrl[8] || ctrl[11] || ctrl[14]) throw Error(PPM_E_RANGE, "work queue overflow");
  int err = 0;
  PPM_CUDA(cudaMemcpy(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) {
    PPM_CUDA(cudaMemset(d_err, 0, sizeof(int)));
    throw Error(PPM_E_TIMEOUT, "a bounded wait in the tensor-core fold ran out");
  }
  if (info) {
    for (int i = 0; i < n; ++i) {
      ppm_result_info& r = info[i];
      const unsigned long long* s = &stats[(size_t)kStats * i];
      r.n_active = (int64_t)(s[0] + s[5]);
      r.n_rings = (int64_t)s[1];
      r.n_dropped_rings = (int64_t)s[2];
      r.n_points = (int64_t)s[3];
      r.n_clamped = (int64_t)s[4];
      r.n_active_integrated = (int64_t)s[0];
      r.status = PPM_OK;
      r.reserved = 0;
    }
  }
}

void Engine::profile(const ppm_params& p, double* flux, double* counts, ppm_result_info* info) {
  NvtxRange range("ppm_profile");
  std::lock_guard<std::mutex> lk(mu);
  if (counts && p.response < 0) throw Error(PPM_E_INVALID, "counts requested without a response");
  BatchImpl B;
  batch_build(B, 1, &p);
  batch_enqueue(B, stream, nullptr);  // plain form: direct launches, no graph
  B.last_stream = stream;
  batch_collect(B, flux, counts, info, stream);
}

// HEALPix elements in a profile's spots (disk 1 areas over the element area,
// one per point source): the size of its share of a batch's work.
double Engine::spot_elements(const ppm_params& p) {
  double e = 0;
  for (int s = 0; s < p.n_spots; ++s) {
    const ppm_spot& sp = p.spots[s];
    e += sp.kind == PPM_SPOT_POINT ? 1.0
                                   : 6.0 * p.n_side * (double)p.n_side * (1.0 - std::cos(std::min(std::fabs(sp.angrad1), pi)));
  }
  return e;
}

// Candidate elements per work tile: the tuned size unless one tile (up to
// `chunk` elements x pts_max phase points) would exceed 1/8 of a CTA slot's
// share of the batch's work, then halved down to small_chunk, so that small
// batches, mixed served batches and single profiles end without a long tail.
int Engine::tile_chunk(double work, long long pts_max) const {
  const double share = work / (8.0 * sm_count * 3);
  int c = tune.chunk;
  while (c > tune.small_chunk && (double)c * pts_max > share) c >>= 1;
  return std::max(c, std::min(tune.chunk, tune.small_chunk));
}

void GroupWork::add(const ppm_params& p, const DevProfile& d) {
  const long long pts = (long long)p.n_bins * std::max(1, p.n_gl);
  pts_max = std::max(pts_max, pts);
  nodes_max = std::max(nodes_max, (int)pts);
  ne_max = std::max(ne_max, d.n_e);
  elements += Engine::spot_elements(p);
  work += Engine::spot_elements(p) * (double)pts;
  for (int s = 0; s < p.n_spots; ++s) {
    const DevSpot& sp = d.spot[s];
    if (sp.kind == PPM_SPOT_POINT)
      rings += sp.i_hi >= sp.i_lo ? 1 : 0;
    else if (sp.i_hi >= sp.i_lo)
      rings += sp.i_hi - sp.i_lo + 1;
  }
}

// Tiling of one kernel group.  The home-cell NSX and the blackbody kernels
// keep the tuned element chunk in every batch, so that a profile's tiles cover
// the same elements alone and in any batch; a batch with few rings is spread
// over the SMs by splitting each tile's phase nodes instead: about 8 tiles per
// CTA slot, but every tile keeps at least kMinNodesPerTile nodes and enough
// (element, node, energy) evaluations to outweigh its prologue (the FP64
// fine-phase sweep and the tables it stages, repeated by every tile of a ring).
// The pooled kernel splits the elements (tile_chunk) and takes all nodes.
void Engine::group_tiling(bool pooled, const GroupWork& w, int chunk_override, int* chunk, int* npt) const {
  if (pooled) {
    *chunk = chunk_override > 0 ? chunk_override : tile_chunk(w.work, w.pts_max);
    *npt = 0;
    return;
  }
  *chunk = chunk_override > 0 ? chunk_override : tune.chunk;
  const double rings = std::max<double>(1.0, (double)w.rings);
  const double want = 8.0 * sm_count * 3;
  double splits_d = std::ceil(want / rings);
  // nodes per tile for kMinEvalsPerTile evaluations at the group's mean active elements per ring
  const double per_ring = std::max(1.0, std::min<double>(w.elements / rings, *chunk));
  const double min_nodes = std::max<double>(kMinNodesPerTile, std::ceil(kMinEvalsPerTile / (per_ring * w.ne_max)));
  splits_d = std::min(splits_d, std::floor(w.nodes_max / min_nodes));
  int splits = (int)std::max(1.0, splits_d);
  if (tune.splits > 0) splits = std::min(tune.splits, std::max(1, w.nodes_max));
  *npt = splits <= 1 ? 0 : (w.nodes_max + splits - 1) / splits;
}

// Work tiles the planner may push for one profile (its queue capacity).
long long Engine::tile_bound(const ppm_params& p, const DevProfile& d, int chunk, int npt) const {
  const int nodes = p.n_bins * std::max(1, p.n_gl);
  const long long per = npt > 0 ? (nodes + npt - 1) / npt : 1;
  long long cap = 0;
  for (int s = 0; s < p.n_spots; ++s) {
    const DevSpot& sp = d.spot[s];
    if (sp.kind == PPM_SPOT_POINT)
      cap += sp.i_hi >= sp.i_lo ? per : 0;
    else if (sp.i_hi >= sp.i_lo)
      cap += (long long)(sp.i_hi - sp.i_lo + 1) * (2 + (4ll * p.n_side + chunk - 1) / chunk) * per;
  }
  return cap;
}

// Whether the home-cell NSX kernel takes profiles on this energy grid.
bool Engine::cell_kernel_takes(int grid) {
  if (tune.kernel != 0 || !has_nsx) return false;
  prepare_grid(grid);
  const Grid& g = grids[grid];
  const IntegrandShape s = choose_shape(true, false, (int)g.E.size(), 2, g.span + 1, g.maxe, 1, true);
  return s.cellk != 0;
}

void Engine::profile_rings(const ppm_params& p, int ring_begin, int ring_end, double* flux, double* counts,
                           ppm_result_info* info) {
  std::lock_guard<std::mutex> lk(mu);
  if (counts && p.response < 0) throw Error(PPM_E_INVALID, "counts requested without a response");
  BatchImpl B;
  batch_build(B, 1, &p, nullptr, ring_begin, ring_end);
  batch_enqueue(B, stream, nullptr);
  B.last_stream = stream;
  batch_collect(B, flux, counts, info, stream);
}

void Engine::profile_batch(int n, const ppm_params* ps, double* flux, double* counts, ppm_result_info* info) {
  NvtxRange range("ppm_profile_batch");
  std::lock_guard<std::mutex> lk(mu);
  BatchImpl B;
  batch_build(B, n, ps);
  batch_enqueue(B, stream, nullptr);
  B.last_stream = stream;
  batch_collect(B, flux, counts, info, stream);
}

IntegrandShape Engine::choose_shape(bool nsx_kernel, bool bb_fp64, int ne_max, int nf_max, int cells_max, int maxe_max,
                                    int bins_max, bool allow_cell, double rings) {
  // home-cell NSX kernel: cpl cells per lane (the last (cpl + 3) / cpl lanes of a warp
  // only supply slice rows), warp sets up to 512 threads
  const int span_max = cells_max - 1;
  const int maxe_t = maxe_max <= 2 ? 2 : (maxe_max <= 4 ? 4 : (maxe_max <= 8 ? 8 : 16));
  if (allow_cell && nsx_kernel && tune.kernel == 0 && maxe_max >= 1 && maxe_max <= 16 && span_max <= 16 * 32 &&
      nsx.nmu < 4096 && bins_max < (1 << 20)) {
    // cells per lane: fewest estimated lane instructions per point (window rows,
    // polynomials, record handling, energy slots), over what the slots' registers allow
    const int cmax = maxe_t <= 4 ? 3 : (maxe_t == 8 ? 2 : 1);
    int cpl = 1;
    long best = -1;
    auto cells_per_warp = [](int c) { return (32 - (c + 3) / c) * c; };  // lanes with home cells x c
    for (int c = 1; c <= cmax; ++c) {
      const long w = (span_max + cells_per_warp(c) - 1) / cells_per_warp(c);
      if (w > 16) continue;
      const long cost = w * (20 * (c + 1) + 30 + 11L * maxe_t * c);
      if (best < 0 || cost < best) {
        best = cost;
        cpl = c;
      }
    }
    if (tune.cpl > 0) cpl = std::min(tune.cpl, cmax);
    const int cell_warps = (span_max + cells_per_warp(cpl) - 1) / cells_per_warp(cpl);
    if (best >= 0 && cell_warps <= 16) {
      // default: about 256 threads (three CTAs of 80 registers per SM measured fastest)
      int sets = std::min(16 / cell_warps, tune.sets > 0 ? tune.sets : std::max(1, 8 / cell_warps));
      IntegrandShape s;
      for (;;) {
        const int nt = 32 * cell_warps * sets;
        s = make_shape(true, nt, 1, 1, tune.chunk, nf_max, lens.n_cp, lens.n_ca, nsx.nE, nsx.nmu, cells_max, true);
        if (s.total <= 200 * 1024 || sets == 1) break;
        --sets;
      }
      s.bb_fp64 = 0;
      s.cell_warps = cell_warps;
      s.cpl = cpl;
      s.maxe_t = maxe_t;
      s.minb = maxe_t <= 8 ? tune.minb : 1;
      return s;
    }
  }
  int ne_t = 1;
  if (ne_max > 512)
    ne_t = 4;
  else if (ne_max > 320)
    ne_t = 2;
  if (tune.ne_t > 0 && tune.ne_t * 512 >= ne_max) ne_t = tune.ne_t;
  int nt = (ne_max + ne_t - 1) / ne_t;
  nt = (nt + 31) / 32 * 32;
  nt = std::max(64, std::min(512, nt));
  // few energies: the blackbody kernel evaluates one phase point per thread
  // (its point-wise path, n_e * 4 <= threads), so size the block by points.
  // The phase-major walk (4 energies or fewer) takes 512 threads, more
  // segments of a ring in flight and half as many CTA slots to fill, unless
  // the batch has rings enough to fill the slots of 256-thread blocks (four
  // per SM); then 256, each ring's prologue shared by half as many threads.
  // Measured on one-profile light curves: 427 rings run faster with 512
  // threads, 671 rings with 256.
  if (!nsx_kernel && ne_max * 4 <= 256) {
    const bool many_rings = rings >= 4.0 * sm_count;
    nt = tune.bb_nt > 0 ? tune.bb_nt : (ne_max <= 4 && !many_rings ? 512 : 256);
  }
  // whole multiples of the warp count keep the one-warp-per-point build balanced
  const int nwarps = nt / 32;
  int pb = std::max(nwarps, (std::min(tune.pb, nt) / nwarps) * nwarps);
  IntegrandShape s;
  for (;;) {
    s = make_shape(nsx_kernel, nt, ne_t, pb, tune.chunk, nf_max, lens.n_cp, lens.n_ca, nsx.nE, nsx.nmu, cells_max);
    if (s.total <= 200 * 1024 || pb <= nwarps) break;
    pb -= nwarps;
  }
  s.bb_fp64 = bb_fp64 ? 1 : 0;
  s.minb = (ne_t <= 2 && nt <= 320) ? std::min(tune.minb, 2) : 1;
  return s;
}

// Coordinate descent over the integrand's launch shape on a sample batch.
std::string Engine::autotune(int n, const ppm_params* sample) {
  NvtxRange range("autotune");
  std::lock_guard<std::mutex> lk(mu);
  PPM_CUDA(cudaSetDevice(cfg.device));
  const Tuning start = tune;
  auto measure = [&](const Tuning& t) -> float {
    tune = t;
    BatchImpl B;
    batch_build(B, n, sample);
    batch_enqueue(B, stream, nullptr);  // warm-up
    PPM_CUDA(cudaEventRecord(ev[0], stream));
    for (int r = 0; r < 2; ++r) batch_enqueue(B, stream, nullptr);
    PPM_CUDA(cudaEventRecord(ev[1], stream));
    PPM_CUDA(cudaEventSynchronize(ev[1]));
    float ms = 0;
    PPM_CUDA(cudaEventElapsedTime(&ms, ev[0], ev[1]));
    return ms / 2;
  };
  std::string rep;
  auto line = [&](const Tuning& t, float ms, const char* note) {
    char buf[160];
    std::snprintf(buf, sizeof(buf), "pb=%d chunk=%d minb=%d ne_t=%d sets=%d cpl=%d kernel=%d : %.3f ms%s\n", t.pb,
                  t.chunk, t.minb, t.ne_t, t.sets, t.cpl, t.kernel, ms, note);
    rep += buf;
  };
  Tuning best = start;
  float best_ms = measure(best);
  line(best, best_ms, " (start)");
  const std::vector<std::pair<int Tuning::*, std::vector<int>>> dims = {
      {&Tuning::pb, {10, 20, 30, 40}},
      {&Tuning::chunk, {256, 512, 1024, 2048}},
      {&Tuning::minb, {1, 2}},
      {&Tuning::ne_t, {0, 2}},
      {&Tuning::sets, {0, 1, 2, 3, 4}},
      {&Tuning::cpl, {0, 1, 2, 3}},
      {&Tuning::kernel, {0, 1}},
  };
  for (const auto& d : dims) {
    for (int v : d.second) {
      Tuning t = best;
      if (t.*(d.first) == v) continue;
      t.*(d.first) = v;
      float ms;
      try {
        ms = measure(t);
      } catch (const Error& e) {
        line(t, -1.0f, " (does not fit)");
        continue;
      }
      line(t, ms, "");
      if (ms < 0.98f * best_ms) {
        best = t;
        best_ms = ms;
      }
    }
  }
  tune = best;
  line(best, best_ms, " (chosen)");
  return rep;
}

// The fold of given flux arrays, the reference's matmul (gpu/matmul.cuh:12-36)
// on its own: the same kernels as the fold stage of a pass.
void Engine::fold(int resp, int mode, int n_prof, int n_bins, const double* alpha, const double* flux, double* counts,
                  bool device, cudaStream_t st) {
  NvtxRange range("ppm_fold");
  std::lock_guard<std::mutex> lk(mu);
  if (resp < 0 || resp >= (int)resps.size()) throw Error(PPM_E_INVALID, "unknown response");
  if (mode < 0 || mode > 2) throw Error(PPM_E_INVALID, "unknown fold");
  if (n_prof < 1 || n_bins < 1 || n_bins > 4096) throw Error(PPM_E_RANGE, "n_profiles >= 1 and n_bins in [1, 4096]");
  if (!alpha || !flux || !counts) throw Error(PPM_E_INVALID, "null alpha, flux or counts");
  if ((long long)n_prof * n_bins > (1ll << 31) / 2) throw Error(PPM_E_RANGE, "too many (profile, bin) rows");
  PPM_CUDA(cudaSetDevice(cfg.device));
  const Resp& r = resps[resp];
  const size_t n_flux = (size_t)n_prof * n_bins * r.n_e, n_counts = (size_t)n_prof * n_bins * r.n_ch;
  std::vector<FoldJob> jobs(n_prof);
  for (int j = 0; j < n_prof; ++j)
    jobs[j] = FoldJob{(long long)j * n_bins * r.n_e, (long long)j * n_bins * r.n_ch, alpha[j]};
  if (!st) st = stream;
  DeviceArena mem;
  const double* d_flux = flux;
  double* d_counts = counts;
  if (device) {
    mem.stream = st;  // stream-ordered: the job list lives until the fold has read it
  } else {
    mem.cache = &block_cache;
    double* f = (double*)mem.alloc(sizeof(double) * n_flux);
    d_counts = (double*)mem.alloc(sizeof(double) * n_counts);
    PPM_CUDA(cudaMemcpyAsync(f, flux, sizeof(double) * n_flux, cudaMemcpyHostToDevice, st));
    d_flux = f;
  }
  FoldJob* d_jobs = (FoldJob*)mem.alloc(sizeof(FoldJob) * jobs.size());
  PPM_CUDA(cudaMemcpyAsync(d_jobs, jobs.data(), sizeof(FoldJob) * jobs.size(), cudaMemcpyHostToDevice, st));
  if (mode == PPM_FOLD_BF16X3 && r.tc_ok)
    PPM_CUDA(fold_tc_launch(r, d_jobs, n_prof, n_bins, d_flux, d_counts, st));
  else
    PPM_CUDA(launch_fold_simt(d_jobs, n_prof, r.d_rsp, r.n_ch, r.n_e, n_bins, d_flux, d_counts, mode != PPM_FOLD_FP32,
                              st));
  if (!device) {
    PPM_CUDA(cudaMemcpyAsync(counts, d_counts, sizeof(double) * n_counts, cudaMemcpyDeviceToHost, st));
    PPM_CUDA(cudaStreamSynchronize(st));
    int err = 0;
    PPM_CUDA(cudaMemcpy(&err, d_err, sizeof(int), cudaMemcpyDeviceToHost));
    if (err) {
      PPM_CUDA(cudaMemset(d_err, 0, sizeof(int)));
      throw Error(PPM_E_TIMEOUT, "a bounded wait in the tensor-core fold ran out");
    }
  }
}

void Engine::output_sizes(const ppm_params& p, int64_t* n_flux, int64_t* n_counts) const {
  validate(p);
  if (n_flux) *n_flux = (int64_t)p.n_bins * (int64_t)grids[p.energy_grid].E.size();
  if (n_counts) *n_counts = p.response >= 0 ? (int64_t)p.n_bins * resps[p.response].n_ch : 0;
}

}  // namespace ppm
