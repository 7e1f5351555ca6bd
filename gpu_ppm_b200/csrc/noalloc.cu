// Allocation-free form of the plain profile path (ppm_profile_noalloc).
//
// Some callers cannot allocate device memory while they run: a sampler that
// reserves every byte of the GPU for its own pool at start-up, a host
// framework whose caching allocator owns the device, or a real-time loop in
// which cudaMalloc's implicit device synchronisation would stall other
// streams.  For them this entry point keeps all of its working state — the
// converted profile, counters, work-queue control words, the ring and
// fine-phase tables, the per-energy cell split and the work queue itself — in
// one file-scope device array of fixed size, and writes results only into the
// caller's device buffers.
//
// Set-up: the first call on a device looks up the array's device address with
// cudaGetSymbolAddress (once per device, with that device current); make that
// first call before any stream capture.  The array is shared by every call and
// keeps the previous call's contents; whatever must start at zero is cleared
// on the stream by each call, and calls that overlap on the GPU race on it.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/ppm.h"
#include "engine.h"

namespace ppm {

namespace {

constexpr size_t kScratchBytes = 1u << 20;  // 1 MiB per device that loads the library
__device__ __align__(256) unsigned char g_profile_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of g_profile_scratch on `dev` (which must be current).
void* scratch_address(int dev) {
  if (dev < 0 || dev >= kMaxDevices) throw Error(PPM_E_RANGE, "ppm_profile_noalloc: device ordinal out of range");
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  if (!g_scratch_addr[dev]) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_profile_scratch);
    if (e != cudaSuccess)
      throw Error(PPM_E_CUDA, std::string("ppm_profile_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    g_scratch_addr[dev] = p;
  }
  return g_scratch_addr[dev];
}

size_t up256(size_t v) { return (v + 255) / 256 * 256; }

}  // namespace

void Engine::profile_noalloc(const ppm_params& p, double* flux_d, double* counts_d, cudaStream_t st) {
  std::lock_guard<std::mutex> lk(mu);
  validate(p);
  if (!flux_d) throw Error(PPM_E_INVALID, "ppm_profile_noalloc: flux_device is required");
  if (counts_d && p.response < 0) throw Error(PPM_E_INVALID, "ppm_profile_noalloc: counts requested without a response");
  {
    cudaError_t e = cudaSetDevice(cfg.device);
    if (e != cudaSuccess) throw Error(PPM_E_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  }
  if (!st) st = stream;
  unsigned char* base = (unsigned char*)scratch_address(cfg.device);

  const Grid& gr = grids[p.energy_grid];
  const int n_e = (int)gr.E.size();
  const int N = p.n_side, nf = p.n_fine;
  const bool nsx_atm = p.atmosphere == PPM_ATM_NSX;

  // layout of the scratch array
  size_t off = 0;
  const size_t o_prof = off;
  off += up256(sizeof(DevProfile));
  const size_t o_stats = off;
  off += up256(sizeof(unsigned long long) * kStats);
  const size_t o_ctrl = off;
  off += up256(sizeof(int) * 16);
  const size_t o_job = off;
  off += up256(sizeof(FoldJob));
  const size_t o_ring = off;
  off += up256(sizeof(double) * 3 * 4 * (size_t)N);
  const size_t o_fine = off;
  off += up256(sizeof(double) * 2 * (size_t)nf);
  const size_t o_rE = off;
  off += up256(sizeof(int) * (size_t)n_e);
  const size_t o_fE = off;
  off += up256(sizeof(float) * (size_t)n_e);
  const size_t o_tiles = off;
  if (off > kScratchBytes)
    throw Error(PPM_E_RANGE, "ppm_profile_noalloc: N_side " + std::to_string(N) + " / n_fine " + std::to_string(nf) +
                                 " tables exceed the 1 MiB scratch array");
  const long long tile_cap = (long long)((kScratchBytes - off) / sizeof(Tile));

  // host-side rows (host memory only)
  std::vector<double> ring_rows, fine_rows;
  compute_ring_rows(N, ring_rows);
  compute_fine_rows(nf, fine_rows);
  DevGrid g{};
  g.n_e = n_e;
  g.E = gr.dE;
  g.invE = gr.dinvE;
  std::vector<int> rE(n_e, 0);
  std::vector<float> fE(n_e, 0.0f);
  if (nsx_atm) {
    // per-energy split of t_E = log10(E) (n_E - 1)/(logEkT_max - logEkT_min), as prepare_grid
    std::vector<int> iE(n_e);
    double lo = 1e300, hi = -1e300;
    int imin = 1 << 30, imax = -(1 << 30);
    for (int i = 0; i < n_e; ++i) {
      double t = std::log10(gr.E[i]) * nsx.inv_dE;
      double fl = std::floor(t);
      iE[i] = (int)fl;
      fE[i] = (float)(t - fl);
      if (fE[i] >= 1.0f) {
        fE[i] = 0.0f;
        iE[i] += 1;
      }
      lo = std::min(lo, t);
      hi = std::max(hi, t);
      imin = std::min(imin, iE[i]);
      imax = std::max(imax, iE[i]);
    }
    for (int i = 0; i < n_e; ++i) rE[i] = iE[i] - imin;
    g.iE_min = imin;
    g.span = imax - imin + 1;
    g.tE_lo = lo;
    g.tE_hi = hi;
  }
  g.rE = (const int*)(base + o_rE);
  g.fE = (const float*)(base + o_fE);

  DevProfile d;
  unsigned long long* stats = (unsigned long long*)(base + o_stats);
  fill_profile(p, d, 0, stats, (const double*)(base + o_ring), (const double*)(base + o_fine), g, ring_rows);
  // work-queue bound (as in batch_build)
  long long cap = 0;
  for (int s = 0; s < p.n_spots; ++s) {
    const DevSpot& sp = d.spot[s];
    if (sp.kind == PPM_SPOT_POINT)
      cap += 1;
    else if (sp.i_hi >= sp.i_lo)
      cap += (long long)(sp.i_hi - sp.i_lo + 1) * (2 + (4ll * N + tune.chunk - 1) / tune.chunk);
  }
  if (cap > tile_cap)
    throw Error(PPM_E_RANGE, "ppm_profile_noalloc: the profile needs up to " + std::to_string(cap) +
                                 " work tiles, the 1 MiB scratch array holds " + std::to_string(tile_cap) +
                                 " (lower N_side or use ppm_profile)");

  auto ck = [](cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw Error(PPM_E_CUDA, std::string("ppm_profile_noalloc: ") + what + ": " + cudaGetErrorString(e));
  };
  // uploads from pageable host memory return once the data is staged
  ck(cudaMemcpyAsync(base + o_prof, &d, sizeof(DevProfile), cudaMemcpyHostToDevice, st), "profile upload");
  ck(cudaMemcpyAsync(base + o_ring, ring_rows.data(), sizeof(double) * ring_rows.size(), cudaMemcpyHostToDevice, st),
     "ring table upload");
  ck(cudaMemcpyAsync(base + o_fine, fine_rows.data(), sizeof(double) * fine_rows.size(), cudaMemcpyHostToDevice, st),
     "fine-phase table upload");
  ck(cudaMemcpyAsync(base + o_rE, rE.data(), sizeof(int) * n_e, cudaMemcpyHostToDevice, st), "cell index upload");
  ck(cudaMemcpyAsync(base + o_fE, fE.data(), sizeof(float) * n_e, cudaMemcpyHostToDevice, st), "cell fraction upload");
  // state that must start at zero: the caller's flux, the counters and the queue control words
  ck(cudaMemsetAsync(flux_d, 0, sizeof(double) * (size_t)p.n_bins * n_e, st), "flux clear");
  ck(cudaMemsetAsync(base + o_stats, 0, sizeof(unsigned long long) * kStats, st), "counter clear");
  ck(cudaMemsetAsync(base + o_ctrl, 0, sizeof(int) * 16, st), "queue clear");

  int* ctrl = (int*)(base + o_ctrl);
  KernelArgs a{};
  a.profiles = (const DevProfile*)(base + o_prof);
  a.lens = lens;
  a.nsx = nsx;
  a.flux = flux_d;
  WorkQueue& q = a.queue;
  q.tiles = (Tile*)(base + o_tiles);
  q.capacity = (int)cap;
  q.n_tiles = ctrl;
  q.next = ctrl + 1;
  q.overflow = ctrl + 2;
  const bool bb64 = !nsx_atm && p.precision == PPM_PREC_FP64;
  a.shape = choose_shape(nsx_atm, bb64, n_e, nf, g.span + 1);
  ck(configure_integrand_smem(a.shape), "shared-memory attribute");
  const int occ = max_active_ctas(a.shape);
  if (occ < 1) throw Error(PPM_E_RANGE, "ppm_profile_noalloc: launch shape does not fit on an SM");
  ck(launch_plan(a.profiles, 1, lens, q, tune.chunk, st), "plan launch");
  ck(launch_integrand(a, (int)std::min<long long>((long long)sm_count * occ, std::max(1ll, cap)), st),
     "integrand launch");
  if (counts_d) {
    const Resp& r = resps[p.response];
    FoldJob job{0, 0, p.exposure_s * (1. / p.n_bins)};
    ck(cudaMemcpyAsync(base + o_job, &job, sizeof(FoldJob), cudaMemcpyHostToDevice, st), "fold job upload");
    const FoldJob* dj = (const FoldJob*)(base + o_job);
    if (p.fold == PPM_FOLD_BF16X3 && r.tc_ok)
      ck(fold_tc_launch(r, dj, 1, p.n_bins, flux_d, counts_d, st), "fold launch");
    else
      ck(launch_fold_simt(dj, 1, r.d_rsp, r.n_ch, r.n_e, p.n_bins, flux_d, counts_d, p.fold != PPM_FOLD_FP32, st),
         "fold launch");
  }
}

}  // namespace ppm
