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
// first call before any stream capture.  The cached address assumes that the
// device's primary context lives until the process exits (no
// cudaDeviceReset in between).  The array is shared by every call and keeps
// the previous call's contents; whatever must start at zero is cleared on the
// stream by each call, and calls that overlap on the GPU race on it.
//
// The call only enqueues work.  Its own status words (the fold's bounded-wait
// flag, the work-queue overflow flag) and diagnostic counters live in the
// array too; ppm_profile_noalloc_result waits for the stream and reports them
// for the last call.  The call refuses a stream that is being captured: its
// uploads come from host memory that is released when it returns.
#include <cuda_runtime.h>

#include <algorithm>
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

// Fixed head of the scratch array: the converted profile, the counters, the
// work-queue control words and the status words; variable-size tables follow.
struct ScratchHead {
  size_t prof, stats, ctrl, status, job, end;
};
ScratchHead scratch_head() {
  ScratchHead h{};
  size_t off = 0;
  h.prof = off;
  off += up256(sizeof(DevProfile));
  h.stats = off;
  off += up256(sizeof(unsigned long long) * kStats);
  h.ctrl = off;
  off += up256(sizeof(int) * 16);
  h.status = off;
  off += up256(sizeof(int) * 4);
  h.job = off;
  off += up256(sizeof(FoldJob));
  h.end = off;
  return h;
}

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
  {
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaError_t e = cudaStreamIsCapturing(st, &cap);
    if (e != cudaSuccess) throw Error(PPM_E_CUDA, std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(e));
    if (cap != cudaStreamCaptureStatusNone)
      throw Error(PPM_E_STATE, "ppm_profile_noalloc: the stream is being captured (the uploads come from host memory "
                               "that is released when the call returns)");
  }
  unsigned char* base = (unsigned char*)scratch_address(cfg.device);

  const Grid& gr = grids[p.energy_grid];
  const int n_e = (int)gr.E.size();
  const int N = p.n_side, nf = p.n_fine;
  const bool nsx_atm = p.atmosphere == PPM_ATM_NSX;

  // layout of the scratch array: the fixed head, then the tables and the work queue
  const ScratchHead hd = scratch_head();
  size_t off = hd.end;
  const size_t o_prof = hd.prof, o_stats = hd.stats, o_ctrl = hd.ctrl, o_status = hd.status, o_job = hd.job;
  const size_t o_ring = off;
  off += up256(sizeof(double) * 3 * 4 * (size_t)N);
  const size_t o_fine = off;
  off += up256(sizeof(double) * kFineStride * (size_t)nf);
  GridSplit split;
  if (nsx_atm) split_grid(gr.E, nsx.inv_dE, split);
  const size_t n_cf = nsx_atm ? split.cell_first.size() : 1;
  const size_t o_rE = off;
  off += up256(sizeof(int) * (size_t)n_e);
  const size_t o_fE = off;
  off += up256(sizeof(float) * (size_t)n_e);
  const size_t o_perm = off;
  off += up256(sizeof(int) * (size_t)n_e);
  const size_t o_fEs = off;
  off += up256(sizeof(float) * (size_t)n_e);
  const size_t o_cf = off;
  off += up256(sizeof(int) * n_cf);
  const int ring_words = 4 * N / 32 + 1;
  const size_t o_rseen = off;
  off += up256(sizeof(unsigned) * kMaxSpots * (size_t)ring_words);
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
  if (nsx_atm) {
    // per-energy split of t_E = log10(E) (n_E - 1)/(logEkT_max - logEkT_min), as prepare_grid
    g.iE_min = split.iE_min;
    g.span = split.span;
    g.tE_lo = split.lo;
    g.tE_hi = split.hi;
    g.maxe = split.maxe;
  } else {
    split.rE.assign(n_e, 0);
    split.fE.assign(n_e, 0.0f);
    split.perm.assign(n_e, 0);
    split.fEs.assign(n_e, 0.0f);
    split.cell_first.assign(1, 0);
  }
  g.rE = (const int*)(base + o_rE);
  g.fE = (const float*)(base + o_fE);
  g.perm = (const int*)(base + o_perm);
  g.fEs = (const float*)(base + o_fEs);
  g.cell_first = (const int*)(base + o_cf);

  DevProfile d;
  unsigned long long* stats = (unsigned long long*)(base + o_stats);
  fill_profile(p, d, 0, stats, (const double*)(base + o_ring), (const double*)(base + o_fine), g, ring_rows);
  d.ring_seen = (unsigned*)(base + o_rseen);
  d.ring_words = ring_words;
  // kernel and tiling as batch_build gives a one-profile batch
  const bool bb64 = !nsx_atm && p.precision == PPM_PREC_FP64;
  IntegrandShape shape = choose_shape(nsx_atm, bb64, n_e, nf, g.span + 1, g.maxe, p.n_bins);
  const bool pooled = nsx_atm && !shape.cellk;
  GroupWork w;
  w.add(p, d);
  int chunk = 0, npt = 0;
  group_tiling(pooled, w, 0, &chunk, &npt);
  const long long cap = tile_bound(p, d, chunk, npt);
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
  ck(cudaMemcpyAsync(base + o_rE, split.rE.data(), sizeof(int) * n_e, cudaMemcpyHostToDevice, st), "cell index upload");
  ck(cudaMemcpyAsync(base + o_fE, split.fE.data(), sizeof(float) * n_e, cudaMemcpyHostToDevice, st),
     "cell fraction upload");
  ck(cudaMemcpyAsync(base + o_perm, split.perm.data(), sizeof(int) * n_e, cudaMemcpyHostToDevice, st),
     "cell order upload");
  ck(cudaMemcpyAsync(base + o_fEs, split.fEs.data(), sizeof(float) * n_e, cudaMemcpyHostToDevice, st),
     "ordered fraction upload");
  ck(cudaMemcpyAsync(base + o_cf, split.cell_first.data(), sizeof(int) * n_cf, cudaMemcpyHostToDevice, st),
     "cell start upload");
  // state that must start at zero: the caller's flux, the counters and the queue control words
  ck(cudaMemsetAsync(flux_d, 0, sizeof(double) * (size_t)p.n_bins * n_e, st), "flux clear");
  ck(cudaMemsetAsync(base + o_stats, 0, sizeof(unsigned long long) * kStats, st), "counter clear");
  ck(cudaMemsetAsync(base + o_ctrl, 0, sizeof(int) * 16, st), "queue clear");
  ck(cudaMemsetAsync(base + o_status, 0, sizeof(int) * 4, st), "status clear");
  ck(cudaMemsetAsync(base + o_rseen, 0, sizeof(unsigned) * kMaxSpots * (size_t)ring_words, st), "ring bits clear");

  int* ctrl = (int*)(base + o_ctrl);
  KernelArgs a{};
  a.profiles = (const DevProfile*)(base + o_prof);
  a.lens = lens;
  a.nsx = nsx;
  a.flux = flux_d;
  a.comp = nullptr;  // no room for a compensation pool: plain atomic additions
  WorkQueue& q = a.queue;
  q.tiles = (Tile*)(base + o_tiles);
  q.capacity = (int)cap;
  q.n_tiles = ctrl;
  q.next = ctrl + 1;
  q.overflow = ctrl + 2;
  a.shape = shape;
  ck(configure_integrand_smem(a.shape), "shared-memory attribute");
  const int occ = max_active_ctas(a.shape);
  if (occ < 1) throw Error(PPM_E_RANGE, "ppm_profile_noalloc: launch shape does not fit on an SM");
  ck(launch_plan(a.profiles, 1, lens, q, chunk, npt, st), "plan launch");
  ck(launch_integrand(a, (int)std::min<long long>((long long)sm_count * occ, std::max(1ll, cap)), st),
     "integrand launch");
  if (counts_d) {
    const Resp& r = resps[p.response];
    FoldJob job{0, 0, p.exposure_s * (1. / p.n_bins)};
    ck(cudaMemcpyAsync(base + o_job, &job, sizeof(FoldJob), cudaMemcpyHostToDevice, st), "fold job upload");
    const FoldJob* dj = (const FoldJob*)(base + o_job);
    if (p.fold == PPM_FOLD_BF16X3 && r.tc_ok)
      ck(fold_tc_launch(r, dj, 1, p.n_bins, flux_d, counts_d, st, (int*)(base + o_status)), "fold launch");
    else
      ck(launch_fold_simt(dj, 1, r.d_rsp, r.n_ch, r.n_e, p.n_bins, flux_d, counts_d, p.fold != PPM_FOLD_FP32, st),
         "fold launch");
  }
}

// Waits for `st` and reports the last ppm_profile_noalloc call's status words
// and counters (host stack copies only: nothing is allocated).
int Engine::profile_noalloc_result(cudaStream_t st, ppm_result_info* info) {
  std::lock_guard<std::mutex> lk(mu);
  auto ck = [](cudaError_t e, const char* what) {
    if (e != cudaSuccess)
      throw Error(PPM_E_CUDA, std::string("ppm_profile_noalloc_result: ") + what + ": " + cudaGetErrorString(e));
  };
  ck(cudaSetDevice(cfg.device), "cudaSetDevice");
  if (!st) st = stream;
  const unsigned char* base = (const unsigned char*)scratch_address(cfg.device);
  const ScratchHead hd = scratch_head();
  unsigned long long stats[kStats];
  int ctrl[16], status[4];
  ck(cudaMemcpyAsync(stats, base + hd.stats, sizeof(stats), cudaMemcpyDeviceToHost, st), "counter read");
  ck(cudaMemcpyAsync(ctrl, base + hd.ctrl, sizeof(ctrl), cudaMemcpyDeviceToHost, st), "queue read");
  ck(cudaMemcpyAsync(status, base + hd.status, sizeof(status), cudaMemcpyDeviceToHost, st), "status read");
  ck(cudaStreamSynchronize(st), "stream wait");
  int code = PPM_OK;
  if (ctrl[2]) code = PPM_E_RANGE;      // work-queue overflow
  else if (status[0]) code = PPM_E_TIMEOUT;  // a bounded wait of the tensor-core fold ran out
  if (info) {
    info->n_active = (int64_t)(stats[0] + stats[5]);
    info->n_rings = (int64_t)stats[1];
    info->n_dropped_rings = (int64_t)stats[2];
    info->n_points = (int64_t)stats[3];
    info->n_clamped = (int64_t)stats[4];
    info->n_active_integrated = (int64_t)stats[0];
    info->status = code;
    info->reserved = 0;
  }
  return code;
}

}  // namespace ppm
