// Engine state shared by the host translation units.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <condition_variable>
#include <deque>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/ppm.h"
#include "kernels.cuh"

namespace ppm {

// NVTX range in the "ppm_b200" domain for the lifetime of the object: names the
// host phases (build, plan, integrand, fold, collect, served batches) in a
// profiler timeline.  Without a profiler attached a push/pop is one call into
// an empty function.
inline nvtxDomainHandle_t nvtx_domain() {
  static nvtxDomainHandle_t d = nvtxDomainCreateA("ppm_b200");
  return d;
}
struct NvtxRange {
  explicit NvtxRange(const char* name) {
    nvtxEventAttributes_t a{};
    a.version = NVTX_VERSION;
    a.size = NVTX_EVENT_ATTRIB_STRUCT_SIZE;
    a.messageType = NVTX_MESSAGE_TYPE_ASCII;
    a.message.ascii = name;
    nvtxDomainRangePushEx(nvtx_domain(), &a);
  }
  ~NvtxRange() { nvtxDomainRangePop(nvtx_domain()); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

// Host rows of the per-N_side ring table and the per-n_fine phase table.
void compute_ring_rows(int N, std::vector<double>& h);
void compute_fine_rows(int nf, std::vector<double>& h);

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

struct DeviceBuffer {
  void* ptr = nullptr;
  size_t cap = 0;
  void reserve(size_t bytes);
  void release();
};

struct HostBuffer {
  void* ptr = nullptr;
  size_t cap = 0;
  void reserve(size_t bytes);
  void release();
};

struct Grid {
  std::vector<double> E;
  double* dE = nullptr;
  double* dinvE = nullptr;
  int* drE = nullptr;
  float* dfE = nullptr;
  int* dperm = nullptr;
  float* dfEs = nullptr;
  int* dcell_first = nullptr;
  int maxe = 0;
  int iE_min = 0, span = 1;
  double tE_lo = 0, tE_hi = 0;
  int nsx_version = -1;
};

struct Resp {
  int grid = 0, n_ch = 0, n_e = 0;
  double* d_rsp = nullptr;
  std::vector<double> h_rsp;
  // tensor-core fold operands: BF16 hi/lo split of rsp, zero padded, in the UMMA core-matrix layout,
  // one block per (channel group, 32-energy chunk)
  bool tc_ok = false;
  int tc_groups = 0, tc_ng = 0, tc_k_chunks = 0;
  void* d_b_hi = nullptr;
  void* d_b_lo = nullptr;
};

// Device allocations owned by one batch.
// Device blocks released by synchronous batches, kept for the next batch so that
// repeated ppm_profile / ppm_profile_batch calls do not pay cudaMalloc/cudaFree
// (cudaFree synchronises the device).  A block is reused for a request of at
// least half its size.  Thread-safe.
class BlockCache {
 public:
  explicit BlockCache(size_t limit = 0) : limit_(limit) {}
  ~BlockCache() { trim(); }
  void set_limit(size_t limit) { limit_ = limit; }
  // a cached block of at least `bytes` (its size in *got), or nullptr
  void* get(size_t bytes, size_t* got);
  // keeps the block (or frees it when the cache would exceed its limit)
  void put(void* p, size_t bytes);
  void trim();

 private:
  std::mutex m_;
  std::multimap<size_t, void*> free_;
  size_t held_ = 0, limit_ = 0;
};

struct DeviceArena {
  std::vector<void*> ptrs;
  std::vector<size_t> sizes;
  size_t bytes_held = 0;
  cudaStream_t stream = nullptr;  // set: stream-ordered allocations (no implicit device synchronisation)
  BlockCache* cache = nullptr;    // set (synchronous batches): blocks come from and return to the cache
  void* alloc(size_t bytes);
  DeviceArena() = default;
  DeviceArena(const DeviceArena&) = delete;
  DeviceArena& operator=(const DeviceArena&) = delete;
  ~DeviceArena();
};

// A converted, uploaded and planned set of profiles with its output pools.
struct BatchImpl {
  int n = 0;
  std::vector<ppm_params> params;
  std::vector<long long> flux_off, counts_off;
  DeviceArena mem;
  DevProfile* d_prof = nullptr;
  double* d_flux = nullptr;
  double* d_comp = nullptr;       // compensation pool of the flux pool's atomic additions
  double* d_counts = nullptr;
  unsigned* d_ring_seen = nullptr;  // ring bits behind the rings-with-active-elements counter
  long long ring_words = 0;
  size_t small_bytes = 0;           // d_stats, d_ring_seen and d_ctrl: one block
  unsigned long long* d_stats = nullptr;
  int* d_ctrl = nullptr;
  FoldJob* d_jobs = nullptr;
  struct Group {
    int g0 = 0, g1 = 0, grid = 0;
    int chunk = 1024, npt = 0;  // candidate elements and phase nodes (0 = all) per tile
    KernelArgs args{};
  };
  struct Fold {
    int resp, n_bins, mode, job0, n_jobs;
  };
  std::vector<Group> groups;
  std::vector<Fold> folds;
  size_t h2d_bytes = 0;
  // pinned host memory the build stages its uploads in, when given (serving: one area per stream slot, untouched
  // until the slot's batch has finished, so the copies run asynchronously); pageable copies otherwise
  void* h_upload = nullptr;
  size_t h_upload_cap = 0;
  cudaGraphExec_t graph = nullptr;
  cudaStream_t last_stream = nullptr;
  int chunk = 1024;                // candidate elements per tile of the home-cell NSX group
  // one blackbody group whose spots are all point sources, at most two flux additions per (bin, energy): one
  // fused launch per pass (the integrand plans, clears and integrates each profile; no memsets, no planner,
  // no compensation pool)
  bool fused_points = false;
  long long* d_fit_off = nullptr;  // counts offset per profile (fit statistics)
  ppm_fit* d_fit = nullptr;
  BatchImpl() = default;
  BatchImpl(const BatchImpl&) = delete;
  BatchImpl& operator=(const BatchImpl&) = delete;
  ~BatchImpl();
};

// Split of an energy grid against the NSX logEkT axis: t_E = log10(E) inv_dE =
// iE_min + rE + fE, plus the energies grouped by home cell rE in t_E order.
struct GridSplit {
  std::vector<int> rE, perm, cell_first;
  std::vector<float> fE, fEs;
  int iE_min = 0, span = 1, maxe = 0;
  double lo = 0, hi = 0;
};
void split_grid(const std::vector<double>& E, double inv_dE, GridSplit& out);

// Work estimate of one kernel group of a batch (the tiling's inputs).
constexpr int kMinNodesPerTile = 8;
constexpr double kMinEvalsPerTile = 65536;  // (element, node, energy) evaluations per tile, at least
struct GroupWork {
  double work = 0;        // phase points, estimated from the spots' areas
  long long pts_max = 1;  // phase points per element, largest profile
  long long rings = 0;    // rings that may hold active elements
  double elements = 0;    // active elements, estimated from the spots' areas
  int nodes_max = 1;      // phase nodes per profile, largest profile
  int ne_max = 1;         // energies per profile, largest grid
  void add(const ppm_params& p, const DevProfile& d);
};

struct Tuning {
  int pb = 20;       // phase points per polynomial sub-batch (rounded to whole warps)
  int chunk = 1024;  // candidate elements per tile
  int small_chunk = 32;  // smallest tile: batches with little work split rings down to this size
  int ne_t = 0;      // energies per thread (0 = automatic)
  int minb = 2;      // CTAs per SM targeted by the register budget
  int kernel = 0;    // NSX integrand: 0 = home-cell kernel where the grid allows, 1 = pooled-polynomial kernel
  int sets = 0;      // home-cell kernel: warp sets per CTA (0 = about 256 threads)
  int cpl = 0;       // home-cell kernel: cells per lane (0 = by estimated cost)
  int splits = 0;    // phase-node splits per element chunk (0 = by the batch's work)
  int bb_nt = 0;     // blackbody point paths (<= 64 energies): threads per CTA (0 = 512 up to 4 energies, else 256)
};

// Observed counts [n_ch][n_bins] for fit statistics.
struct Observed {
  int resp = -1, n_bins = 0, n_ch = 0;
  double* d_counts = nullptr;
  double lgamma_sum = 0;  // sum lgamma(d + 1)
};

struct GraphEntry {
  cudaGraphExec_t exec = nullptr;
};

struct Ticket;

class Engine {
 public:
  explicit Engine(const ppm_engine_config& c);
  ~Engine();

  void load_lensing(const ppm_lensing_desc& d);
  void load_nsx(const ppm_nsx_desc& d);
  int add_grid(int n_e, const double* E);
  int add_response(int grid, int n_ch, const double* rsp);

  void profile(const ppm_params& p, double* flux, double* counts, ppm_result_info* info);
  void profile_batch(int n, const ppm_params* ps, double* flux, double* counts, ppm_result_info* info);
  // ring_begin/ring_end: only HEALPix rings i in [ring_begin, ring_end) (point sources count as ring 0)
  // chunk: candidate elements per tile (0 = the tuned batch value)
  void batch_build(BatchImpl& B, int n, const ppm_params* ps, cudaStream_t copy_stream = nullptr, int ring_begin = 0,
                   int ring_end = 1 << 30, int chunk = 0);
  // candidate elements per tile for a batch of about `work` phase points, pts_max per element
  int tile_chunk(double work, long long pts_max) const;
  static double spot_elements(const ppm_params& p);
  size_t request_bytes(const ppm_params& p) const;
  void warm_tables(const ppm_params& p);
  void batch_enqueue(BatchImpl& B, cudaStream_t st, cudaEvent_t* events);
  void batch_capture(BatchImpl& B);
  void batch_launch(BatchImpl& B, cudaStream_t st);
  void batch_collect(BatchImpl& B, double* flux, double* counts, ppm_result_info* info, cudaStream_t st);
  int kernels_per_pass(const BatchImpl& B) const;
  void batch_launch_timed(BatchImpl& B, cudaStream_t st, float* ms);
  void output_sizes(const ppm_params& p, int64_t* n_flux, int64_t* n_counts) const;
  // response fold alone; host buffers (copied, waits) or device buffers (enqueued on st)
  void fold(int resp, int mode, int n_prof, int n_bins, const double* alpha, const double* flux, double* counts,
            bool device, cudaStream_t st);
  void profile_noalloc(const ppm_params& p, double* flux_d, double* counts_d, cudaStream_t st);
  int profile_noalloc_result(cudaStream_t st, ppm_result_info* info);
  int add_observed(int resp, int n_bins, const double* counts);
  void batch_fit(BatchImpl& B, int obs, ppm_fit* out, cudaStream_t st);
  void profile_fit(const ppm_params& p, int obs, ppm_fit* out, ppm_result_info* info);
  void profile_rings(const ppm_params& p, int ring_begin, int ring_end, double* flux, double* counts,
                     ppm_result_info* info);
  std::string autotune(int n, const ppm_params* sample);

  // serving
  uint64_t submit(const ppm_params& p, double* flux, double* counts);
  int poll(uint64_t t);
  int wait(uint64_t t, int timeout_ms, ppm_result_info* info);
  double latency_us(uint64_t t);
  void release_ticket(uint64_t t);
  int serve_trace(ppm_serve_batch_trace* out, int cap);
  void serve_shutdown();

  ppm_engine_config cfg;
  Tuning tune;
  int sm_count = 0;
  cudaStream_t stream = nullptr;

 private:
  friend struct Server;
  void validate(const ppm_params& p) const;
  void to_device(const ppm_params& p, DevProfile& d, long long flux_off, unsigned long long* stats);
  void fill_profile(const ppm_params& p, DevProfile& d, long long flux_off, unsigned long long* stats,
                    const double* ring, const double* fine, const DevGrid& grid, const std::vector<double>& rt);
  void prepare_grid(int id);
  DevGrid dev_grid(int id);
  const double* ring_table(int N);
  const double* fine_table(int nf);
  // rings: rings the group's spots span (sizes the blackbody phase-major walk's blocks; 0 = unknown)
  IntegrandShape choose_shape(bool nsx_kernel, bool bb_fp64, int ne_max, int nf_max, int cells_max, int maxe_max = 0,
                              int bins_max = 0, bool allow_cell = true, double rings = 0);
  bool cell_kernel_takes(int grid);
  void group_tiling(bool pooled, const GroupWork& w, int chunk_override, int* chunk, int* npt) const;
  long long tile_bound(const ppm_params& p, const DevProfile& d, int chunk, int npt) const;
  void fold_tc_prepare(Resp& r);
  // error: word the kernel sets when a bounded wait runs out (nullptr = the engine's d_err)
  cudaError_t fold_tc_launch(const Resp& r, const FoldJob* jobs, int n_jobs, int n_bins, const double* flux,
                             double* counts, cudaStream_t st, int* error = nullptr);
  void track(void* p);

  std::mutex mu;
  bool has_lens = false, has_nsx = false;
  int nsx_version = 0;
  DevLens lens{};
  DevNsx nsx{};
  std::vector<double> nsx_mu;
  std::vector<Grid> grids;
  std::vector<Resp> resps;
  std::vector<Observed> observed;
  BlockCache block_cache;
  std::map<int, double*> ring_tabs, fine_tabs;
  std::map<int, std::vector<double>> host_rings;
  std::vector<void*> owned;
  cudaEvent_t ev[4];
  int* d_err = nullptr;  // set by kernels whose bounded waits ran out

  // serving state
  struct Server* server = nullptr;
};

}  // namespace ppm
