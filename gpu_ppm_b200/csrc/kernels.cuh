// Launch-side declarations of the engine kernels (defined in kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "device.cuh"

namespace ppm {

// Shared-memory carve-up of the integrand kernels; host and device compute it
// from the same inputs so the launch size always matches what the kernel uses.
struct IntegrandShape {
  int nt;         // threads per CTA
  int ne_t;       // energies per thread (1, 2 or 4)
  int pb;         // phase points per batch
  int max_cand;   // candidate elements per tile
  int n_fine;     // largest n_fine among the profiles
  int n_cp, n_ca; // lensing row lengths
  int nE, nmu;    // NSX slice
  int cells;      // Q cells per point (span + 1)
  bool nsx;
  int bb_fp64;    // blackbody variant: 1 = FP64 integrand, 0 = FP32
  int minb;       // CTAs per SM the register budget is compiled for (1 or 2)
  // home-cell NSX kernel: one lane per energy cell, record groups of cell_warps warps
  int cellk;      // 1 = home-cell kernel, 0 = pooled-polynomial kernel
  int maxe_t;     // energy slots per home cell the home-cell kernel is compiled for (2, 4, 8, 16)
  int cell_warps; // warps covering the cells of one point (32 x cpl cells per warp)
  int cpl;        // home cells per lane (1..3)
  int ldS;        // floats between the slice rows in shared memory (odd: conflict-free column reads)
  // offsets in bytes
  int off_j, off_P, off_F, off_Z, off_MU, off_mu, off_S, off_union, off_rows, off_batch, off_Q, total;
  int off_hidx;   // home-cell kernel: the tile's phase_o bracket table ([n_fine + 1] uint16), 0 elsewhere
};

IntegrandShape make_shape(bool nsx, int nt, int ne_t, int pb, int max_cand, int n_fine, int n_cp, int n_ca, int nE,
                          int nmu, int cells, bool cellk = false);

struct KernelArgs {
  const DevProfile* profiles;
  DevLens lens;
  DevNsx nsx;
  WorkQueue queue;
  double* flux;  // pool
  double* comp;  // compensation pool of the flux pool's atomic additions (nullptr: plain additions)
  IntegrandShape shape;
  // > 0: fused point-source mode of the blackbody kernel (no queue, no planner): CTA b takes profile b of
  // n_fused, clears its flux and counters, drops or integrates each point spot's single tile
  int n_fused;
};

// chunk: candidate elements per tile; nodes_per_tile: phase nodes per tile (<= 0: all of a profile's)
cudaError_t launch_plan(const DevProfile* profiles, int n_profiles, const DevLens& lens, const WorkQueue& q, int chunk,
                        int nodes_per_tile, cudaStream_t st);
// flux[i] += comp[i], i < n
cudaError_t launch_add_comp(double* flux, const double* comp, long long n, int sm_count, cudaStream_t st);
cudaError_t launch_integrand(const KernelArgs& a, int grid, cudaStream_t st);
// counts[c][b] = alpha * sum_E rsp[c][E] * flux[b][E] for each listed profile, FP64 or FP32 SIMT
struct FoldJob {
  long long flux_off, counts_off;
  double alpha;
};
cudaError_t launch_fold_simt(const FoldJob* jobs, int n_jobs, const double* rsp, int n_ch, int n_e, int n_bins,
                             const double* flux, double* counts, bool fp64, cudaStream_t st);
int max_active_ctas(const IntegrandShape& s);
// Raises the dynamic shared-memory limit of every integrand variant on the
// current device; done once per device, safe to call from several threads.
cudaError_t configure_integrand_smem(const IntegrandShape& s);
// Runs `set_up` once per device ordinal (the current device), under a lock;
// a failed set-up is retried by the next call.
cudaError_t once_per_device(int slot, cudaError_t (*set_up)());

}  // namespace ppm
