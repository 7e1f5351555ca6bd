// Fit statistics of model counts against observed counts (ppm_batch_fit,
// ppm_profile_fit): the reduced-chi2 helper cal_chi2 of p_devarshi24st.py:43-49
// and the Poisson log-likelihood, evaluated on the device right after the fold
// so that a sampler's likelihood loop reads back a few scalars per proposal
// instead of the [n_ch][n_bins] count arrays.
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "../../include/ppm.h"
#include "engine.h"

namespace ppm {

namespace {

#define FIT_CUDA(call)                                                                           \
  do {                                                                                           \
    cudaError_t e_ = (call);                                                                     \
    if (e_ != cudaSuccess) throw Error(PPM_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

constexpr int kFitThreads = 256;

// One CTA per profile.  Per-thread partial sums over a fixed stride, then a
// fixed-order warp and block reduction: the result does not depend on timing.
__global__ void __launch_bounds__(kFitThreads) fit_kernel(const long long* counts_off, const double* counts,
                                                          const double* obs, int n_el, double lgamma_sum,
                                                          ppm_fit* out) {
  __shared__ double s_red[3][kFitThreads / 32];
  __shared__ long long s_nz[kFitThreads / 32];
  __shared__ int s_bad[kFitThreads / 32];
  const double* m = counts + counts_off[blockIdx.x];
  double M = 0.0, S = 0.0, L = 0.0;
  long long nz = 0;
  int bad = 0;
  for (int i = threadIdx.x; i < n_el; i += kFitThreads) {
    const double mi = m[i], di = obs[i];
    M += mi;
    if (mi > 0.0) {
      const double r = di - mi;
      S += r * r / mi;
      L += di * log(mi) - mi;
    } else {
      ++nz;
      if (di != 0.0) bad = 1;
      L -= mi;
    }
  }
  for (int o = 16; o > 0; o >>= 1) {
    M += __shfl_down_sync(0xffffffffu, M, o);
    S += __shfl_down_sync(0xffffffffu, S, o);
    L += __shfl_down_sync(0xffffffffu, L, o);
    nz += __shfl_down_sync(0xffffffffu, nz, o);
    bad |= __shfl_down_sync(0xffffffffu, bad, o);
  }
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    s_red[0][warp] = M;
    s_red[1][warp] = S;
    s_red[2][warp] = L;
    s_nz[warp] = nz;
    s_bad[warp] = bad;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    M = S = L = 0.0;
    nz = 0;
    bad = 0;
    for (int w = 0; w < kFitThreads / 32; ++w) {
      M += s_red[0][w];
      S += s_red[1][w];
      L += s_red[2][w];
      nz += s_nz[w];
      bad |= s_bad[w];
    }
    ppm_fit f;
    f.chi2 = M > 0.0 ? S * (1e6 / M) : (double)NAN;
    f.loglike = bad ? -(double)INFINITY : L - lgamma_sum;
    f.model_total = M;
    f.n_zero_model = nz;
    out[blockIdx.x] = f;
  }
}

}  // namespace

int Engine::add_observed(int resp, int n_bins, const double* counts) {
  std::lock_guard<std::mutex> lk(mu);
  FIT_CUDA(cudaSetDevice(cfg.device));
  if (resp < 0 || resp >= (int)resps.size()) throw Error(PPM_E_INVALID, "no such response");
  if (n_bins <= 0) throw Error(PPM_E_INVALID, "n_bins must be positive");
  if (!counts) throw Error(PPM_E_INVALID, "null observed counts");
  Observed o;
  o.resp = resp;
  o.n_bins = n_bins;
  o.n_ch = resps[resp].n_ch;
  const size_t n = (size_t)o.n_ch * n_bins;
  for (size_t i = 0; i < n; ++i) {
    if (!(counts[i] >= 0.0) || !std::isfinite(counts[i]))
      throw Error(PPM_E_INVALID, "observed counts must be finite and non-negative");
    o.lgamma_sum += std::lgamma(counts[i] + 1.0);
  }
  FIT_CUDA(cudaMalloc(&o.d_counts, sizeof(double) * n));
  track(o.d_counts);
  FIT_CUDA(cudaMemcpy(o.d_counts, counts, sizeof(double) * n, cudaMemcpyHostToDevice));
  observed.push_back(o);
  return (int)observed.size() - 1;
}

void Engine::batch_fit(BatchImpl& B, int obs, ppm_fit* out, cudaStream_t st) {
  FIT_CUDA(cudaSetDevice(cfg.device));
  if (obs < 0 || obs >= (int)observed.size()) throw Error(PPM_E_INVALID, "no such observed data");
  if (!out) throw Error(PPM_E_INVALID, "null output");
  const Observed& o = observed[obs];
  for (int i = 0; i < B.n; ++i)
    if (B.params[i].response != o.resp || B.params[i].n_bins != o.n_bins)
      throw Error(PPM_E_INVALID, "profile " + std::to_string(i) +
                                     " does not use the observed data's response and bin count");
  if (!st) st = B.last_stream ? B.last_stream : stream;
  if (!B.d_fit) {
    B.d_fit_off = (long long*)B.mem.alloc(sizeof(long long) * (size_t)B.n);
    B.d_fit = (ppm_fit*)B.mem.alloc(sizeof(ppm_fit) * (size_t)B.n);
    FIT_CUDA(cudaMemcpyAsync(B.d_fit_off, B.counts_off.data(), sizeof(long long) * (size_t)B.n,
                             cudaMemcpyHostToDevice, st));
  }
  if (B.n > 0) {
    fit_kernel<<<B.n, kFitThreads, 0, st>>>(B.d_fit_off, B.d_counts, o.d_counts, o.n_ch * o.n_bins, o.lgamma_sum,
                                             B.d_fit);
    FIT_CUDA(cudaGetLastError());
    FIT_CUDA(cudaMemcpyAsync(out, B.d_fit, sizeof(ppm_fit) * (size_t)B.n, cudaMemcpyDeviceToHost, st));
  }
  FIT_CUDA(cudaStreamSynchronize(st));
}

void Engine::profile_fit(const ppm_params& p, int obs, ppm_fit* out, ppm_result_info* info) {
  std::lock_guard<std::mutex> lk(mu);
  BatchImpl B;
  batch_build(B, 1, &p);
  batch_enqueue(B, stream, nullptr);
  B.last_stream = stream;
  batch_fit(B, obs, out, stream);
  batch_collect(B, nullptr, nullptr, info, stream);
}

}  // namespace ppm
