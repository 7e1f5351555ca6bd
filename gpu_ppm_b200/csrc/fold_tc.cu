// Tensor-core response fold (placeholder until the tcgen05 kernel lands).
#include "engine.h"

namespace ppm {

void Engine::fold_tc_prepare(Resp& r) { r.tc_ok = false; }

cudaError_t Engine::fold_tc_launch(const Resp& r, const FoldJob* jobs, int n_jobs, int n_bins, const double* flux,
                                   double* counts, cudaStream_t st) {
  (void)r;
  (void)jobs;
  (void)n_jobs;
  (void)n_bins;
  (void)flux;
  (void)counts;
  (void)st;
  return cudaErrorNotSupported;
}

}  // namespace ppm
