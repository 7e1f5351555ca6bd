/*
 * ref_os1_gpu_harness.cu — runs the reference's own CUDA blackbody program
 * (gpu/os1_gpu.cu from fizban007/gpu_ppm, compiled unchanged for sm_100a with
 * the reference's GPU flags plus -DNDEBUG) on its ten OS1 stars, after one
 * warm-up star, `repeats` times each, so that the engine can be timed beside
 * it.  Built by oracle/Makefile into oracle/_ref/.  TEST INFRASTRUCTURE ONLY.
 *
 * The program's scenarios and grid are compile-time (N_side 256, 128 output
 * phases, 3x fine phases, E = 1 keV, kT = 0.35 keV: gpu/os1_gpu.cu:16-30, the
 * stars at :54-63).  Each calc_one_star (:304-349) times its kernel with CUDA
 * events, prints "Time taken: <ms> ms" and writes output/os1<x>_gpu.txt.
 *
 * Usage: ref_os1_gpu [repeats], run with tables/lensing/std and output/ in the
 * current directory.  Inputs stay inside the program's tables: the star's u
 * (0.34-0.36) lies inside the lensing u axis, VecHunt indices are clamped by the
 * program, and cos(alpha) below the table's axis reads earlier rows of the same
 * allocation (u's row index is ~56), never outside it.
 */
#define main ppm_reference_gpu_main
#include "os1_gpu.cu"
#undef main

int main(int argc, char** argv) {
  const int repeats = argc > 1 ? std::atoi(argv[1]) : 3;
  if (repeats < 1 || repeats > 100) {
    std::fprintf(stderr, "repeats must be 1..100\n");
    return 2;
  }
  float* grid = nullptr;
  cudaMalloc(&grid, N_output_phase * sizeof(float));
  cudaMemcpy(grid, output_phase_grid.data(), N_output_phase * sizeof(float), cudaMemcpyHostToDevice);
  Lens lens("std");
  const StarData* stars[] = {&os1a, &os1b, &os1c, &os1d, &os1e, &os1f, &os1g, &os1h, &os1i, &os1j};
  calc_one_star(os1a, lens, grid);  // warm-up: module load and first launch
  for (const StarData* s : stars)
    for (int r = 0; r < repeats; ++r) calc_one_star(*s, lens, grid);
  cudaFree(grid);
  lens.free_gpu_memory();
  return 0;
}
