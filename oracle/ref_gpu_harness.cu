/*
 * ref_gpu_harness.cu — runs the reference's own CUDA program
 * (gpu/devarshi24st_gpu.cu from fizban007/gpu_ppm, compiled unchanged for
 * sm_100a with the reference's GPU flags plus -DNDEBUG) on scenarios read
 * from a file, so that the engine can be timed beside it on the same GPU.
 * Built by oracle/Makefile into oracle/_ref/.  TEST INFRASTRUCTURE ONLY.
 *
 * The program's star is compile-time (M, R_eq, spin, inclination, 32 phase
 * bins, logT, D: gpu/devarshi24st_gpu.cu:22-44); a scenario sets the spots,
 * N_side, N_fine and the GL points per bin.  Each scenario runs calc_one_star
 * (:433-511), which times its kernel and cuBLAS fold with CUDA events and
 * writes output/<name>_<setting>_{time,counts}_gpu.txt.
 *
 * Usage: ref_devarshi_gpu <scenario-file>, run with the current directory laid
 * out as the reference expects (tables/lensing/std, tables/ism_inst/std,
 * ext/model_data/nsx_H_v200804.out, output/).  Scenario lines:
 *   name N_side N_fine N_pts std theta1 phi1 angrad1 theta2 phi2 angrad2
 *
 * Inputs stay inside the program's tables by construction: the star's u
 * (Rs/R = 0.34-0.35) and logg (14.2-14.3) lie well inside the lensing and NSX
 * axes, the energy stencil and every VecHunt index are clamped by the program
 * itself, and cos(alpha) below the lensing table's axis reads earlier rows of
 * the same allocation (the row index of u is ~56), never outside it.
 */
#define main ppm_reference_gpu_main
#include "devarshi24st_gpu.cu"
#undef main

int main(int argc, char** argv) {
  if (argc < 2) {
    std::fprintf(stderr, "usage: %s <scenario-file>\n", argv[0]);
    return 2;
  }
  std::ifstream in(argv[1]);
  if (!in) {
    std::fprintf(stderr, "cannot open %s\n", argv[1]);
    return 2;
  }
  NSX nsx;
  Lens lens("std");
  IsmInst ism_inst("std");
  std::string name, setting;
  int N_side, N_fine, N_pts;
  double t1, p1, a1, t2, p2, a2;
  int rc = 0;
  while (in >> name >> N_side >> N_fine >> N_pts >> setting >> t1 >> p1 >> a1 >> t2 >> p2 >> a2) {
    // gl.cuh tabulates 1-6 points per bin; the kernel's dynamic shared memory is 90 KB
    if (setting != "std" || N_side < 1 || N_fine < 2 || N_pts < 1 || N_pts > 6 ||
        4 * N_side + 5 * (N_fine + 1) + c.N_logEkT * c.N_mu > 90 * 1024 / 4) {
      std::fprintf(stderr, "scenario %s: unsupported (setting std only, 1-6 points per bin, and 4 N_side + "
                           "5 (N_fine + 1) floats must fit beside the NSX slice in 90 KB)\n", name.c_str());
      rc = 2;
      break;
    }
    StarData s{t1, p1, a1, t2, p2, a2, name};
    calc_one_star(s, lens, nsx, ism_inst, N_side, N_fine, N_pts, setting);
  }
  nsx.free_gpu_memory();
  lens.free_gpu_memory();
  ism_inst.free_gpu_memory();
  return rc;
}
