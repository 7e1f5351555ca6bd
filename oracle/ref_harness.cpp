/*
 * ref_harness.cpp — drives the reference's own CPU programs
 * (cpu/devarshi24st_cpu.cpp, cpu/os1_cpu.cpp, cpu/t_interp.cpp from
 * fizban007/gpu_ppm, compiled unchanged with `-Dmain=ppm_reference_main`) on
 * scenarios read from a file, so that their outputs can pin the oracle.
 * Built by oracle/Makefile into oracle/_ref/.  TEST INFRASTRUCTURE ONLY.
 *
 * Usage: ref_<program> <scenario-file>, run with the current directory laid
 * out as the reference expects (tables/, ext/model_data/, output/).
 * Scenario lines (whitespace separated):
 *   devarshi: name N_side N_fine N_pts setting theta1 phi1 angrad1 theta2 phi2 angrad2
 *   os1:      name nu spot_center_theta obs_theta angular_radius beaming
 *   tinterp:  name N_fine N_pts obs_theta theta angrad interp_type
 */
#include "grid.hpp"
#include "lensing.hpp"
#include "unit.hpp"
#if defined(REF_DEVARSHI) || defined(REF_TINTERP)
#include "ism_inst.hpp"
#include "nsx.hpp"
#endif

static long long g_oob_messages = 0;

extern "C" int ppm_ref_printf(const char* fmt, ...) {
  if (std::strstr(fmt, "out of bounds") != nullptr) {
    ++g_oob_messages;
    return 0;
  }
  va_list ap;
  va_start(ap, fmt);
  int r = std::vfprintf(stderr, fmt, ap);
  va_end(ap);
  return r;
}

#if defined(REF_DEVARSHI)
// Same layout as StarData at cpu/devarshi24st_cpu.cpp:12-15.
struct StarData {
  double theta1, phi1, angrad1, theta2, phi2, angrad2;
  std::string name;
};
void calc_one_star(StarData s, Lensing& lt, NSX& nsx, IsmInst& ism_inst, int N_side, int N_fine_phase,
                   int N_points_per_phase_bin, std::string const& setting);
#elif defined(REF_OS1)
// Same layout as StarData at cpu/os1_cpu.cpp:11-15.
struct StarData {
  double frequency_nu, spot_center_theta, obs_theta, angular_radius;
  std::string name;
  char beaming;
};
void calc_one_star(StarData s, Lensing& lt);
#elif defined(REF_TINTERP)
// Same layout as StarData at cpu/t_interp.cpp:11-17.
struct StarData {
  double obs_theta;
  double theta, angrad;
  int interp_type;
  std::string name;
};
void calc_one_star(StarData s, Lensing& lens, NSX& nsx, int N_fine_phase, int N_points_per_phase_bin);
#endif

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
  Lensing lt("std");
#if defined(REF_DEVARSHI)
  NSX nsx;
  IsmInst ism("std");
  std::string name, setting;
  int N_side, N_fine, N_pts;
  double t1, p1, a1, t2, p2, a2;
  while (in >> name >> N_side >> N_fine >> N_pts >> setting >> t1 >> p1 >> a1 >> t2 >> p2 >> a2) {
    StarData s{t1, p1, a1, t2, p2, a2, name};
    calc_one_star(s, lt, nsx, ism, N_side, N_fine, N_pts, setting);
  }
#elif defined(REF_OS1)
  std::string name;
  double nu, th, ot, ar;
  char beaming;
  while (in >> name >> nu >> th >> ot >> ar >> beaming) {
    StarData s{nu, th, ot, ar, name, beaming};
    calc_one_star(s, lt);
  }
#elif defined(REF_TINTERP)
  NSX nsx;
  std::string name;
  int N_fine, N_pts, interp;
  double ot, th, ar;
  while (in >> name >> N_fine >> N_pts >> ot >> th >> ar >> interp) {
    StarData s{ot, th, ar, interp, name};
    calc_one_star(s, lt, nsx, N_fine, N_pts);
  }
#endif
  std::fprintf(stderr, "ppm_ref: out-of-range lookups reported by the reference: %lld\n", g_oob_messages);
  return 0;
}
