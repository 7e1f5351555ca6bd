// ppm_run — drop-in driver for the reference's programs, on the engine's C ABI.
//
// Runs the scenarios of gpu/devarshi24st_gpu.cu, gpu/os1_gpu.cu and
// cpu/t_interp.cpp with the reference's star constants, reading the same
// input files from the current directory and writing the same output files:
//
//   ppm_run devarshi <scenario-file>
//       lines: name N_side N_fine N_pts setting theta1 phi1 angrad1 theta2 phi2 angrad2
//       star: M=1.4, Re=12 km, nu=300 Hz, inclination 2.391, D=0.15 kpc, exposure 1e6 s,
//       32 bins, logT=6 (gpu/devarshi24st_gpu.cu:22-44)
//       inputs:  tables/lensing/std, ext/model_data/nsx_H_v200804.out, tables/ism_inst/std
//       output:  output/<name>_<setting>_counts_gpu.txt (gpu/devarshi24st_gpu.cu:491-505)
//   ppm_run os1 <scenario-file>
//       lines: name nu spot_center_theta obs_theta angular_radius beaming(i|s|c)
//       star: M=1.4, Re=12, kT=0.35 keV, E=1 keV, D=0.2 kpc, N_side 256, 128 phases
//       (gpu/os1_gpu.cu:18-36); point source when angular_radius < 0.1
//       output:  output/<name>_gpu.txt (gpu/os1_gpu.cu:330-344)
//   ppm_run tinterp <scenario-file>
//       lines: name N_fine N_pts obs_theta theta angrad interp_type (cpu/t_interp.cpp:20-32)
//       output:  output/<name>_flux_gpu.txt, 256 rows x 1024 energies
//   ppm_run ism_inst std|high|ultra
//       c_ism_inst.py: reads ext/model_data/{nicer-rmf6s-teamonly-array50_full_matrix.txt,
//       nicer-consim135p-teamonly-array50_arf.txt, interstellar_phot_frac.txt}, keeps
//       energies [0, 1800) and channels [30, 300), 128 / 256 / 512 observed energies
//       (c_ism_inst.py:5-26), writes tables/ism_inst/<setting>/{num,E_obs,rsp}.txt
//   ppm_run ism_inst <rmf> <arf> <ism|-> <i_e_min> <i_e_max> <i_ch_min> <i_ch_max> <n_e_obs> <out_dir>
//       the same with explicit files, ranges and output folder (no GPU needed)
//
// Errors are reported with the engine's status codes and messages; the
// process exits non-zero instead of the reference's exit(EXIT_FAILURE).
#include <sys/stat.h>

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <string>
#include <vector>

#include "../../include/ppm.h"

namespace {

constexpr double kPi = 3.14159265358979323846;

int fail(int rc, const char* what) {
  std::fprintf(stderr, "ppm_run: %s failed (%d): %s\n", what, rc, ppm_last_error_string());
  return 1;
}

ppm_params base_params() {
  ppm_params p{};
  p.mass_msun = 1.4;
  p.r_eq_km = 12.0;
  p.n_spots = 1;
  p.response = -1;
  p.precision = PPM_PREC_FP32;
  p.fold = PPM_FOLD_BF16X3;
  return p;
}

// nsx_H_v200804 (cpu/nsx.hpp:25-37 / gpu/nsx.cuh:54-66)
ppm_nsx_desc v200804_axes() {
  ppm_nsx_desc a{};
  a.n_logT = 35;
  a.n_logg = 14;
  a.n_logEkT = 166;
  a.n_mu = 67;
  a.logT_min = 5.10;
  a.logT_max = 6.80;
  a.logg_min = 13.7;
  a.logg_max = 15.0;
  a.logEkT_min = -1.30;
  a.logEkT_max = 2.00;
  return a;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 3) {
    std::fprintf(stderr, "usage: %s devarshi|os1|tinterp <scenario-file>\n       %s ism_inst std|high|ultra\n",
                 argv[0], argv[0]);
    return 2;
  }
  const std::string mode = argv[1];
  if (mode == "ism_inst") {  // response preparation: host only
    int rc;
    if (argc == 3) {
      const std::string setting = argv[2];
      const int n_obs = setting == "ultra" ? 512 : (setting == "high" ? 256 : (setting == "std" ? 128 : 0));
      if (!n_obs) {
        std::fprintf(stderr, "ppm_run: unknown ism_inst setting %s\n", setting.c_str());
        return 2;
      }
      const std::string out = "tables/ism_inst/" + setting;
      for (const std::string d : {std::string("tables"), std::string("tables/ism_inst"), out})
        if (::mkdir(d.c_str(), 0755) != 0 && errno != EEXIST) return fail(PPM_E_IO, ("creating " + d).c_str());
      rc = ppm_ism_inst_prepare("ext/model_data/nicer-rmf6s-teamonly-array50_full_matrix.txt",
                                "ext/model_data/nicer-consim135p-teamonly-array50_arf.txt",
                                "ext/model_data/interstellar_phot_frac.txt", 0, 1800, 30, 300, n_obs, out.c_str());
    } else if (argc == 11) {
      const std::string ism = argv[4];
      rc = ppm_ism_inst_prepare(argv[2], argv[3], ism == "-" ? nullptr : argv[4], std::atoi(argv[5]), std::atoi(argv[6]),
                                std::atoi(argv[7]), std::atoi(argv[8]), std::atoi(argv[9]), argv[10]);
    } else {
      std::fprintf(stderr, "usage: %s ism_inst std|high|ultra\n       %s ism_inst <rmf> <arf> <ism|-> <i_e_min> "
                           "<i_e_max> <i_ch_min> <i_ch_max> <n_e_obs> <out_dir>\n", argv[0], argv[0]);
      return 2;
    }
    return rc ? fail(rc, "response preparation") : 0;
  }
  std::ifstream in(argv[2]);
  if (!in) {
    std::fprintf(stderr, "ppm_run: cannot open %s\n", argv[2]);
    return 2;
  }
  ppm_engine_config cfg{};
  ppm_engine* e = nullptr;
  int rc = ppm_engine_create(&cfg, &e);
  if (rc) return fail(rc, "ppm_engine_create");
  rc = ppm_engine_load_lensing_dir(e, "tables/lensing/std");
  if (rc) return fail(rc, "loading tables/lensing/std");

  if (mode == "devarshi") {
    ppm_nsx_desc axes = v200804_axes();
    rc = ppm_engine_load_nsx_file(e, "ext/model_data/nsx_H_v200804.out", &axes);
    if (rc) return fail(rc, "loading the NSX table");
    int32_t grid = 0, rsp = 0;
    rc = ppm_engine_load_ism_inst_dir(e, "tables/ism_inst/std", &grid, &rsp);
    if (rc) return fail(rc, "loading tables/ism_inst/std");
    std::string name, setting;
    int N_side, N_fine, N_pts;
    double t1, p1, a1, t2, p2, a2;
    while (in >> name >> N_side >> N_fine >> N_pts >> setting >> t1 >> p1 >> a1 >> t2 >> p2 >> a2) {
      ppm_params p = base_params();
      p.spin_hz = 300.0;
      p.inclination_rad = 2.391;
      p.distance_kpc = 0.15;
      p.exposure_s = 1e6;
      p.spots[0] = ppm_spot{t1, p1, a1, t2, p2, a2, 6.0, 0.0, PPM_SPOT_HEALPIX, 0};
      p.atmosphere = PPM_ATM_NSX;
      p.interp = PPM_INTERP_2L2C_LE;
      p.n_side = N_side;
      p.n_bins = 32;
      p.n_gl = N_pts;
      p.n_fine = N_fine;
      p.energy_grid = grid;
      p.response = rsp;
      int64_t nf = 0, nc = 0;
      rc = ppm_output_sizes(e, &p, &nf, &nc);
      if (rc) return fail(rc, "ppm_output_sizes");
      std::vector<double> counts(nc);
      rc = ppm_profile(e, &p, nullptr, counts.data(), nullptr);
      if (rc) return fail(rc, ("profile " + name).c_str());
      const std::string out = "output/" + name + "_" + setting + "_counts_gpu.txt";
      rc = ppm_write_counts(out.c_str(), (int32_t)(nc / 32), 32, counts.data(), 16);
      if (rc) return fail(rc, ("writing " + out).c_str());
    }
  } else if (mode == "os1") {
    const double E1 = 1.0;
    int32_t grid = 0;
    rc = ppm_engine_add_energy_grid(e, 1, &E1, &grid);
    if (rc) return fail(rc, "energy grid");
    std::string name;
    double nu, th, ot, ar;
    char beam;
    while (in >> name >> nu >> th >> ot >> ar >> beam) {
      ppm_params p = base_params();
      p.spin_hz = nu;
      p.inclination_rad = ot;
      p.distance_kpc = 0.2;
      p.spots[0] = ppm_spot{th, 0.0, ar, 0.0, 0.0, 0.0, 0.0, 0.35, ar < 0.1 ? PPM_SPOT_POINT : PPM_SPOT_HEALPIX, 0};
      p.atmosphere = PPM_ATM_BLACKBODY;
      p.beaming = beam == 's' ? PPM_BEAM_SIN2 : (beam == 'c' ? PPM_BEAM_COS2 : PPM_BEAM_ISO);
      p.precision = PPM_PREC_FP64;
      p.n_side = 256;
      p.n_bins = 128;
      p.n_gl = 0;
      p.n_fine = 3 * 128;
      p.energy_grid = grid;
      std::vector<double> flux(128);
      rc = ppm_profile(e, &p, flux.data(), nullptr, nullptr);
      if (rc) return fail(rc, ("profile " + name).c_str());
      const std::string out = "output/" + name + "_gpu.txt";
      rc = ppm_write_row(out.c_str(), 128, flux.data(), 16);
      if (rc) return fail(rc, ("writing " + out).c_str());
    }
  } else if (mode == "tinterp") {
    ppm_nsx_desc axes = v200804_axes();
    rc = ppm_engine_load_nsx_file(e, "ext/model_data/nsx_H_v200804.out", &axes);
    if (rc) return fail(rc, "loading the NSX table");
    // linspace(0.1, 5, 1024) as cpu/ut.hpp:8-16 builds it
    std::vector<double> E(1024);
    const double step = (5.0 - 0.1) / (1024 - 1);
    for (int i = 0; i < 1024; ++i) E[i] = 0.1 + i * step;
    int32_t grid = 0;
    rc = ppm_engine_add_energy_grid(e, 1024, E.data(), &grid);
    if (rc) return fail(rc, "energy grid");
    std::string name;
    int N_fine, N_pts, interp;
    double ot, th, ar;
    while (in >> name >> N_fine >> N_pts >> ot >> th >> ar >> interp) {
      ppm_params p = base_params();
      p.spin_hz = 600.0;
      p.inclination_rad = ot;
      p.distance_kpc = 0.15;
      p.spots[0] = ppm_spot{th, 0.0, ar, 0.0, 0.0, 0.0, 6.0, 0.0, PPM_SPOT_POINT, 0};
      p.atmosphere = PPM_ATM_NSX;
      p.interp = interp;
      p.n_side = 1;
      p.n_bins = 256;
      p.n_gl = N_pts;
      p.n_fine = N_fine;
      p.energy_grid = grid;
      std::vector<double> flux(256 * 1024);
      rc = ppm_profile(e, &p, flux.data(), nullptr, nullptr);
      if (rc) return fail(rc, ("profile " + name).c_str());
      const std::string out = "output/" + name + "_flux_gpu.txt";
      rc = ppm_write_counts(out.c_str(), 256, 1024, flux.data(), 16);
      if (rc) return fail(rc, ("writing " + out).c_str());
    }
  } else {
    std::fprintf(stderr, "ppm_run: unknown mode %s\n", mode.c_str());
    return 2;
  }
  ppm_engine_destroy(e);
  (void)kPi;
  return 0;
}
