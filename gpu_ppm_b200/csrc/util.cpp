// Error reporting, version string and the reference's text output formats.
#include <cstdio>
#include <string>

#include "../../include/ppm.h"
#include "common.h"

namespace ppm {
static thread_local std::string g_last_error;
int set_error(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}
void clear_error() { g_last_error.clear(); }
}  // namespace ppm

extern "C" const char* ppm_last_error_string(void) { return ppm::g_last_error.c_str(); }
extern "C" const char* ppm_version(void) { return "ppm_b200 0.1 (sm_100a)"; }

// N_CH lines of n_bins space-separated values (gpu/devarshi24st_gpu.cu:491-505,
// cpu/devarshi24st_cpu.cpp:246-258): "%.<precision>g " per value, newline per row.
extern "C" int ppm_write_counts(const char* path, int32_t n_ch, int32_t n_bins, const double* counts,
                                int32_t precision) {
  if (!path || !counts || n_ch <= 0 || n_bins <= 0) return ppm::set_error(PPM_E_INVALID, "ppm_write_counts: bad argument");
  FILE* f = std::fopen(path, "w");
  if (!f) return ppm::set_error(PPM_E_IO, std::string("ppm_write_counts: cannot open ") + path);
  int prec = precision > 0 ? precision : 16;
  for (int c = 0; c < n_ch; ++c) {
    for (int b = 0; b < n_bins; ++b) std::fprintf(f, "%.*g ", prec, counts[(size_t)c * n_bins + b]);
    std::fputc('\n', f);
  }
  if (std::fclose(f) != 0) return ppm::set_error(PPM_E_IO, std::string("ppm_write_counts: write failed ") + path);
  return PPM_OK;
}

// One line of values (cpu/os1_cpu.cpp:185-193).
extern "C" int ppm_write_row(const char* path, int32_t n, const double* values, int32_t precision) {
  if (!path || !values || n <= 0) return ppm::set_error(PPM_E_INVALID, "ppm_write_row: bad argument");
  FILE* f = std::fopen(path, "w");
  if (!f) return ppm::set_error(PPM_E_IO, std::string("ppm_write_row: cannot open ") + path);
  int prec = precision > 0 ? precision : 16;
  for (int i = 0; i < n; ++i) std::fprintf(f, "%.*g ", prec, values[i]);
  std::fputc('\n', f);
  if (std::fclose(f) != 0) return ppm::set_error(PPM_E_IO, std::string("ppm_write_row: write failed ") + path);
  return PPM_OK;
}
