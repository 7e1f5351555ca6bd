// Host-side helpers shared by the engine translation units: error reporting
// and the physical constants of the reference (gpu/unit.cuh:1-20,
// cpu/unit.hpp:1-25), kept with the same values and spelling of the
// expressions so that derived constants round identically.
#pragma once

#include <string>

namespace ppm {

// Records `msg` as this thread's last error and returns `code`.
int set_error(int code, const std::string& msg);
void clear_error();

namespace units {
constexpr double schwarzschild_radius_of_sun_in_km = 2.9532501;
constexpr double sqrt_km3_over_s2_GMsun = 2.745011592867327e-6;
constexpr double pi = 3.14159265358979323846;
constexpr double two_pi = 2. * pi;
constexpr double h_in_keV_s = 4.135668e-18;
constexpr double c_in_m_s = 299792458.;
constexpr double c_in_km_s = c_in_m_s / 1e3;
constexpr double c_in_cm_s = c_in_m_s * 1e2;
constexpr double Ibb_constant = 2. / (h_in_keV_s * h_in_keV_s * h_in_keV_s * c_in_cm_s * c_in_cm_s);
constexpr double kpc_in_km = 3.08567758e+16;
constexpr double planck = 6.62607015E-27;
constexpr double boltzmann_keV_per_K = 8.617333262E-8;
}  // namespace units

}  // namespace ppm
