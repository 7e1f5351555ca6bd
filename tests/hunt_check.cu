// Host check that hunt_from (the blackbody point-wise path's warm-started
// phase_o hunt) and walk_bracket (the phase-major walk's unit steps) bracket
// exactly as vhunt's bisection on non-decreasing arrays, from any starting
// index: same clamped index, same fraction.
// Random arrays with repeated values, x inside, at and outside the nodes.
// Built and run by tests/test_hunt.py; prints "<cases> <mismatches>".
#include <cstdio>
#include <random>
#include <vector>

#include "device.cuh"

int main() {
  std::mt19937_64 rng(7);
  std::uniform_real_distribution<double> u01(0.0, 1.0);
  long long cases = 0, bad = 0;
  for (int trial = 0; trial < 20000; ++trial) {
    const int n = 2 + (int)(rng() % 400);
    std::vector<double> xx(n);
    double v = u01(rng) - 0.5;
    for (int i = 0; i < n; ++i) {
      if (rng() % 5) v += 1e-4 + 1e-2 * u01(rng);  // one step in five repeats the previous value
      xx[i] = v;
    }
    const double lo = xx[0] - 0.05, hi = xx[n - 1] + 0.05;
    for (int q = 0; q < 16; ++q) {
      const double x = (rng() % 4 == 0) ? xx[rng() % n] : lo + (hi - lo) * u01(rng);
      const int hint = (int)(rng() % (unsigned)(n + 1)) - 1;  // any previous answer, -1 .. n-1
      double a_ref;
      const int i_ref = ppm::vhunt(xx.data(), n, x, a_ref);
      const int i = ppm::clampi(ppm::hunt_from(xx.data(), n, x, hint), 0, n - 2);
      const double a = (x - xx[i]) / (xx[i + 1] - xx[i]);
      const int iw = ppm::walk_bracket(xx.data(), n, x, ppm::clampi(hint, 0, n - 2));
      ++cases;
      const bool same_a = (a == a_ref) || (a != a && a_ref != a_ref);
      if (i != i_ref || !same_a || iw != i_ref) ++bad;
    }
  }
  std::printf("%lld %lld\n", cases, bad);
  return bad != 0;
}
