// ORACLE - test and benchmark infrastructure only.  A second, independent
// statement of the engine's Plummer initial conditions (the reference has no
// Plummer generator), so that the CPU legs of the benchmark (the reference
// build in oracle/_ref and the oracle port) build the very same bodies as the
// GPU arm without loading the product library.  tests/test_oracle.py checks
// it against the engine's nbody_plummer value for value.
//
// Sampling (Aarseth, Henon & Wielen 1974): cumulative mass fraction
// u = r^3 / (1 + r^2)^(3/2), capped at 0.999, inverted for r; isotropic
// directions; speed v = q v_esc(r) with q drawn by von Neumann rejection
// against q^2 (1 - q^2)^(7/2) under the bound 0.1; equal masses 1/n; centre
// of mass moved to rest at the origin; scaled from Plummer units
// (G = M = a = 1) to Henon units (E = -1/4).  The random stream is
// xoshiro256** (Blackman & Vigna 2018) seeded by splitmix64, 53-bit uniforms
// in [0, 1); the draws are taken in the order radius, cos(theta), phi,
// (q, g) pairs, cos(theta_v), phi_v for each body in turn.
#include <cmath>
#include <cstdint>

namespace {

uint64_t rotl64(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }

struct Stream {
  uint64_t w[4];
};

void stream_seed(Stream& st, uint64_t seed) {
  for (int k = 0; k < 4; ++k) {
    seed += 0x9E3779B97F4A7C15ull;
    uint64_t m = seed;
    m = (m ^ (m >> 30)) * 0xBF58476D1CE4E5B9ull;
    m = (m ^ (m >> 27)) * 0x94D049BB133111EBull;
    st.w[k] = m ^ (m >> 31);
  }
}

double stream_uniform(Stream& st) {
  uint64_t* w = st.w;
  const uint64_t out = rotl64(w[1] * 5, 7) * 9;
  const uint64_t sh = w[1] << 17;
  w[2] ^= w[0];
  w[3] ^= w[1];
  w[1] ^= w[2];
  w[0] ^= w[3];
  w[2] ^= sh;
  w[3] = rotl64(w[3], 45);
  return static_cast<double>(out >> 11) * 0x1.0p-53;
}

// unit vector from (cos theta, phi) scaled by len
void along(double len, double ct, double ph, double* a, double* b, double* c) {
  const double st = std::sqrt(std::fmax(0.0, 1.0 - ct * ct));
  *a = len * st * std::cos(ph);
  *b = len * st * std::sin(ph);
  *c = len * ct;
}

}  // namespace

extern "C" void orc_plummer(int n, uint64_t seed, double* x, double* y, double* z, double* m,
                            double* vx, double* vy, double* vz) {
  const double two_pi = 2.0 * 3.14159265358979323846;
  Stream st;
  stream_seed(st, seed);
  for (int i = 0; i < n; ++i) {
    double u = stream_uniform(st);
    while (u <= 0.0 || u > 0.999) u = stream_uniform(st);
    const double r = 1.0 / std::sqrt(std::pow(u, -2.0 / 3.0) - 1.0);
    const double ct = 1.0 - 2.0 * stream_uniform(st);
    const double ph = two_pi * stream_uniform(st);
    along(r, ct, ph, &x[i], &y[i], &z[i]);
    double q = 0.0;
    for (;;) {
      q = stream_uniform(st);
      const double g = 0.1 * stream_uniform(st);
      if (!(g > q * q * std::pow(1.0 - q * q, 3.5))) break;
    }
    const double speed = q * std::sqrt(2.0) * std::pow(1.0 + r * r, -0.25);
    const double cv = 1.0 - 2.0 * stream_uniform(st);
    const double pv = two_pi * stream_uniform(st);
    along(speed, cv, pv, &vx[i], &vy[i], &vz[i]);
    m[i] = 1.0 / n;
  }
  double* f[6] = {x, y, z, vx, vy, vz};
  double mean[6];
  for (int k = 0; k < 6; ++k) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += f[k][i];
    mean[k] = s / n;
  }
  const double len = 3.0 * 3.14159265358979323846 / 16.0;
  const double vel = std::sqrt(16.0 / (3.0 * 3.14159265358979323846));
  for (int k = 0; k < 6; ++k)
    for (int i = 0; i < n; ++i) f[k][i] = (f[k][i] - mean[k]) * (k < 3 ? len : vel);
}
