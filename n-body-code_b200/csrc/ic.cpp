// Host-side initial conditions (deterministic, allocation-free w.r.t. the GPU).
//
// nbody_plummer       Plummer sphere, Henon units, Aarseth-Henon-Wielen (1974)
//                     sampling from a seeded xoshiro256** stream (new; the
//                     reference has no Plummer generator).
// nbody_reference_ic  the reference's own initial conditions
//                     (src/nbody.cpp:69-114), reproduced value for value:
//                     the same libstdc++ std::mt19937(42) and
//                     uniform_real_distribution<double>(-1, 1) draws in the same
//                     order, the same power-law mass transform, and the same
//                     virial rescale (a float 1/sqrt(Q) from the reference's
//                     potential with its m_j*m_j term, src/utils.cpp:148,
//                     summed serially in the reference's order).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>

#include "../../include/nbody_cuda.h"

namespace {

// xoshiro256** (Blackman & Vigna, 2018) seeded through splitmix64.
struct Xoshiro256 {
  uint64_t s[4];
  explicit Xoshiro256(uint64_t seed) {
    uint64_t z = seed;
    for (auto& w : s) {
      z += 0x9E3779B97F4A7C15ull;
      uint64_t t = z;
      t = (t ^ (t >> 30)) * 0xBF58476D1CE4E5B9ull;
      t = (t ^ (t >> 27)) * 0x94D049BB133111EBull;
      w = t ^ (t >> 31);
    }
  }
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t next() {
    const uint64_t r = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  // uniform in [0, 1) with 53 random bits
  double uniform() { return static_cast<double>(next() >> 11) * 0x1.0p-53; }
};

constexpr double kPi = 3.14159265358979323846;

}  // namespace

extern "C" nbody_status nbody_plummer(int n, uint64_t seed, double* x, double* y, double* z,
                                      double* m, double* vx, double* vy, double* vz) {
  if (n < 1 || !x || !y || !z || !m || !vx || !vy || !vz) return NBODY_ERR_INVALID_ARG;
  Xoshiro256 rng(seed);
  // Plummer model units (G = M = a = 1): E = -3 pi / 64.  Henon units
  // (E = -1/4) scale lengths by 3 pi / 16 and velocities by sqrt(16 / (3 pi)).
  const double rscale = 3.0 * kPi / 16.0;
  const double vscale = std::sqrt(16.0 / (3.0 * kPi));
  for (int i = 0; i < n; ++i) {
    // radius from the cumulative mass M(r) = r^3 / (1 + r^2)^(3/2), mass
    // fraction capped at 0.999 (r <= ~38.7 a) to avoid far outliers
    double u;
    do {
      u = rng.uniform();
    } while (u <= 0.0 || u > 0.999);
    const double r = 1.0 / std::sqrt(std::pow(u, -2.0 / 3.0) - 1.0);
    const double cz = 1.0 - 2.0 * rng.uniform();
    const double ph = 2.0 * kPi * rng.uniform();
    const double sz = std::sqrt(std::max(0.0, 1.0 - cz * cz));
    x[i] = r * sz * std::cos(ph);
    y[i] = r * sz * std::sin(ph);
    z[i] = r * cz;
    // speed as a fraction q of the local escape speed, von Neumann rejection
    // on g(q) = q^2 (1 - q^2)^(7/2) (max < 0.1)
    double q, g;
    do {
      q = rng.uniform();
      g = 0.1 * rng.uniform();
    } while (g > q * q * std::pow(1.0 - q * q, 3.5));
    const double v = q * std::sqrt(2.0) * std::pow(1.0 + r * r, -0.25);
    const double cw = 1.0 - 2.0 * rng.uniform();
    const double pw = 2.0 * kPi * rng.uniform();
    const double sw = std::sqrt(std::max(0.0, 1.0 - cw * cw));
    vx[i] = v * sw * std::cos(pw);
    vy[i] = v * sw * std::sin(pw);
    vz[i] = v * cw;
    m[i] = 1.0 / n;
  }
  // centre of mass at rest at the origin, then Henon scaling
  double c[6] = {0, 0, 0, 0, 0, 0};
  for (int i = 0; i < n; ++i) {
    c[0] += x[i]; c[1] += y[i]; c[2] += z[i];
    c[3] += vx[i]; c[4] += vy[i]; c[5] += vz[i];
  }
  for (double& v : c) v /= n;
  for (int i = 0; i < n; ++i) {
    x[i] = (x[i] - c[0]) * rscale;
    y[i] = (y[i] - c[1]) * rscale;
    z[i] = (z[i] - c[2]) * rscale;
    vx[i] = (vx[i] - c[3]) * vscale;
    vy[i] = (vy[i] - c[4]) * vscale;
    vz[i] = (vz[i] - c[5]) * vscale;
  }
  return NBODY_OK;
}

extern "C" nbody_status nbody_reference_ic(int n, double eps2, double* x, double* y, double* z,
                                           double* m, double* vx, double* vy, double* vz) {
  if (n < 1 || !x || !y || !z || !m || !vx || !vy || !vz) return NBODY_ERR_INVALID_ARG;
  constexpr double vmax = 1.0, rmax = 1.0, mmin = 0.01, mmax = 1.0;  // src/main.cpp:73-76
  std::mt19937 gen(42);
  std::uniform_real_distribution<double> uni(-1.0, 1.0);
  for (int k = 0; k < n;) {
    const double px = uni(gen) * rmax, py = uni(gen) * rmax, pz = uni(gen) * rmax;
    if (px * px + py * py + pz * pz < rmax * rmax) {
      x[k] = px;
      y[k] = py;
      z[k] = pz;
      ++k;
    }
  }
  const double alpha = -2.35 + 1.0;
  const double lo = std::pow(mmin, alpha), hi = std::pow(mmax, alpha);
  for (int i = 0; i < n; ++i) {
    vx[i] = uni(gen) * vmax;
    vy[i] = uni(gen) * vmax;
    vz[i] = uni(gen) * vmax;
    m[i] = std::pow((hi - lo) * uni(gen) + lo, 1.0 / alpha);
  }
  double T = 0.0;
  for (int i = 0; i < n; ++i)
    T += 0.5 * m[i] * (vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i]);
  double U = 0.0;
  for (int i = 0; i < n; ++i) {
    double row = 0.0;
    for (int j = i + 1; j < n; ++j) {
      const double ddx = (x[i] - x[j]) * (x[i] - x[j]);
      const double ddy = (y[i] - y[j]) * (y[i] - y[j]);
      const double ddz = (z[i] - z[j]) * (z[i] - z[j]);
      row -= m[j] * m[j] * (1. / std::sqrt(ddx + ddy + ddz + eps2));
    }
    U += row;
  }
  const float scale = 1.0 / std::sqrt(-2.0 * T / U);
  for (int i = 0; i < n; ++i) {
    vx[i] = vx[i] * scale;
    vy[i] = vy[i] * scale;
    vz[i] = vz[i] * scale;
  }
  return NBODY_OK;
}
