// ORACLE — test infrastructure only.  A serial CPU restatement of the
// reference's FP64 Hermite-4 N-body path with the softening eps^2 as a
// runtime argument (the reference hard-codes EPS2 = 1e-7: include/kernel.h:13,
// include/utils.h:14).  Only tests/, __graft_entry__.smoke() and bench.py's
// CPU-baseline leg load it, and only as the checker.  The product never does.
//
// Pinning: at eps^2 = 1e-7 every function here is compared bit-for-bit with
// the unmodified reference compiled from its own sources (oracle/_ref, built
// by oracle/Makefile) and with the committed fixtures in tests/golden/ that
// tests/golden/make_golden.py generated from that build.  To make bit-identity
// possible the floating-point operation order of each reference loop is kept
// exactly (left-to-right sums, the same products), and both sides are
// compiled with the same flags (-O3, no -march, no fast-math, so no FMA
// contraction on x86-64).
//
// Reference functions restated (file:line in the reference tree):
//   orc_invsqrt2d         src/utils.cpp:155-165   InvSqrt2D
//   orc_force_fp64        src/kernel.cpp:1164-1224 force_calculation (FP64)
//   orc_force_f32         src/kernel.cpp:1101-1163 force_calculation (_F32)
//   orc_predict           src/nbody.cpp:152-163   NBody::prediction
//   orc_snapcrackle       src/nbody.cpp:165-179   NBody::snapandcrackle
//   orc_correct           src/nbody.cpp:181-196   NBody::correction
//   orc_updatedt          src/nbody.cpp:198-222   NBody::updatedt
//   orc_initialdt         src/nbody.cpp:131-150   NBody::initialdt
//   orc_kinetic           src/utils.cpp:125-135   compute_kinetic
//   orc_potential         src/utils.cpp:137-153   compute_potential (compat=1
//                         keeps the reference's m_j*m_j term; compat=0 uses
//                         m_i*m_j)
//   orc_initialize        src/nbody.cpp:69-114    NBody::initialize
//   orc_hermite_fixed     src/nbody.cpp:224-289   timestepping without updatedt
// New (no reference counterpart), used as checkers for the GPU engine:
//   orc_force_rows_fp64   direct j-sum for selected i-rows (large-N sampling)
//   orc_force_rows_f32    the same with the _F32 pair arithmetic
//   orc_potential_rows    per-row potential phi_i = -sum_{j!=i} m_j/r_ij
//   orc_force_jvp         tangent (forward-mode derivative) of the pair
//                         acc/jerk along a direction (dx, dv, dm)
//   orc_hermite_tlm       tangent-linear model of the fixed-dt Hermite run:
//                         the trajectory of orc_hermite_fixed and its
//                         directional derivative, the reference for the
//                         adjoint (reverse-mode) gradients
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <random>
#include <vector>

namespace {

// Reference constants: ETA0/ETA (include/nbody.h:15-16), the Taylor
// coefficients (include/nbody.h:17-19).
constexpr double kEta0 = 1.0e-4;
constexpr double kEta = 1.0e-2;
constexpr double kSixth = 1.0 / 6.0;
constexpr double k24th = 1.0 / 24.0;
constexpr double k120th = 1.0 / 120.0;

}  // namespace

extern "C" {

// 1/sqrt(x): integer seed 0x5FE6ED2102DCBFDA - (bits >> 1), then four
// Newton-type refinements with the reference's coefficients.  The constants
// are the reference's algorithm (src/utils.cpp:155-165) and must stay
// identical for bit parity.
double orc_invsqrt2d(double x) {
  const double half = 0.5 * x;
  int64_t bits;
  memcpy(&bits, &x, sizeof bits);
  bits = 0x5FE6ED2102DCBFDALL - (bits >> 1);
  double y;
  memcpy(&y, &bits, sizeof y);
  y *= 1.50087895511633457 - half * y * y;
  y *= 1.50000057967625766 - half * y * y;
  y *= 1.5000000000002520 - half * y * y;
  y *= 1.5000000000000000 - half * y * y;
  return y;
}

// Symmetric FP64 pair loop over j < i (Newton's third law), serial.
// r_ij = x_j - x_i; q = (r^2+eps^2)^(-3/2); qdotq = -3 (r.v) / (r^2+eps^2).
void orc_force_fp64(int n, double eps2, const double* x, const double* y, const double* z,
                    const double* m, const double* vx, const double* vy, const double* vz,
                    double* ax, double* ay, double* az, double* jx, double* jy, double* jz) {
  for (int i = 0; i < n; ++i) {
    ax[i] = ay[i] = az[i] = 0.0;
    jx[i] = jy[i] = jz[i] = 0.0;
  }
  for (int i = 0; i < n; ++i) {
    const double xi = x[i], yi = y[i], zi = z[i];
    const double vxi = vx[i], vyi = vy[i], vzi = vz[i];
    const double mi = m[i];
    for (int j = 0; j < i; ++j) {
      const double rx = x[j] - xi, ry = y[j] - yi, rz = z[j] - zi;
      const double ux = vx[j] - vxi, uy = vy[j] - vyi, uz = vz[j] - vzi;
      const double s = rx * rx + ry * ry + rz * rz + eps2;
      const double rv = rx * ux + ry * uy + rz * uz;
      const double inv = orc_invsqrt2d(s);
      const double inv2 = inv * inv;
      const double q = inv * inv2;
      const double c = -3.0 * rv * inv2;
      const double wi = mi * q;
      const double wj = m[j] * q;
      ax[i] += rx * wj;
      ay[i] += ry * wj;
      az[i] += rz * wj;
      ax[j] -= rx * wi;
      ay[j] -= ry * wi;
      az[j] -= rz * wi;
      jx[i] += wj * (ux + c * rx);
      jy[i] += wj * (uy + c * ry);
      jz[i] += wj * (uz + c * rz);
      jx[j] -= wi * (ux + c * rx);
      jy[j] -= wi * (uy + c * ry);
      jz[j] -= wi * (uz + c * rz);
    }
  }
}

// The reference's _F32 flavour: separations formed in double and rounded to
// float, float pair arithmetic, double accumulation.  Casts spell out the
// precision of every reference expression (where a double constant such as
// EPS2 or -3.0 promotes a float expression to double before it is stored
// back to float).
void orc_force_f32(int n, double eps2, const double* x, const double* y, const double* z,
                   const double* m, const double* vx, const double* vy, const double* vz,
                   double* ax, double* ay, double* az, double* jx, double* jy, double* jz) {
  for (int i = 0; i < n; ++i) {
    ax[i] = ay[i] = az[i] = 0.0;
    jx[i] = jy[i] = jz[i] = 0.0;
  }
  for (int i = 0; i < n; ++i) {
    for (int j = 0; j < i; ++j) {
      const float rx = (float)(x[j] - x[i]);
      const float ry = (float)(y[j] - y[i]);
      const float rz = (float)(z[j] - z[i]);
      const float ux = (float)(vx[j] - vx[i]);
      const float uy = (float)(vy[j] - vy[i]);
      const float uz = (float)(vz[j] - vz[i]);
      const float r2f = rx * rx + ry * ry + rz * rz;
      const float s = (float)((double)r2f + eps2);
      const float rv = rx * ux + ry * uy + rz * uz;
      const float inv = (float)orc_invsqrt2d((double)s);
      const float inv2 = inv * inv;
      const float q = inv2 * inv;
      const float c = (float)((-3.0 * (double)rv) * (double)inv2);
      const float wi = (float)(m[i] * (double)q);
      const float wj = (float)(m[j] * (double)q);
      ax[i] += (double)(rx * wj);
      ay[i] += (double)(ry * wj);
      az[i] += (double)(rz * wj);
      ax[j] -= (double)(rx * wi);
      ay[j] -= (double)(ry * wi);
      az[j] -= (double)(rz * wi);
      jx[i] += (double)(wj * (ux + c * rx));
      jy[i] += (double)(wj * (uy + c * ry));
      jz[i] += (double)(wj * (uz + c * rz));
      jx[j] -= (double)(wi * (ux + c * rx));
      jy[j] -= (double)(wi * (uy + c * ry));
      jz[j] -= (double)(wi * (uz + c * rz));
    }
  }
}

// Direct (non-symmetric) FP64 sum over all j != i for a list of i-rows, with
// the libm 1/sqrt.  A checker for large N where the O(N^2) symmetric loop is
// too slow; it differs from orc_force_fp64 only by summation order.
// out is [6][nrows]: ax, ay, az, jx, jy, jz.
void orc_force_rows_fp64(int n, double eps2, const double* x, const double* y, const double* z,
                         const double* m, const double* vx, const double* vy, const double* vz,
                         int nrows, const int* rows, double* out) {
  for (int k = 0; k < nrows; ++k) {
    const int i = rows[k];
    double a0 = 0, a1 = 0, a2 = 0, j0 = 0, j1 = 0, j2 = 0;
    for (int j = 0; j < n; ++j) {
      if (j == i) continue;
      const double rx = x[j] - x[i], ry = y[j] - y[i], rz = z[j] - z[i];
      const double ux = vx[j] - vx[i], uy = vy[j] - vy[i], uz = vz[j] - vz[i];
      const double s = rx * rx + ry * ry + rz * rz + eps2;
      const double rv = rx * ux + ry * uy + rz * uz;
      const double inv = 1.0 / std::sqrt(s);
      const double inv2 = inv * inv;
      const double w = m[j] * inv * inv2;
      const double c = -3.0 * rv * inv2;
      a0 += w * rx;
      a1 += w * ry;
      a2 += w * rz;
      j0 += w * (ux + c * rx);
      j1 += w * (uy + c * ry);
      j2 += w * (uz + c * rz);
    }
    out[0 * nrows + k] = a0;
    out[1 * nrows + k] = a1;
    out[2 * nrows + k] = a2;
    out[3 * nrows + k] = j0;
    out[4 * nrows + k] = j1;
    out[5 * nrows + k] = j2;
  }
}

// The _F32 pair arithmetic of orc_force_f32 (src/kernel.cpp:1101-1163) as a
// direct sum over all j != i for a list of i-rows: every pair's float terms
// are those the symmetric loop produces for that row (negating both
// separations leaves each rounded float product and sum negated exactly), only
// the order of the double accumulation differs.  The large-N accuracy floor
// of the mixed kernels.  out is [6][nrows].
void orc_force_rows_f32(int n, double eps2, const double* x, const double* y, const double* z,
                        const double* m, const double* vx, const double* vy, const double* vz,
                        int nrows, const int* rows, double* out) {
  for (int k = 0; k < nrows; ++k) {
    const int i = rows[k];
    double a0 = 0, a1 = 0, a2 = 0, j0 = 0, j1 = 0, j2 = 0;
    for (int j = 0; j < n; ++j) {
      if (j == i) continue;
      const float rx = (float)(x[j] - x[i]);
      const float ry = (float)(y[j] - y[i]);
      const float rz = (float)(z[j] - z[i]);
      const float ux = (float)(vx[j] - vx[i]);
      const float uy = (float)(vy[j] - vy[i]);
      const float uz = (float)(vz[j] - vz[i]);
      const float r2f = rx * rx + ry * ry + rz * rz;
      const float s = (float)((double)r2f + eps2);
      const float rv = rx * ux + ry * uy + rz * uz;
      const float inv = (float)orc_invsqrt2d((double)s);
      const float inv2 = inv * inv;
      const float q = inv2 * inv;
      const float c = (float)((-3.0 * (double)rv) * (double)inv2);
      const float wj = (float)(m[j] * (double)q);
      a0 += (double)(rx * wj);
      a1 += (double)(ry * wj);
      a2 += (double)(rz * wj);
      j0 += (double)(wj * (ux + c * rx));
      j1 += (double)(wj * (uy + c * ry));
      j2 += (double)(wj * (uz + c * rz));
    }
    out[0 * nrows + k] = a0;
    out[1 * nrows + k] = a1;
    out[2 * nrows + k] = a2;
    out[3 * nrows + k] = j0;
    out[4 * nrows + k] = j1;
    out[5 * nrows + k] = j2;
  }
}

// phi_i = -sum_{j != i} m_j / sqrt(r_ij^2 + eps^2) for selected rows.
void orc_potential_rows(int n, double eps2, const double* x, const double* y, const double* z,
                        const double* m, int nrows, const int* rows, double* phi) {
  for (int k = 0; k < nrows; ++k) {
    const int i = rows[k];
    double p = 0.0;
    for (int j = 0; j < n; ++j) {
      if (j == i) continue;
      const double rx = x[j] - x[i], ry = y[j] - y[i], rz = z[j] - z[i];
      p -= m[j] / std::sqrt(rx * rx + ry * ry + rz * rz + eps2);
    }
    phi[k] = p;
  }
}

// x += v dt + a dt^2/2 + jerk dt^3/6 ; v += a dt + jerk dt^2/2 (in place).
void orc_predict(int n, double dt, double* x, double* y, double* z, double* vx, double* vy,
                 double* vz, const double* ax, const double* ay, const double* az,
                 const double* jx, const double* jy, const double* jz) {
  for (int i = 0; i < n; ++i) {
    x[i] += vx[i] * dt + 0.5 * ax[i] * dt * dt + kSixth * jx[i] * dt * dt * dt;
    y[i] += vy[i] * dt + 0.5 * ay[i] * dt * dt + kSixth * jy[i] * dt * dt * dt;
    z[i] += vz[i] * dt + 0.5 * az[i] * dt * dt + kSixth * jz[i] * dt * dt * dt;
    vx[i] += ax[i] * dt + 0.5 * jx[i] * dt * dt;
    vy[i] += ay[i] * dt + 0.5 * jy[i] * dt * dt;
    vz[i] += az[i] * dt + 0.5 * jz[i] * dt * dt;
  }
}

// Second and third derivatives of a from the Hermite interpolant between
// (a, jerk) at t and (a1, jerk1) at t+dt.  Arrays are [3][n] blocks.
void orc_snapcrackle(int n, double dt, const double* a, const double* jk, const double* a1,
                     const double* j1, double* a2, double* a3) {
  for (int c = 0; c < 3; ++c) {
    for (int i = 0; i < n; ++i) {
      const int k = c * n + i;
      const double inv2 = 1.0 / (dt * dt);
      const double inv3 = 1.0 / (dt * dt * dt);
      a2[k] = 2.0 * inv2 * (-3.0 * (a[k] - a1[k]) - (2.0 * jk[k] + j1[k]) * dt);
      a3[k] = 6.0 * inv3 * (2.0 * (a[k] - a1[k]) + (jk[k] + j1[k]) * dt);
    }
  }
}

// x += a2 dt^4/24 + a3 dt^5/120 ; v += a2 dt^3/6 + a3 dt^4/24 on predicted
// x, v.  x and v are [3][n] blocks.
void orc_correct(int n, double dt, double* x, double* v, const double* a2, const double* a3) {
  const double dt3 = dt * dt * dt;
  const double dt4 = dt3 * dt;
  const double dt5 = dt4 * dt;
  for (int c = 0; c < 3; ++c) {
    for (int i = 0; i < n; ++i) {
      const int k = c * n + i;
      x[k] += k24th * a2[k] * dt4 + k120th * a3[k] * dt5;
      v[k] += kSixth * a2[k] * dt3 + k24th * a3[k] * dt4;
    }
  }
}

// Aarseth criterion min_i sqrt(eta (|a||a2| + |jerk|^2) / (|jerk||a3| + |a2|^2)).
// a, jk, a2, a3 are [3][n] blocks.
double orc_updatedt(int n, double eta, const double* a, const double* jk, const double* a2,
                    const double* a3) {
  double best = std::numeric_limits<double>::max();
  for (int i = 0; i < n; ++i) {
    const double A2 = a[i] * a[i] + a[n + i] * a[n + i] + a[2 * n + i] * a[2 * n + i];
    const double A = std::sqrt(A2);
    const double J2 = jk[i] * jk[i] + jk[n + i] * jk[n + i] + jk[2 * n + i] * jk[2 * n + i];
    const double J = std::sqrt(J2);
    const double S2 = a2[i] * a2[i] + a2[n + i] * a2[n + i] + a2[2 * n + i] * a2[2 * n + i];
    const double S = std::sqrt(S2);
    const double C2 = a3[i] * a3[i] + a3[n + i] * a3[n + i] + a3[2 * n + i] * a3[2 * n + i];
    const double C = std::sqrt(C2);
    const double num = A * S + J2;
    const double den = J * C + S2;
    const double d = std::sqrt(eta * num / den);
    if (d < best) best = d;
  }
  return best;
}

double orc_eta(void) { return kEta; }
double orc_eta0(void) { return kEta0; }

// min_i eta0 |a| / |jerk|.  a, jk are [3][n] blocks.
double orc_initialdt(int n, double eta0, const double* a, const double* jk) {
  double best = std::numeric_limits<double>::max();
  for (int i = 0; i < n; ++i) {
    const double A = std::sqrt(a[i] * a[i] + a[n + i] * a[n + i] + a[2 * n + i] * a[2 * n + i]);
    const double J =
        std::sqrt(jk[i] * jk[i] + jk[n + i] * jk[n + i] + jk[2 * n + i] * jk[2 * n + i]);
    const double d = eta0 * A / J;
    if (d < best) best = d;
  }
  return best;
}

double orc_kinetic(int n, const double* m, const double* vx, const double* vy, const double* vz) {
  double t = 0.0;
  for (int i = 0; i < n; ++i) {
    const double v2x = vx[i] * vx[i], v2y = vy[i] * vy[i], v2z = vz[i] * vz[i];
    t += 0.5 * m[i] * (v2x + v2y + v2z);
  }
  return t;
}

// U = sum_i sum_{j>i} -(m_j m_j | m_i m_j) / sqrt(r^2 + eps^2); the inner sum
// per i is formed first, then added to U (the reference's grouping).
double orc_potential(int n, double eps2, int compat, const double* x, const double* y,
                     const double* z, const double* m) {
  double u = 0.0;
  for (int i = 0; i < n; ++i) {
    double row = 0.0;
    for (int j = i + 1; j < n; ++j) {
      const double dxx = (x[i] - x[j]) * (x[i] - x[j]);
      const double dyy = (y[i] - y[j]) * (y[i] - y[j]);
      const double dzz = (z[i] - z[j]) * (z[i] - z[j]);
      const double inv = 1. / std::sqrt(dxx + dyy + dzz + eps2);
      row -= (compat ? m[j] * m[j] : m[j] * m[i]) * inv;
    }
    u += row;
  }
  return u;
}

// The reference initial conditions: std::mt19937(42) driving
// uniform_real_distribution<double>(-1, 1); rejection-sampled positions in a
// sphere of radius rmax; velocities uniform in a cube of half-width vmax;
// masses m = (u (mmax^a - mmin^a) + mmin^a)^(1/a) with a = -2.35 + 1;
// velocities then scaled by a float 1/sqrt(Q), Q = -2T/U from the reference's
// potential (m_j*m_j term).
void orc_initialize(int n, double vmax, double rmax, double mmin, double mmax, double eps2,
                    double* x, double* y, double* z, double* m, double* vx, double* vy,
                    double* vz) {
  std::mt19937 gen(42);
  std::uniform_real_distribution<double> u(-1.0, 1.0);
  const double alpha = -2.35 + 1.0;
  int k = 0;
  while (k < n) {
    const double px = u(gen) * rmax;
    const double py = u(gen) * rmax;
    const double pz = u(gen) * rmax;
    if (px * px + py * py + pz * pz < rmax * rmax) {
      x[k] = px;
      y[k] = py;
      z[k] = pz;
      ++k;
    }
  }
  const double lo = std::pow(mmin, alpha);
  const double hi = std::pow(mmax, alpha);
  const double inva = 1.0 / alpha;
  for (int i = 0; i < n; ++i) {
    vx[i] = u(gen) * vmax;
    vy[i] = u(gen) * vmax;
    vz[i] = u(gen) * vmax;
    const double t = (hi - lo) * u(gen) + lo;
    m[i] = std::pow(t, inva);
  }
  const double T = orc_kinetic(n, m, vx, vy, vz);
  const double U = orc_potential(n, eps2, 1, x, y, z, m);
  const double Q = -2.0 * T / U;
  const float scale = 1.0 / std::sqrt(Q);
  for (int i = 0; i < n; ++i) {
    vx[i] = vx[i] * scale;
    vy[i] = vy[i] * scale;
    vz[i] = vz[i] * scale;
  }
}

// Fixed-dt Hermite-4 run (the reference's timestepping with dt held fixed):
// force at t=0, then nsteps x {predict, force, snap/crackle, correct, swap}.
// precision 0 = FP64 force, 1 = the _F32 force.  x..vz in/out; a/jerk out as
// [6][n] (ax, ay, az, jx, jy, jz).  dt_next_out gets the last step's
// adaptive criterion (not applied), may be null.
void orc_hermite_fixed(int n, double eps2, double dt, int nsteps, int precision, double* x,
                       double* y, double* z, const double* m, double* vx, double* vy,
                       double* vz, double* derivs, double* dt_next_out) {
  auto force = precision ? orc_force_f32 : orc_force_fp64;
  std::vector<double> d0(6 * (size_t)n), d1(6 * (size_t)n), a2(3 * (size_t)n),
      a3(3 * (size_t)n), xs(3 * (size_t)n), vs(3 * (size_t)n);
  double* A = d0.data();
  double* B = d1.data();
  force(n, eps2, x, y, z, m, vx, vy, vz, A, A + n, A + 2 * n, A + 3 * n, A + 4 * n, A + 5 * n);
  memcpy(xs.data(), x, n * sizeof(double));
  memcpy(xs.data() + n, y, n * sizeof(double));
  memcpy(xs.data() + 2 * n, z, n * sizeof(double));
  memcpy(vs.data(), vx, n * sizeof(double));
  memcpy(vs.data() + n, vy, n * sizeof(double));
  memcpy(vs.data() + 2 * n, vz, n * sizeof(double));
  double* X = xs.data();
  double* V = vs.data();
  double dtn = 0.0;
  for (int s = 0; s < nsteps; ++s) {
    orc_predict(n, dt, X, X + n, X + 2 * n, V, V + n, V + 2 * n, A, A + n, A + 2 * n, A + 3 * n,
                A + 4 * n, A + 5 * n);
    force(n, eps2, X, X + n, X + 2 * n, m, V, V + n, V + 2 * n, B, B + n, B + 2 * n, B + 3 * n,
          B + 4 * n, B + 5 * n);
    orc_snapcrackle(n, dt, A, A + 3 * n, B, B + 3 * n, a2.data(), a3.data());
    orc_correct(n, dt, X, V, a2.data(), a3.data());
    dtn = orc_updatedt(n, kEta, A, A + 3 * n, a2.data(), a3.data());
    std::swap(A, B);
  }
  memcpy(x, X, n * sizeof(double));
  memcpy(y, X + n, n * sizeof(double));
  memcpy(z, X + 2 * n, n * sizeof(double));
  memcpy(vx, V, n * sizeof(double));
  memcpy(vy, V + n, n * sizeof(double));
  memcpy(vz, V + 2 * n, n * sizeof(double));
  memcpy(derivs, A, 6 * (size_t)n * sizeof(double));
  if (dt_next_out) *dt_next_out = dtn;
}

// Directional derivative of (acc, jerk) at (x, v, m) along (dx, dv, dm); direct
// j-sum with the libm 1/sqrt.  Arrays are [3][n] blocks (x, v, dx, dv, and
// the outputs da, dj); m and dm have n values.
void orc_force_jvp(int n, double eps2, const double* x, const double* v, const double* m,
                   const double* dx, const double* dv, const double* dm, double* da, double* dj) {
  for (int i = 0; i < n; ++i) {
    double A[3] = {0, 0, 0}, J[3] = {0, 0, 0};
    for (int j = 0; j < n; ++j) {
      if (j == i) continue;
      double r[3], u[3], dr[3], du[3];
      for (int c = 0; c < 3; ++c) {
        r[c] = x[c * n + j] - x[c * n + i];
        u[c] = v[c * n + j] - v[c * n + i];
        dr[c] = dx[c * n + j] - dx[c * n + i];
        du[c] = dv[c * n + j] - dv[c * n + i];
      }
      const double s = r[0] * r[0] + r[1] * r[1] + r[2] * r[2] + eps2;
      const double ds = 2.0 * (r[0] * dr[0] + r[1] * dr[1] + r[2] * dr[2]);
      const double y = 1.0 / std::sqrt(s);
      const double q = y * y * y;
      const double dq = -1.5 * q * ds / s;
      const double w = r[0] * u[0] + r[1] * u[1] + r[2] * u[2];
      const double dw = dr[0] * u[0] + dr[1] * u[1] + dr[2] * u[2] + r[0] * du[0] + r[1] * du[1] + r[2] * du[2];
      const double c3 = -3.0 * w / s;
      const double dc = -3.0 * (dw / s - w * ds / (s * s));
      for (int c = 0; c < 3; ++c) {
        A[c] += dm[j] * q * r[c] + m[j] * dq * r[c] + m[j] * q * dr[c];
        const double g = u[c] + c3 * r[c];
        J[c] += dm[j] * q * g + m[j] * dq * g + m[j] * q * (du[c] + dc * r[c] + c3 * dr[c]);
      }
    }
    for (int c = 0; c < 3; ++c) {
      da[c * n + i] = A[c];
      dj[c * n + i] = J[c];
    }
  }
}

// Fixed-dt Hermite run (the trajectory of orc_hermite_fixed, FP64) together
// with its tangent along (dx0, dv0, dm).  X, V, DX, DV are [3][n] blocks,
// in/out; m, dm have n values.  The corrector tangent uses its expanded
// linear form x1 = xp - 0.15 h^2 (a0 - a1) - h^3 (7/60 j0 + 1/30 j1),
// v1 = vp - 0.5 h (a0 - a1) - h^2 (5/12 j0 + 1/12 j1).
void orc_hermite_tlm(int n, double eps2, double h, int nsteps, double* X, double* V,
                     const double* m, double* DX, double* DV, const double* dm) {
  const size_t N3 = 3 * (size_t)n;
  std::vector<double> d0(6 * (size_t)n), d1(6 * (size_t)n), a2(N3), a3(N3);
  std::vector<double> t0(6 * (size_t)n), t1(6 * (size_t)n);  // tangents of (a, j)
  double* A = d0.data();
  double* B = d1.data();
  double* TA = t0.data();
  double* TB = t1.data();
  orc_force_fp64(n, eps2, X, X + n, X + 2 * n, m, V, V + n, V + 2 * n, A, A + n, A + 2 * n,
                 A + 3 * n, A + 4 * n, A + 5 * n);
  orc_force_jvp(n, eps2, X, V, m, DX, DV, dm, TA, TA + 3 * n);
  const double h2 = h * h, h3 = h2 * h;
  for (int s = 0; s < nsteps; ++s) {
    for (size_t k = 0; k < N3; ++k) {  // tangent predictor
      const double tx = DX[k] + h * DV[k] + 0.5 * h2 * TA[k] + (h3 / 6.0) * TA[N3 + k];
      const double tv = DV[k] + h * TA[k] + 0.5 * h2 * TA[N3 + k];
      DX[k] = tx;
      DV[k] = tv;
    }
    orc_predict(n, h, X, X + n, X + 2 * n, V, V + n, V + 2 * n, A, A + n, A + 2 * n, A + 3 * n,
                A + 4 * n, A + 5 * n);
    orc_force_fp64(n, eps2, X, X + n, X + 2 * n, m, V, V + n, V + 2 * n, B, B + n, B + 2 * n,
                   B + 3 * n, B + 4 * n, B + 5 * n);
    orc_force_jvp(n, eps2, X, V, m, DX, DV, dm, TB, TB + 3 * n);
    for (size_t k = 0; k < N3; ++k) {  // tangent corrector
      const double dA = TA[k] - TB[k];
      DX[k] += -0.15 * h2 * dA - h3 * ((7.0 / 60.0) * TA[N3 + k] + (1.0 / 30.0) * TB[N3 + k]);
      DV[k] += -0.5 * h * dA - h2 * ((5.0 / 12.0) * TA[N3 + k] + (1.0 / 12.0) * TB[N3 + k]);
    }
    orc_snapcrackle(n, h, A, A + 3 * n, B, B + 3 * n, a2.data(), a3.data());
    orc_correct(n, h, X, V, a2.data(), a3.data());
    std::swap(A, B);
    std::swap(TA, TB);
  }
}

}  // extern "C"
