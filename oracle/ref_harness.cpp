// Test infrastructure: a C-ABI harness around the UNMODIFIED reference CPU
// code, compiled from the reference tree by oracle/Makefile into oracle/_ref/.
// Only tests, the golden-fixture script and bench.py's CPU-baseline legs call
// it.  Nothing in the product links it.
//
// It drives the reference's own public NBody members and methods
// (include/nbody.h:24-51) and its force_calculation (include/kernel.h:15-19):
//   ref_initialize      -> NBody::initialize          (src/nbody.cpp:69-114)
//   ref_force           -> force_calculation           (src/kernel.cpp:1164-1224,
//                                                       or 1101-1163 when built -D_F32)
//   ref_hermite_fixed   -> NBody::timestepping minus updatedt, i.e. a fixed-dt
//                          Hermite step (src/nbody.cpp:224-289)
//   ref_kinetic/potential, ref_initialdt/updatedt -> src/utils.cpp:125-153,
//                          src/nbody.cpp:131-150, 198-222
//   ref_step_sampled    -> one Hermite step whose force evaluation computes only
//                          the i-rows that rank 0 of an S-rank job owns
//                          (src/kernel.cpp:1185), for the bounded CPU baseline.
#include "nbody.h"

#include <omp.h>

#include <cstring>

namespace {

constexpr double kVmax = 1.0, kRmax = 1.0, kMmin = 0.01, kMmax = 1.0;  // src/main.cpp:73-76

void load_state(NBody& nb, int n, const double* x, const double* y, const double* z,
                const double* m, const double* vx, const double* vy, const double* vz) {
  const size_t b = (size_t)n * sizeof(double);
  memcpy(nb.h_par_x, x, b);
  memcpy(nb.h_par_y, y, b);
  memcpy(nb.h_par_z, z, b);
  memcpy(nb.h_par_w, m, b);
  memcpy(nb.h_vel_x, vx, b);
  memcpy(nb.h_vel_y, vy, b);
  memcpy(nb.h_vel_z, vz, b);
}

void swap_derivs(NBody& nb) {
  std::swap(nb.h_acc_x, nb.h_acc1_x);
  std::swap(nb.h_acc_y, nb.h_acc1_y);
  std::swap(nb.h_acc_z, nb.h_acc1_z);
  std::swap(nb.h_adot_x, nb.h_a1dot_x);
  std::swap(nb.h_adot_y, nb.h_a1dot_y);
  std::swap(nb.h_adot_z, nb.h_a1dot_z);
}

}  // namespace

extern "C" {

double ref_eps2(void) { return EPS2; }

int ref_max_threads(void) { return omp_get_max_threads(); }

void ref_set_threads(int t) {
  if (t > 0) omp_set_num_threads(t);
}

// Bodies from the reference's own initialiser: mt19937(42), unit sphere,
// cube velocities, power-law masses, virial rescale (src/nbody.cpp:69-114).
void ref_initialize(int n, double* x, double* y, double* z, double* m, double* vx, double* vy,
                    double* vz) {
  NBody nb(n, kVmax, kRmax, kMmin, kMmax);
  nb.initialize();
  const size_t b = (size_t)n * sizeof(double);
  memcpy(x, nb.h_par_x, b);
  memcpy(y, nb.h_par_y, b);
  memcpy(z, nb.h_par_z, b);
  memcpy(m, nb.h_par_w, b);
  memcpy(vx, nb.h_vel_x, b);
  memcpy(vy, nb.h_vel_y, b);
  memcpy(vz, nb.h_vel_z, b);
}

// One call of the reference's force_calculation on one rank.
void ref_force(int n, const double* x, const double* y, const double* z, const double* m,
               const double* vx, const double* vy, const double* vz, double* ax, double* ay,
               double* az, double* jx, double* jy, double* jz) {
  Sys sys;
  sys.N = n;
  sys.rank = 0;
  sys.size = 1;
  sys.start = 0;
  sys.end = n;
  force_calculation(const_cast<double*>(x), const_cast<double*>(y), const_cast<double*>(z),
                    const_cast<double*>(m), const_cast<double*>(vx), const_cast<double*>(vy),
                    const_cast<double*>(vz), ax, ay, az, jx, jy, jz, sys);
}

double ref_kinetic(int n, const double* m, const double* vx, const double* vy, const double* vz) {
  return compute_kinetic(const_cast<double*>(m), const_cast<double*>(vx), const_cast<double*>(vy),
                         const_cast<double*>(vz), n);
}

// The reference's potential, including its m_j*m_j term (src/utils.cpp:148).
double ref_potential(int n, const double* x, const double* y, const double* z, const double* m) {
  return compute_potential(const_cast<double*>(x), const_cast<double*>(y), const_cast<double*>(z),
                           const_cast<double*>(m), n);
}

// Fixed-dt Hermite run through the reference's own methods:
// force(t=0) -> nsteps x {prediction, force -> acc1/a1dot, snapandcrackle,
// correction, swap}.  In/out: x..vz (m is read).  Out: acc/jerk at the end.
// Optionally also returns the a2dot/a3dot of the last step.
void ref_hermite_fixed(int n, double dt, int nsteps, double* x, double* y, double* z,
                       const double* m, double* vx, double* vy, double* vz, double* ax,
                       double* ay, double* az, double* jx, double* jy, double* jz,
                       double* dt_next_out) {
  NBody nb(n, kVmax, kRmax, kMmin, kMmax);
  load_state(nb, n, x, y, z, m, vx, vy, vz);
  Sys& sys = nb.sys;
  force_calculation(nb.h_par_x, nb.h_par_y, nb.h_par_z, nb.h_par_w, nb.h_vel_x, nb.h_vel_y,
                    nb.h_vel_z, nb.h_acc_x, nb.h_acc_y, nb.h_acc_z, nb.h_adot_x, nb.h_adot_y,
                    nb.h_adot_z, sys);
  nb.dt = dt;
  double dtn = 0.0;
  for (int s = 0; s < nsteps; ++s) {
    nb.prediction();
    force_calculation(nb.h_par_x, nb.h_par_y, nb.h_par_z, nb.h_par_w, nb.h_vel_x, nb.h_vel_y,
                      nb.h_vel_z, nb.h_acc1_x, nb.h_acc1_y, nb.h_acc1_z, nb.h_a1dot_x,
                      nb.h_a1dot_y, nb.h_a1dot_z, sys);
    nb.snapandcrackle();
    nb.correction();
    dtn = nb.updatedt();  // adaptive criterion of this step (reported, not applied)
    swap_derivs(nb);
  }
  const size_t b = (size_t)n * sizeof(double);
  memcpy(x, nb.h_par_x, b);
  memcpy(y, nb.h_par_y, b);
  memcpy(z, nb.h_par_z, b);
  memcpy(vx, nb.h_vel_x, b);
  memcpy(vy, nb.h_vel_y, b);
  memcpy(vz, nb.h_vel_z, b);
  memcpy(ax, nb.h_acc_x, b);
  memcpy(ay, nb.h_acc_y, b);
  memcpy(az, nb.h_acc_z, b);
  memcpy(jx, nb.h_adot_x, b);
  memcpy(jy, nb.h_adot_y, b);
  memcpy(jz, nb.h_adot_z, b);
  if (dt_next_out) *dt_next_out = dtn;
}

// The reference's adaptive run, stock cycle() (src/nbody.cpp:291-380) on the
// reference initial conditions: returns E0, E_final and the dt history.
void ref_cycle(int n, int ncycle, double* e0, double* efin, double* err) {
  NBody nb(n, kVmax, kRmax, kMmin, kMmax);
  nb.cycle(ncycle);
  *e0 = nb.sys.initE;
  *efin = nb.sys.finE;
  *err = nb.sys.Err;
}

double ref_initialdt(int n, const double* ax, const double* ay, const double* az,
                     const double* jx, const double* jy, const double* jz) {
  NBody nb(n, kVmax, kRmax, kMmin, kMmax);
  const size_t b = (size_t)n * sizeof(double);
  memcpy(nb.h_acc_x, ax, b);
  memcpy(nb.h_acc_y, ay, b);
  memcpy(nb.h_acc_z, az, b);
  memcpy(nb.h_adot_x, jx, b);
  memcpy(nb.h_adot_y, jy, b);
  memcpy(nb.h_adot_z, jz, b);
  return nb.initialdt();
}

// --- bounded CPU-baseline sample -------------------------------------------
// A persistent NBody so that repeated timed steps reuse its arrays.
struct RefBench {
  NBody* nb;
  int size;
};

void* ref_bench_create(int n, double dt, int sample_ranks, const double* x, const double* y,
                       const double* z, const double* m, const double* vx, const double* vy,
                       const double* vz) {
  RefBench* rb = new RefBench;
  rb->nb = new NBody(n, kVmax, kRmax, kMmin, kMmax);
  rb->size = sample_ranks > 0 ? sample_ranks : 1;
  load_state(*rb->nb, n, x, y, z, m, vx, vy, vz);
  NBody& nb = *rb->nb;
  nb.dt = dt;
  // Derivatives at t=0 for the first predictor: computed with the same
  // sampled decomposition (only timing matters for this object).
  nb.sys.size = rb->size;
  force_calculation(nb.h_par_x, nb.h_par_y, nb.h_par_z, nb.h_par_w, nb.h_vel_x, nb.h_vel_y,
                    nb.h_vel_z, nb.h_acc_x, nb.h_acc_y, nb.h_acc_z, nb.h_adot_x, nb.h_adot_y,
                    nb.h_adot_z, nb.sys);
  return rb;
}

// One fixed-dt Hermite step.  The force evaluation runs only rank 0's share
// of an S-rank job (i = thid, thid + S*nthreads, ...; src/kernel.cpp:1185),
// i.e. ~1/S of the symmetric pairs.  Returns seconds of
// [pred, force, snap+corr] in t3.
void ref_bench_step(void* h, double* t3) {
  RefBench* rb = (RefBench*)h;
  NBody& nb = *rb->nb;
  nb.sys.size = rb->size;
  nb.sys.rank = 0;
  double t0 = omp_get_wtime();
  nb.prediction();
  double t1 = omp_get_wtime();
  force_calculation(nb.h_par_x, nb.h_par_y, nb.h_par_z, nb.h_par_w, nb.h_vel_x, nb.h_vel_y,
                    nb.h_vel_z, nb.h_acc1_x, nb.h_acc1_y, nb.h_acc1_z, nb.h_a1dot_x,
                    nb.h_a1dot_y, nb.h_a1dot_z, nb.sys);
  double t2 = omp_get_wtime();
  nb.snapandcrackle();
  nb.correction();
  swap_derivs(nb);
  double t3e = omp_get_wtime();
  t3[0] = t1 - t0;
  t3[1] = t2 - t1;
  t3[2] = t3e - t2;
}

void ref_bench_destroy(void* h) {
  RefBench* rb = (RefBench*)h;
  delete rb->nb;
  delete rb;
}

}  // extern "C"
