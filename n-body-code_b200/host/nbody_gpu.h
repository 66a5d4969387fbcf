// nbody_b200::NBody - the reference's NBody class surface (include/nbody.h:24-59)
// with every phase running on the GPU engine (include/nbody_cuda.h).
//
// Public members keep the reference's names: the SoA host arrays h_par_x ...
// h_adot_z, dt, T, U and the run-state struct sys (include/utils.h:31-53).
// The device holds the authoritative state; the host arrays are filled by
// download() and by cycle() at its end, and pushed by upload().
//
// Methods map onto the reference's (src/nbody.cpp):
//   initialize()      69-114   reference initial conditions (or a Plummer sphere)
//   initialdt()       131-150  acc/jerk of the current state + initial criterion
//   prediction()      152-163
//   force_calculation()        acc/jerk of the predicted state (kernel.cpp)
//   correction()      165-196  snapandcrackle + correction + a<->a1 swap, fused
//   updatedt()        198-222  the Aarseth criterion of the last correction
//   timestepping()    224-289  one graph-replayed step
//   cycle(n)          291-380  the reference's run: ICs, E0, n steps, final E
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "nbody_cuda.h"

namespace nbody_b200 {

// The reference's run-state fields (include/utils.h:31-53).
struct Sys {
  int N = 0, start = 0, end = 0, rank = 0, size = 1, nthreads = 1, thid = 0;
  double t_eval = 0, t_pred = 0, t_corr = 0, t_eval_init = 0;
  double kernel_time = 0, kernel_time_init = 0;
  std::vector<double> t_evalv, t_predv, t_corrv;
  double initE = 0, finE = 0, Q = 0, Err = 0;
  int num_cores = 0;
};

struct Options {
  double eps2 = 1.0e-7;        // the reference's EPS2 (include/kernel.h:13)
  int precision = NBODY_FP64;  // or NBODY_MIXED
  double fixed_dt = 0.0;       // > 0: shared fixed step; <= 0: adaptive (the reference)
  bool plummer = false;        // Plummer sphere instead of the reference ICs
  uint64_t seed = 1;           // Plummer seed
  bool reference_energy = true;  // the reference's printed potential (m_j^2 term)
  int device = 0;
  bool tune = false;
  int pair_variant = 0;        // mixed kernel (nbody_config.pair_variant; 0 = automatic)
  std::string load_path;       // start from a state file instead of fresh ICs
};

class NBody {
 public:
  double alpha;
  double n = -2.35;
  double T = 0, U = 0;
  int size = 1, rank = 0;
  Sys sys;
  double *h_par_x, *h_par_y, *h_par_z, *h_par_w;
  double *h_vel_x, *h_vel_y, *h_vel_z;
  double *h_acc_x, *h_acc_y, *h_acc_z;
  double *h_adot_x, *h_adot_y, *h_adot_z;
  double dt = 0;

  NBody(int Nparticles, double v_max, double r_max, double m_min, double m_max,
        const Options& opt = Options());
  ~NBody();
  NBody(const NBody&) = delete;
  NBody& operator=(const NBody&) = delete;

  void initialize();
  void initializewithzeros();
  double initialdt();
  void prediction();
  void force_calculation();
  void correction();
  double updatedt();
  void timestepping();
  void cycle(int ncycle);

  void upload();                   // host arrays -> device
  void download();                 // device -> host arrays (x, v, acc, jerk)
  void energy(double* T, double* U);
  void save(const std::string& path);
  double time() const;
  nbody_engine* engine() { return eng_; }

 private:
  void check(nbody_status s, const char* what) const;
  int N;
  double vmax, rmax, mmin, mmax;
  Options opt_;
  nbody_engine* eng_ = nullptr;
  std::vector<double> store_;
};

}  // namespace nbody_b200
