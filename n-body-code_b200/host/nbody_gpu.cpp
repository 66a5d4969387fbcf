// nbody_b200::NBody over the GPU engine; see nbody_gpu.h.
#include "nbody_gpu.h"

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <stdexcept>

namespace nbody_b200 {

NBody::NBody(int Nparticles, double v_max, double r_max, double m_min, double m_max,
             const Options& opt)
    : N(Nparticles), vmax(v_max), rmax(r_max), mmin(m_min), mmax(m_max), opt_(opt) {
  alpha = n + 1.0;
  sys.N = N;
  sys.start = 0;
  sys.end = N;
  store_.assign(static_cast<size_t>(13) * N, 0.0);
  double* p = store_.data();
  double** arrs[13] = {&h_par_x, &h_par_y, &h_par_z, &h_par_w, &h_vel_x, &h_vel_y, &h_vel_z,
                       &h_acc_x, &h_acc_y, &h_acc_z, &h_adot_x, &h_adot_y, &h_adot_z};
  for (int k = 0; k < 13; ++k) *arrs[k] = p + static_cast<size_t>(k) * N;
  nbody_config c;
  nbody_config_init(&c);
  c.n = N;
  c.eps2 = opt.eps2;
  c.precision = opt.precision;
  c.device = opt.device;
  c.dt = opt.fixed_dt;
  c.tune = opt.tune ? 1 : 0;
  c.pair_variant = opt.pair_variant;
  check(nbody_create(&eng_, &c), "nbody_create");
  nbody_timers t;
  check(nbody_get_timers(eng_, &t), "nbody_get_timers");
  sys.num_cores = t.num_sms;
}

NBody::~NBody() { nbody_destroy(eng_); }

void NBody::check(nbody_status s, const char* what) const {
  if (s != NBODY_OK)
    throw std::runtime_error(std::string(what) + ": " + nbody_status_string(s) + ": " +
                             nbody_last_error());
}

void NBody::initialize() {
  if (!opt_.load_path.empty()) {
    int n = 0;
    double t = 0, d = 0, e2 = 0;
    check(nbody_read_state_file(opt_.load_path.c_str(), N, &n, &t, &d, &e2, h_par_x, h_par_y,
                                h_par_z, h_par_w, h_vel_x, h_vel_y, h_vel_z),
          "nbody_read_state_file");
    if (n != N) throw std::runtime_error("state file body count differs from --N");
    upload();
    check(nbody_set_time(eng_, t, d), "nbody_set_time");
    return;
  }
  if (opt_.plummer)
    check(nbody_plummer(N, opt_.seed, h_par_x, h_par_y, h_par_z, h_par_w, h_vel_x, h_vel_y, h_vel_z),
          "nbody_plummer");
  else
    check(nbody_reference_ic(N, opt_.eps2, h_par_x, h_par_y, h_par_z, h_par_w, h_vel_x, h_vel_y,
                             h_vel_z),
          "nbody_reference_ic");
  upload();
}

void NBody::initializewithzeros() {
  for (int i = 0; i < N; ++i)
    h_par_x[i] = h_par_y[i] = h_par_z[i] = h_par_w[i] = h_vel_x[i] = h_vel_y[i] = h_vel_z[i] = 0.0;
  upload();
}

void NBody::upload() {
  check(nbody_set_state(eng_, h_par_x, h_par_y, h_par_z, h_par_w, h_vel_x, h_vel_y, h_vel_z),
        "nbody_set_state");
}

void NBody::download() {
  check(nbody_get_state(eng_, h_par_x, h_par_y, h_par_z, h_vel_x, h_vel_y, h_vel_z),
        "nbody_get_state");
  check(nbody_get_derivs(eng_, h_acc_x, h_acc_y, h_acc_z, h_adot_x, h_adot_y, h_adot_z),
        "nbody_get_derivs");
}

double NBody::initialdt() {
  check(nbody_acc_jerk(eng_), "nbody_acc_jerk");
  nbody_timers t;
  check(nbody_get_timers(eng_, &t), "nbody_get_timers");
  sys.t_eval_init = t.eval_init_ms * 1e-3;
  dt = t.dt;
  return dt;
}

void NBody::prediction() { check(nbody_predict(eng_), "nbody_predict"); }
void NBody::force_calculation() { check(nbody_eval_predicted(eng_), "nbody_eval_predicted"); }
void NBody::correction() { check(nbody_correct(eng_), "nbody_correct"); }

double NBody::updatedt() {
  nbody_timers t;
  check(nbody_get_timers(eng_, &t), "nbody_get_timers");
  dt = t.dt;
  return dt;
}

void NBody::timestepping() {
  check(nbody_step(eng_, 1), "nbody_step");
  nbody_timers t;
  check(nbody_get_timers(eng_, &t), "nbody_get_timers");
  sys.t_pred = t.pred_ms * 1e-3;
  sys.t_eval = t.eval_ms * 1e-3;
  sys.t_corr = t.corr_ms * 1e-3;
  dt = t.dt;
}

void NBody::energy(double* t, double* u) {
  check(nbody_energy(eng_, opt_.reference_energy ? 1 : 0, t, u), "nbody_energy");
}

double NBody::time() const {
  nbody_timers t;
  check(nbody_get_timers(eng_, &t), "nbody_get_timers");
  return t.t;
}

void NBody::save(const std::string& path) {
  download();
  nbody_timers t;
  check(nbody_get_timers(eng_, &t), "nbody_get_timers");
  check(nbody_write_state_file(path.c_str(), N, t.t, t.dt, opt_.eps2, h_par_x, h_par_y, h_par_z,
                               h_par_w, h_vel_x, h_vel_y, h_vel_z),
        "nbody_write_state_file");
}

// The reference's cycle() (src/nbody.cpp:291-380): initial conditions, the
// first force evaluation and dt, E0, then ncycle steps with per-phase
// timers.  The energy is evaluated at the end only; the reference evaluates
// it after every cycle but prints only the last value.
void NBody::cycle(int ncycle) {
  sys.t_evalv.assign(ncycle, 0.0);
  sys.t_predv.assign(ncycle, 0.0);
  sys.t_corrv.assign(ncycle, 0.0);
  initialize();
  initialdt();
  energy(&T, &U);
  sys.initE = T + U;
  for (int i = 0; i < ncycle; ++i) {
    timestepping();
    sys.t_predv[i] = sys.t_pred;
    sys.t_evalv[i] = sys.t_eval;
    sys.t_corrv[i] = sys.t_corr;
  }
  energy(&T, &U);
  sys.finE = T + U;
  sys.Q = -2.0 * T / U;
  sys.Err = std::abs(sys.finE - sys.initE) / std::abs(sys.initE);
  download();
}

}  // namespace nbody_b200
