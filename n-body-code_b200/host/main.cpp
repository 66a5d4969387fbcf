// nbody_app - the reference's command-line driver (src/main.cpp) on the GPU
// engine.  Same flags and output table:
//   nbody_app [--N <n>] [--Ncycle <c>]
// prints the per-cycle PRED / EVAL / CORR times, the initial evaluation time,
// initial and final energy, Q, Err, wall time and the device's SM count.
// Extra flags (all optional; the defaults reproduce the reference's run):
//   --eps <e>              softening length (eps^2 = e^2; default eps^2 = 1e-7)
//   --dt <h>               fixed shared step (default: adaptive, as the reference)
//   --precision fp64|mixed
//   --ic reference|plummer --seed <s>
//   --energy reference|physical   potential with the reference's m_j^2 term
//                                  (default for reference ICs) or m_i m_j
//   --load <file> / --dump <file>  state files (nbody_read/write_state_file)
//   --device <d> --tune
//   --pair-variant <v>     mixed kernel: 0 automatic, 1-3 hi/lo forms, 4 tile-relative
#include <chrono>
#include <cmath>
#include <cstdio>
#include <ctime>
#include <iomanip>
#include <iostream>
#include <stdexcept>
#include <string>
#include <sys/time.h>

#include "nbody_gpu.h"

namespace {

constexpr int kColWidth = 15;  // src/main.cpp:11

double timestamp() {
  timeval tv;
  gettimeofday(&tv, nullptr);
  return tv.tv_sec + tv.tv_usec * 1e-6;
}

int usage(const std::string& arg) {
  std::cerr << "Unknown or incomplete argument: " << arg << std::endl;
  std::cerr << "Usage: ./nbody_app [--N <value>] [--Ncycle <value>] [--eps <e>] [--dt <h>] "
               "[--precision fp64|mixed] [--ic reference|plummer] [--seed <s>] "
               "[--energy reference|physical] [--load <file>] [--dump <file>] [--device <d>] "
               "[--tune] [--pair-variant <v>]"
            << std::endl;
  return 1;
}

}  // namespace

int main(int argc, char* argv[]) {
  int N = 16384, Ncycle = 10;  // src/main.cpp:16-17
  nbody_b200::Options opt;
  std::string energy_mode, dump_path;
  for (int i = 1; i < argc; ++i) {
    const std::string arg = argv[i];
    const bool has = i + 1 < argc;
    try {
      if (arg == "--N" && has) {
        N = std::stoi(argv[++i]);
        if (N <= 0) throw std::invalid_argument("N must be positive.");
      } else if (arg == "--Ncycle" && has) {
        Ncycle = std::stoi(argv[++i]);
        if (Ncycle <= 0) throw std::invalid_argument("Ncycle must be positive.");
      } else if (arg == "--eps" && has) {
        const double e = std::stod(argv[++i]);
        opt.eps2 = e * e;
      } else if (arg == "--dt" && has) {
        opt.fixed_dt = std::stod(argv[++i]);
      } else if (arg == "--precision" && has) {
        const std::string p = argv[++i];
        if (p != "fp64" && p != "mixed") return usage(arg);
        opt.precision = p == "mixed" ? NBODY_MIXED : NBODY_FP64;
      } else if (arg == "--ic" && has) {
        const std::string p = argv[++i];
        if (p != "reference" && p != "plummer") return usage(arg);
        opt.plummer = p == "plummer";
      } else if (arg == "--seed" && has) {
        opt.seed = std::stoull(argv[++i]);
      } else if (arg == "--energy" && has) {
        energy_mode = argv[++i];
        if (energy_mode != "reference" && energy_mode != "physical") return usage(arg);
      } else if (arg == "--load" && has) {
        opt.load_path = argv[++i];
      } else if (arg == "--dump" && has) {
        dump_path = argv[++i];
      } else if (arg == "--device" && has) {
        opt.device = std::stoi(argv[++i]);
      } else if (arg == "--tune") {
        opt.tune = true;
      } else if (arg == "--pair-variant" && has) {
        opt.pair_variant = std::stoi(argv[++i]);
      } else {
        return usage(arg);
      }
    } catch (const std::exception& e) {
      std::cerr << "Error parsing " << arg << ": " << e.what() << std::endl;
      return 1;
    }
  }
  opt.reference_energy = energy_mode.empty() ? !opt.plummer : energy_mode == "reference";

  std::cout << "Using N = " << N << ", Ncycle = " << Ncycle << std::endl;
  const double vmax = 1.0, mmin = 0.01, mmax = 1.0, rmax = 1.0;  // src/main.cpp:73-76
  try {
    const auto t0 = std::chrono::steady_clock::now();
    nbody_b200::NBody nbody(N, vmax, rmax, mmin, mmax, opt);
    nbody.cycle(Ncycle);
    const double wall =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();

    std::cout << std::fixed << std::setprecision(9);
    std::cout << "Time stamp(start): " << timestamp() << std::endl << std::endl;
    std::cout << std::setw(kColWidth) << "N" << std::setw(kColWidth) << "NPES"
              << std::setw(kColWidth) << "PRED" << std::setw(kColWidth) << "EVAL"
              << std::setw(kColWidth) << "CORR" << std::setw(kColWidth) << "NCYCLE" << std::endl;
    std::cout << std::string(kColWidth * 6, '-') << std::endl;
    for (int i = 0; i < Ncycle; ++i)
      std::cout << std::setw(kColWidth) << N << std::setw(kColWidth) << nbody.sys.size
                << std::setw(kColWidth) << nbody.sys.t_predv[i] << std::setw(kColWidth)
                << nbody.sys.t_evalv[i] << std::setw(kColWidth) << nbody.sys.t_corrv[i]
                << std::setw(kColWidth) << i << std::endl;
    std::cout << "\nInitial Evaluation Time: " << nbody.sys.t_eval_init << std::endl;
    std::cout << "Initial Energy: " << nbody.sys.initE << std::endl;
    std::cout << "Final Energy: " << nbody.sys.finE << std::endl;
    std::cout << "Q = " << nbody.sys.Q << std::endl;
    std::cout << "Err = " << nbody.sys.Err << std::endl;
    std::cout << "WALL time: " << wall << " seconds" << std::endl;
    std::cout << "Total active cores: " << nbody.sys.num_cores << std::endl << std::endl;
    std::cout << "Time stamp (end): " << timestamp() << std::endl;
    if (!dump_path.empty()) nbody.save(dump_path);
  } catch (const std::exception& e) {
    std::cerr << "nbody_app: " << e.what() << std::endl;
    return 2;
  }
  return 0;
}
