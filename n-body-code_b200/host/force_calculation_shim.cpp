// The reference-side binding: a drop-in definition of the reference's
//   void force_calculation(13 x double*, Sys&)        (include/kernel.h:15-19)
// that forwards to libnbody_cuda (include/nbody_cuda.h).  A maintainer adds
// this file to the reference's build in place of src/kernel.cpp and links
// -lnbody_cuda; NBody (src/nbody.cpp) and the driver (src/main.cpp) are
// unchanged.  It compiles against the reference's own headers (for Sys and
// EPS2), which are on the include path of that build.
//
// Semantics kept from the reference: the six outputs are zeroed and rows
// [sys.start, sys.end) are filled, so the per-rank MPI_Allreduce that follows
// in NBody (src/nbody.cpp:240-246, 318-324) assembles the full result; with
// one rank start = 0, end = N.  Softening is the reference's EPS2.  The
// precision defaults to FP64; NBODY_PRECISION=mixed selects the mixed path.
// Errors abort with the library's message (the reference's force back ends
// have no error return).
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "kernel.h"       // reference: EPS2, force_calculation declaration
#include "nbody_cuda.h"   // this engine
#include "utils.h"        // reference: Sys

void force_calculation(double* __restrict x, double* __restrict y, double* __restrict z,
                       double* __restrict m, double* __restrict vx, double* __restrict vy,
                       double* __restrict vz, double* __restrict ax, double* __restrict ay,
                       double* __restrict az, double* __restrict jx, double* __restrict jy,
                       double* __restrict jz, Sys& sys) {
  static const int precision = [] {
    const char* p = std::getenv("NBODY_PRECISION");
    return (p && std::strcmp(p, "mixed") == 0) ? NBODY_MIXED : NBODY_FP64;
  }();
  const nbody_status s = nbody_force_calculation(sys.N, EPS2, precision, sys.start, sys.end, x, y,
                                                 z, m, vx, vy, vz, ax, ay, az, jx, jy, jz);
  if (s != NBODY_OK) {
    std::fprintf(stderr, "force_calculation (libnbody_cuda): %s: %s\n", nbody_status_string(s),
                 nbody_last_error());
    std::abort();
  }
}
