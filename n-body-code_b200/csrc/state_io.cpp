// Binary SoA state files (resume and exchange with the oracle).
//
// Layout, little-endian: a 64-byte header
//   char magic[8] = "NBODYST1"; int32 version = 1; int32 n;
//   double t; double dt; double eps2; 24 bytes zero
// followed by seven float64 arrays of n values: x, y, z, m, vx, vy, vz.
#include <cstdio>
#include <cstring>

#include "../../include/nbody_cuda.h"
#include "errors.h"

namespace {

struct Header {
  char magic[8];
  int32_t version;
  int32_t n;
  double t, dt, eps2;
  char pad[24];
};
static_assert(sizeof(Header) == 64, "state header is 64 bytes");
constexpr char kMagic[8] = {'N', 'B', 'O', 'D', 'Y', 'S', 'T', '1'};

}  // namespace

extern "C" nbody_status nbody_write_state_file(const char* path, int n, double t, double dt,
                                               double eps2, const double* x, const double* y,
                                               const double* z, const double* m,
                                               const double* vx, const double* vy,
                                               const double* vz) {
  if (!path || n < 1 || !x || !y || !z || !m || !vx || !vy || !vz)
    return nbody_set_error(NBODY_ERR_INVALID_ARG, "nbody_write_state_file: bad argument");
  FILE* f = std::fopen(path, "wb");
  if (!f) return nbody_set_error(NBODY_ERR_INVALID_ARG, "cannot open %s for writing", path);
  Header h;
  std::memset(&h, 0, sizeof h);
  std::memcpy(h.magic, kMagic, 8);
  h.version = 1;
  h.n = n;
  h.t = t;
  h.dt = dt;
  h.eps2 = eps2;
  bool ok = std::fwrite(&h, sizeof h, 1, f) == 1;
  const double* arr[7] = {x, y, z, m, vx, vy, vz};
  for (int k = 0; ok && k < 7; ++k) ok = std::fwrite(arr[k], sizeof(double), n, f) == (size_t)n;
  ok = (std::fclose(f) == 0) && ok;
  return ok ? NBODY_OK : nbody_set_error(NBODY_ERR_INVALID_ARG, "short write to %s", path);
}

extern "C" nbody_status nbody_read_state_file(const char* path, int n_max, int* n, double* t,
                                              double* dt, double* eps2, double* x, double* y,
                                              double* z, double* m, double* vx, double* vy,
                                              double* vz) {
  if (!path || !n) return nbody_set_error(NBODY_ERR_INVALID_ARG, "nbody_read_state_file: bad argument");
  FILE* f = std::fopen(path, "rb");
  if (!f) return nbody_set_error(NBODY_ERR_INVALID_ARG, "cannot open %s", path);
  Header h;
  if (std::fread(&h, sizeof h, 1, f) != 1 || std::memcmp(h.magic, kMagic, 8) != 0 ||
      h.version != 1 || h.n < 1) {
    std::fclose(f);
    return nbody_set_error(NBODY_ERR_INVALID_ARG, "%s is not a state file", path);
  }
  *n = h.n;
  if (t) *t = h.t;
  if (dt) *dt = h.dt;
  if (eps2) *eps2 = h.eps2;
  double* arr[7] = {x, y, z, m, vx, vy, vz};
  bool want = false;
  for (auto p : arr) want = want || p;
  if (!want) {  // header query only
    std::fclose(f);
    return NBODY_OK;
  }
  if (h.n > n_max) {
    std::fclose(f);
    return nbody_set_error(NBODY_ERR_INVALID_ARG, "%s holds %d bodies, buffers hold %d", path, h.n, n_max);
  }
  bool ok = true;
  for (int k = 0; ok && k < 7; ++k) {
    if (!arr[k]) return std::fclose(f), nbody_set_error(NBODY_ERR_INVALID_ARG, "null array");
    ok = std::fread(arr[k], sizeof(double), h.n, f) == (size_t)h.n;
  }
  std::fclose(f);
  return ok ? NBODY_OK : nbody_set_error(NBODY_ERR_INVALID_ARG, "%s is truncated", path);
}
