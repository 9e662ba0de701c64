// Test driver: runs PAWAN's own offline time loop __integration::integrate
// (src/integration/integration.cpp:96-132) on particles read from a file,
// either with PAWAN's OpenMP backend (__parallel + __rk4/__rk3) or with the
// drop-in GPU classes (__gpu + __rk4gpu/__rk3gpu), writing <out>.wake and
// <out>.diagnosis through PAWAN's own writers.
//
//   dropin_check ref|gpu|gpu64|gpuasync|gpu64async rk4|rk3 <particles.bin> <dt> <nsteps> <out-prefix> [nu]
//
// particles.bin: int64 n, then n*3 positions, n*3 strengths, n radii, n volumes (FP64).
// The *async modes call integrate on the __rk4gpu / __rk3gpu itself, which
// keeps the state on the device and writes the .wake records from
// asynchronous snapshots (__gpu::integrate_on_device); the others call it
// through __integration *, PAWAN's own loop.  The wall time of integrate goes
// to stderr as "integrate_seconds <s>".
//
// A second mode runs PAWAN's strength solve __resolve::rebuild
// (src/resolve/resolve.cpp:12-63) on one of PAWAN's own __vring wakes
// (src/wake/vring.cpp), whose O(N^2) part is __interaction::resolve ->
// influence(), with either backend, and writes the solved strengths (FP64)
// to <out-prefix>.strengths:
//
//   dropin_check resolve ref|gpu|gpu64 <nLayers> <nAzi> <sigma> <out-prefix>
//
// A third mode runs PAWAN's relaxation __interaction::relax(stepnum)
// (interaction.cpp:367-371: each wake's split, then merge, wake.cpp:61-165)
// once, with either backend, on particles read from a file:
//
//   dropin_check relax ref|gpu|gpu64 <particles.bin> <ages.bin> <stepnum> <out-prefix>
//
// ages.bin: int64 n, then n birth steps (_active) and n birth strengths.  The
// wake is laid out as in the coupled run (__wake::initialise_memory,
// wake.cpp:27-44: MAXNUMPARTICLES rows, _npidx = n) so split can append.
// Output <out-prefix>.relax: int64 n, then n*3 positions, n*3 strengths,
// n radii, n volumes, n birth strengths, n birth steps (FP64).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <chrono>
#include <string>
#include <vector>

#include "pawan_gpu_dropin.h"
#include "src/interaction/parallel.h"
#include "src/io/io.h"
#include "src/resolve/resolve.h"
#include "src/wake/vring.h"

namespace {

struct file_wake : public pawan::__wake {
  explicit file_wake(const std::vector<double> &d, int64_t n) : pawan::__wake() {
    gsl_matrix_free(_position); gsl_matrix_free(_velocity); gsl_matrix_free(_vorticity);
    gsl_matrix_free(_retvorcity); gsl_vector_free(_radius); gsl_vector_free(_volume);
    gsl_vector_free(_birthstrength); gsl_matrix_free(_vorticityfield); gsl_vector_free(_active);
    create_particles((int)n);
    for (int64_t i = 0; i < n; ++i) {
      for (int k = 0; k < 3; ++k) {
        gsl_matrix_set(_position, i, k, d[3 * i + k]);
        gsl_matrix_set(_vorticity, i, k, d[3 * n + 3 * i + k]);
      }
      gsl_vector_set(_radius, i, d[6 * n + i]);
      gsl_vector_set(_volume, i, d[7 * n + i]);
    }
  }
};

// A wake with PAWAN's coupled-run layout (capacity MAXNUMPARTICLES) holding n particles.
struct coupled_wake : public pawan::__wake {
  coupled_wake(const std::vector<double> &d, const std::vector<double> &ages, int64_t n) : pawan::__wake() {
    gsl_matrix_free(_position); gsl_matrix_free(_velocity); gsl_matrix_free(_vorticity);
    gsl_matrix_free(_retvorcity); gsl_vector_free(_radius); gsl_vector_free(_volume);
    gsl_vector_free(_birthstrength); gsl_matrix_free(_vorticityfield); gsl_vector_free(_active);
    initialise_memory();
    for (int64_t i = 0; i < n; ++i) {
      for (int k = 0; k < 3; ++k) {
        gsl_matrix_set(_position, i, k, d[3 * i + k]);
        gsl_matrix_set(_vorticity, i, k, d[3 * n + 3 * i + k]);
      }
      gsl_vector_set(_radius, i, d[6 * n + i]);
      gsl_vector_set(_volume, i, d[7 * n + i]);
      gsl_vector_set(_active, i, ages[i]);
      gsl_vector_set(_birthstrength, i, ages[n + i]);
    }
    _npidx = (size_t)n;
    _numParticles = (size_t)n;
    _size = 2 * _numParticles * 3;
  }
};

struct path_io : public pawan::__io {
  std::string p;
  explicit path_io(const std::string &s) : p(s) {}
  FILE *create_binary_file(std::string suffix) override { return fopen((p + suffix).c_str(), "wb"); }
};

struct ref_parallel : public pawan::__parallel {
  ref_parallel(pawan::__wake *W, double nu) : pawan::__parallel(W) { _nu = nu; }
};

}  // namespace

int run_resolve(int argc, char **argv) {
  if (argc < 7) {
    fprintf(stderr, "usage: %s resolve ref|gpu|gpu64 nLayers nAzi sigma out\n", argv[0]);
    return 2;
  }
  const std::string backend = argv[2];
  pawan::__wake *W = new pawan::__vring(1.0, 0.1, atoi(argv[3]), atoi(argv[4]), atof(argv[5]));
  path_io io(argv[6]);
  pawan::__interaction *S = nullptr;
  if (backend == "ref") {
    S = new ref_parallel(W, 1e-4);
  } else {
    pgpu_config cfg;
    pgpu_config_default(&cfg);
    cfg.nu = 1e-4;
    cfg.precision = backend == "gpu64" ? PGPU_FP64 : PGPU_FP32C;
    S = new pawan::__gpu(W, cfg);
  }
  pawan::__resolve R;
  R.rebuild(S, &io);
  gsl_vector *st = gsl_vector_calloc(S->_size);
  S->getStates(st);
  FILE *f = fopen((std::string(argv[6]) + ".strengths").c_str(), "wb");
  if (!f) return 3;
  fwrite(st->data, sizeof(double), st->size, f);
  fclose(f);
  gsl_vector_free(st);
  fflush(NULL);
  delete S;
  delete W;
  return 0;
}

static bool read_doubles(const char *path, int64_t per, std::vector<double> &d, int64_t &n) {
  FILE *f = fopen(path, "rb");
  if (!f) return false;
  bool ok = fread(&n, sizeof(n), 1, f) == 1 && n >= 0;
  if (ok) {
    d.resize((size_t)(per * n));
    ok = fread(d.data(), sizeof(double), d.size(), f) == d.size();
  }
  fclose(f);
  return ok;
}

int run_relax(int argc, char **argv) {
  if (argc < 7) {
    fprintf(stderr, "usage: %s relax ref|gpu|gpu64 particles.bin ages.bin stepnum out\n", argv[0]);
    return 2;
  }
  const std::string backend = argv[2];
  std::vector<double> d, ages;
  int64_t n = 0, na = 0;
  if (!read_doubles(argv[3], 8, d, n) || !read_doubles(argv[4], 2, ages, na) || na != n) return 3;
  coupled_wake W(d, ages, n);
  pawan::__interaction *S = nullptr;
  if (backend == "ref") {
    S = new ref_parallel(&W, 1e-4);
  } else {
    pgpu_config cfg;
    pgpu_config_default(&cfg);
    cfg.nu = 1e-4;
    cfg.precision = backend == "gpu64" ? PGPU_FP64 : PGPU_FP32C;
    S = new pawan::__gpu(&W, cfg);
  }
  size_t stepnum = (size_t)atoll(argv[5]);
  S->relax(stepnum);
  FILE *f = fopen((std::string(argv[6]) + ".relax").c_str(), "wb");
  if (!f) return 3;
  const int64_t m = (int64_t)W._numParticles;
  fwrite(&m, sizeof(m), 1, f);
  for (int64_t i = 0; i < m; ++i)
    for (int k = 0; k < 3; ++k) { double v = gsl_matrix_get(W._position, i, k); fwrite(&v, sizeof(v), 1, f); }
  for (int64_t i = 0; i < m; ++i)
    for (int k = 0; k < 3; ++k) { double v = gsl_matrix_get(W._vorticity, i, k); fwrite(&v, sizeof(v), 1, f); }
  for (int64_t i = 0; i < m; ++i) { double v = gsl_vector_get(W._radius, i); fwrite(&v, sizeof(v), 1, f); }
  for (int64_t i = 0; i < m; ++i) { double v = gsl_vector_get(W._volume, i); fwrite(&v, sizeof(v), 1, f); }
  for (int64_t i = 0; i < m; ++i) { double v = gsl_vector_get(W._birthstrength, i); fwrite(&v, sizeof(v), 1, f); }
  for (int64_t i = 0; i < m; ++i) { double v = gsl_vector_get(W._active, i); fwrite(&v, sizeof(v), 1, f); }
  fclose(f);
  fflush(NULL);
  delete S;
  return 0;
}

int main(int argc, char **argv) {
  if (argc > 1 && std::string(argv[1]) == "resolve") return run_resolve(argc, argv);
  if (argc > 1 && std::string(argv[1]) == "relax") return run_relax(argc, argv);
  if (argc < 7) {
    fprintf(stderr, "usage: %s ref|gpu|gpu64 rk4|rk3 particles.bin dt nsteps out [nu]\n", argv[0]);
    return 2;
  }
  const std::string mode = argv[1], scheme = argv[2];
  const double dt = atof(argv[4]);
  const int nsteps = atoi(argv[5]);
  const double nu = argc > 7 ? atof(argv[7]) : 1e-4;
  FILE *f = fopen(argv[3], "rb");
  if (!f) return 3;
  int64_t n = 0;
  if (fread(&n, sizeof(n), 1, f) != 1) return 3;
  std::vector<double> d(8 * n);
  if (fread(d.data(), sizeof(double), d.size(), f) != d.size()) return 3;
  fclose(f);

  file_wake W(d, n);
  path_io io(argv[6]);
  pawan::__interaction *S = nullptr;
  pawan::__integration *I = nullptr;
  const double T = dt * nsteps;
  const bool async = mode.size() > 5 && mode.compare(mode.size() - 5, 5, "async") == 0;
  const auto t0 = std::chrono::steady_clock::now();
  if (mode == "ref") {
    S = new ref_parallel(&W, nu);
    I = scheme == "rk3" ? (pawan::__integration *)new pawan::__rk3(T, nsteps) : new pawan::__rk4(T, nsteps);
  } else {
    pgpu_config cfg;
    pgpu_config_default(&cfg);
    cfg.nu = nu;
    cfg.precision = mode.compare(0, 5, "gpu64") == 0 ? PGPU_FP64 : PGPU_FP32C;
    S = new pawan::__gpu(&W, cfg);
    if (scheme == "rk3") {
      auto *R = new pawan::__rk3gpu(T, nsteps);
      I = R;
      if (async) R->integrate(S, &io, true);
    } else {
      auto *R = new pawan::__rk4gpu(T, nsteps);
      I = R;
      if (async) R->integrate(S, &io, true);
    }
  }
  if (!async) I->integrate(S, &io, true);
  fflush(NULL);
  fprintf(stderr, "integrate_seconds %.6f\n",
          std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count());
  delete I;
  delete S;
  return 0;
}
