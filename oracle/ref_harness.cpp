/*
 * C entry points around PAWAN's own, unmodified classes so the Python tests and
 * the CPU-baseline leg of bench.py can drive the reference solver through
 * ctypes.  TEST INFRASTRUCTURE ONLY: this is the checker, never the product.
 *
 * Hooks used (subclassing only, no PAWAN source is edited):
 *   - oracle_wake      : calls the protected __wake::create_particles(n)
 *                        (src/wake/wake.h:35, wake.cpp:10-25) so a wake holds
 *                        exactly n particles instead of MAXNUMPARTICLES rows.
 *   - oracle_sys<B>    : sets the protected viscosity _nu (interaction.h:25),
 *                        which the base constructor hard-codes to 1.56e-5
 *                        (interaction.cpp:15), and reads the protected
 *                        diagnostics members after diagnose().
 *   - oracle_int<B>    : exposes the protected virtual step()
 *                        (integration.h:37, rk4.h:25, rk3.h:25).
 *   - oracle_io        : overrides the virtual create_binary_file (io.h:53)
 *                        because the reference hard-codes its data root
 *                        (io.cpp:14).
 */
#include <stdint.h>
#include <string>
#include <vector>

#include "src/interaction/interaction.h"
#include "src/interaction/parallel.h"
#include "src/integration/integration.h"
#include "src/integration/rk3.h"
#include "src/integration/rk4.h"
#include "src/io/io.h"
#include "src/wake/wake.h"
#include "src/interaction/gaussian.h"

// Five-argument kernel that interaction.cpp:465 calls; forwards to the
// six-argument kernel of the build: the Gaussian one (gaussian.h:47-60), or the
// high-order one (highorder.h:54-61) when ref_highorder.h is force-included,
// which also turns the include of gaussian.h above into an empty one.
void KERNEL(const double &rho, const double &sigma, double &q, double &F, double &Z) {
  double n = 0.0;
  KERNEL(rho, sigma, q, F, Z, n);
}

namespace {

struct oracle_wake : public pawan::__wake {
  explicit oracle_wake(int n) : pawan::__wake() {
    // __wake() allocated one particle; replace it with n rows.
    gsl_matrix_free(_position);
    gsl_matrix_free(_velocity);
    gsl_matrix_free(_vorticity);
    gsl_matrix_free(_retvorcity);
    gsl_vector_free(_radius);
    gsl_vector_free(_volume);
    gsl_vector_free(_birthstrength);
    gsl_matrix_free(_vorticityfield);
    gsl_vector_free(_active);
    create_particles(n);
  }
};

struct sys_iface {
  virtual ~sys_iface() {}
  virtual pawan::__interaction *sys() = 0;
  virtual void diag(double *out) = 0;
};

template <class B>
struct oracle_sys : public B, public sys_iface {
  oracle_sys(pawan::__wake *W, double nu) : B(W) { this->_nu = nu; }
  pawan::__interaction *sys() override { return this; }
  void diag(double *out) override {
    this->diagnose();
    for (int k = 0; k < 3; ++k) out[k] = gsl_vector_get(this->_totalVorticity, k);
    for (int k = 0; k < 3; ++k) out[3 + k] = gsl_vector_get(this->_linearImpulse, k);
    for (int k = 0; k < 3; ++k) out[6 + k] = gsl_vector_get(this->_angularImpulse, k);
    out[9] = this->_helicity;
    out[10] = this->_enstrophy;
    out[11] = this->_enstrophyF;
    out[12] = this->_kineticEnergy;
    out[13] = this->_kineticEnergyF;
    out[14] = this->_Zc;
  }
};

template <class B>
struct oracle_int : public B {
  oracle_int(double t, size_t n) : B(t, n) {}
  void do_step(double dt, pawan::__system *S, gsl_vector *st) { this->step(dt, S, st); }
};
// Plain __integration's step is explicit Euler (integration.cpp:198-208).
struct oracle_euler : public pawan::__integration {
  oracle_euler(double t, size_t n) : pawan::__integration(t, n) {}
  void do_step(double dt, pawan::__system *S, gsl_vector *st) { this->step(dt, S, st); }
};

struct oracle_io : public pawan::__io {
  std::string path;
  explicit oracle_io(const std::string &p) : path(p) {}
  FILE *create_binary_file(std::string suffix) override { return fopen((path + suffix).c_str(), "wb"); }
  FILE *open_binary_file(std::string suffix) override { return fopen((path + suffix).c_str(), "rb"); }
};

struct handle {
  std::vector<oracle_wake *> wakes;
  sys_iface *S = nullptr;
};

}  // namespace

extern "C" {

// backend: 0 = serial __interaction, 1 = OpenMP __parallel (the default
// backend in src/pawan.cpp:48).
void *ref_create(int nwakes, const int64_t *n, double nu, int backend) {
  handle *h = new handle;
  for (int w = 0; w < nwakes; ++w) h->wakes.push_back(new oracle_wake((int)n[w]));
  if (backend == 1) h->S = new oracle_sys<pawan::__parallel>(h->wakes[0], nu);
  else h->S = new oracle_sys<pawan::__interaction>(h->wakes[0], nu);
  for (int w = 1; w < nwakes; ++w) h->S->sys()->addWake(h->wakes[w]);
  return h;
}

void ref_destroy(void *hp) {
  handle *h = (handle *)hp;
  delete h->S;
  for (auto *w : h->wakes) delete w;
  delete h;
}

void ref_set_wake(void *hp, int w, const double *pos, const double *alpha, const double *radius,
                  const double *volume) {
  oracle_wake *W = ((handle *)hp)->wakes[w];
  for (size_t i = 0; i < W->_numParticles; ++i) {
    for (int k = 0; k < 3; ++k) {
      gsl_matrix_set(W->_position, i, k, pos[3 * i + k]);
      gsl_matrix_set(W->_vorticity, i, k, alpha[3 * i + k]);
    }
    gsl_vector_set(W->_radius, i, radius[i]);
    gsl_vector_set(W->_volume, i, volume[i]);
  }
}

void ref_get_wake(void *hp, int w, double *pos, double *alpha) {
  oracle_wake *W = ((handle *)hp)->wakes[w];
  for (size_t i = 0; i < W->_numParticles; ++i)
    for (int k = 0; k < 3; ++k) {
      pos[3 * i + k] = gsl_matrix_get(W->_position, i, k);
      alpha[3 * i + k] = gsl_matrix_get(W->_vorticity, i, k);
    }
}

void ref_solve(void *hp) { ((handle *)hp)->S->sys()->solve(); }

// PAWAN's resolve() (interaction.cpp:59-62: influence() over all wakes), then
// each wake's _vorticityfield, wakes concatenated in order.
void ref_influence(void *hp, double *field) {
  handle *h = (handle *)hp;
  h->S->sys()->resolve();
  size_t row = 0;
  for (oracle_wake *W : h->wakes)
    for (size_t i = 0; i < W->_numParticles; ++i, ++row)
      for (int k = 0; k < 3; ++k) field[3 * row + k] = gsl_matrix_get(W->_vorticityfield, i, k);
}

void ref_get_rates(void *hp, int w, double *vel, double *dalpha) {
  oracle_wake *W = ((handle *)hp)->wakes[w];
  for (size_t i = 0; i < W->_numParticles; ++i)
    for (int k = 0; k < 3; ++k) {
      vel[3 * i + k] = gsl_matrix_get(W->_velocity, i, k);
      dalpha[3 * i + k] = gsl_matrix_get(W->_retvorcity, i, k);
    }
}

// scheme: 0 = Euler, 1 = RK3, 2 = RK4.  Mirrors the body of the offline
// integrate loop (integration.cpp:112-116) without its per-step file dumps.
void ref_step(void *hp, int scheme, double dt, int nsteps) {
  handle *h = (handle *)hp;
  pawan::__interaction *S = h->S->sys();
  gsl_vector *states = gsl_vector_calloc(S->_totalmaxsize);
  oracle_euler eu(dt * nsteps, nsteps);
  oracle_int<pawan::__rk3> r3(dt * nsteps, nsteps);
  oracle_int<pawan::__rk4> r4(dt * nsteps, nsteps);
  for (int i = 0; i < nsteps; ++i) {
    S->getStates(states);
    if (scheme == 2) r4.do_step(dt, S, states);
    else if (scheme == 1) r3.do_step(dt, S, states);
    else eu.do_step(dt, S, states);
  }
  gsl_vector_free(states);
}

// out: total vorticity(3), linear impulse(3), angular impulse(3), helicity,
// enstrophy, enstrophyF, kinetic energy, kinetic energyF, Zc  (15 doubles),
// the record writediagnosis emits (interaction.cpp:325-335).
void ref_diagnose(void *hp, double *out) { ((handle *)hp)->S->diag(out); }

void ref_getvi(void *hp, const double *r, double *out) {
  gsl_vector *rv = gsl_vector_calloc(3), *vi = gsl_vector_calloc(3);
  for (int k = 0; k < 3; ++k) gsl_vector_set(rv, k, r[k]);
  ((handle *)hp)->S->sys()->getVi(rv, vi, 0);
  for (int k = 0; k < 3; ++k) out[k] = gsl_vector_get(vi, k);
  gsl_vector_free(rv);
  gsl_vector_free(vi);
}

// Runs the reference's own offline time loop __integration::integrate
// (integration.cpp:96-132), which writes <path>.wake and, with diagnose,
// <path>.diagnosis.  integrate() never closes the .diagnosis stream, so all
// output streams are flushed before returning.
void ref_integrate(void *hp, int scheme, double t, int n, int diagnose, const char *path) {
  handle *h = (handle *)hp;
  oracle_io io(path);
  if (scheme == 2) { pawan::__rk4 I(t, (size_t)n); I.integrate(h->S->sys(), &io, diagnose != 0); }
  else if (scheme == 1) { pawan::__rk3 I(t, (size_t)n); I.integrate(h->S->sys(), &io, diagnose != 0); }
  else { pawan::__integration I(t, (size_t)n); I.integrate(h->S->sys(), &io, diagnose != 0); }
  fflush(NULL);
}

// PAWAN's own particle merge __wake::merge (wake.cpp:112-159) on wake w, after
// setting the particles' birth steps (_active) that its age test reads.
void ref_merge(void *hp, int w, const double *active, int64_t stepnum) {
  oracle_wake *W = ((handle *)hp)->wakes[w];
  for (size_t i = 0; i < W->_numParticles; ++i) gsl_vector_set(W->_active, i, active[i]);
  size_t s = (size_t)stepnum;
  W->merge(s);
}

void ref_get_particles(void *hp, int w, double *pos, double *alpha, double *radius, double *volume) {
  oracle_wake *W = ((handle *)hp)->wakes[w];
  ref_get_wake(hp, w, pos, alpha);
  for (size_t i = 0; i < W->_numParticles; ++i) {
    radius[i] = gsl_vector_get(W->_radius, i);
    volume[i] = gsl_vector_get(W->_volume, i);
  }
}

double ref_wtime(void) { return omp_get_wtime(); }

}  // extern "C"
