/*
 * Drop-in GPU backend for PAWAN's C++ class surface.
 *
 * Compiled inside a PAWAN build (against PAWAN's own headers and GSL) and
 * linked with libpawan_gpu.so.  Selecting the GPU is then a one-line change
 * in a PAWAN driver (src/pawan.cpp:47-48):
 *
 *     pawan::__interaction *S = new pawan::__parallel(W);     // CPU, OpenMP
 *     pawan::__interaction *S = new pawan::__gpu(W, cfg);      // B200
 *     pawan::__integration *IN = new pawan::__rk4(T, n);       // CPU stages
 *     pawan::__integration *IN = new pawan::__rk4gpu(T, n);    // stages on the GPU
 *     IN->integrate(S, IO, true);                              // unchanged
 *
 * Declaring IN as a pawan::__rk4gpu * (or __rk3gpu *) instead keeps the state
 * on the device for the whole run and writes each step's .wake record from
 * an asynchronous download while the next step computes
 * (__gpu::integrate_on_device); the files are the same.
 *
 * __gpu overrides the virtual members of __interaction that carry the hot
 * path (interaction.h:192-244): solve, diagnose, addWake, relax, and the
 * protected influence behind resolve().  Particle data stays
 * authoritative in the host __wake matrices, exactly as in PAWAN; every solve
 * uploads the current positions/strengths and writes the rates back into
 * __wake::_velocity / _retvorcity, so getRates/getStates/setStates/write keep
 * PAWAN's own behaviour.  __rk4gpu / __rk3gpu override the protected step()
 * (integration.h:37, rk4.h:25, rk3.h:25): the whole step runs on the device
 * (one CUDA graph per step), and the state vector and the wakes are updated
 * afterwards, as PAWAN's step leaves them (rk4.cpp:66-68).
 *
 * Kernel: __gpu always uses the regularisation kernel this PAWAN build was
 * compiled with (pawan_kernel() below), whatever cfg.kernel says, so that it
 * computes what the __interaction it replaces would.
 *
 * Errors: a non-zero pgpu_* status becomes std::runtime_error carrying
 * pgpu_last_error().  A GPU integrator given a system that is not a __gpu
 * throws std::invalid_argument (there is no CPU fallback).
 */
#ifndef PAWAN_GPU_DROPIN_H_
#define PAWAN_GPU_DROPIN_H_

#include <stdio.h>

#include <vector>

#include "pawan_gpu.h"
#include "src/integration/rk3.h"
#include "src/integration/rk4.h"
#include "src/interaction/interaction.h"

namespace pawan {

// PGPU_KERNEL_* of the kernel compiled into this PAWAN build: HIGHORDER /
// GAUSSIAN (interaction_utils.h:13-20) make interaction.h include either
// highorder.h, which defines HIGHORDER_H_, or gaussian.h.
inline int pawan_kernel() {
#ifdef HIGHORDER_H_
  return PGPU_KERNEL_HIGHORDER;
#else
  return PGPU_KERNEL_GAUSSIAN;
#endif
}

class __gpu : public __interaction {
 public:
  __gpu(__wake *W, const pgpu_config &cfg);
  __gpu(__wake *W1, __wake *W2, const pgpu_config &cfg);
  ~__gpu();

  void addWake(__wake *W) override;
  void solve() override;
  void diagnose() override;
  // __interaction::relax (interaction.cpp:367-371), each wake's split then
  // merge (wake.cpp:161-165): PAWAN's own O(N) split on the host wake, then
  // the O(N^2) merge through pgpu_merge (candidates on the device, PAWAN's
  // sequential loop replayed on the host), written back to the host wake.
  void relax(size_t &stepnum) override;

  // Advances the wakes `nsteps` steps on the device (scheme PGPU_RK3 / PGPU_RK4
  // / PGPU_EULER) starting from the host wakes, then writes the new state back
  // into them.
  void device_step(int scheme, double dt, int nsteps);
  // __integration::integrate (integration.cpp:24-60) with the state kept on
  // the device from the first step to the last.  After each step an
  // asynchronous snapshot (pgpu_snapshot_begin, two slots in turn) brings the
  // state back while the next step runs, and a writer thread copies it into
  // the host wakes and writes the step's .wake record with PAWAN's own
  // __interaction::write; the diagnostics, when asked for, are computed on the
  // device after each step and written with PAWAN's writediagnosis.  The
  // .wake and .diagnosis files hold what PAWAN's loop writes, record for
  // record, and the host wakes end at the final state.
  void integrate_on_device(int scheme, double dt, size_t nsteps, __io *IO, bool diagnose);
  // Velocity induced at npts points (row-major) by all wakes, each particle
  // with its own radius (getVi, interaction.cpp:453-477).
  void probe(const double *pts, long npts, double *vel);
  pgpu_ctx *context() { return _ctx; }

 protected:
  // __interaction::influence (interaction.cpp:212-260), which resolve()
  // (interaction.cpp:59-62) calls, and so PAWAN's __resolve::rebuild
  // (resolve.cpp:12-63): the vorticity field of every particle from all
  // wakes, on the device, written to each wake's _vorticityfield.  (The
  // base's one- and two-wake overloads are private and not used here.)
  void influence() override;

 private:
  void check(int rc) const;
  void layout();  // creates the device wakes on first use
  void upload();
  void download_state();
  void diagnose_on_device();  // diagnose() without the upload of the host wakes
  // Waits for snapshot `slot`, copies it into the host wakes and writes the
  // .wake record of time t.
  void write_snapshot(FILE *f, double t, int slot);
  pgpu_config _cfg;
  pgpu_ctx *_ctx = nullptr;
  std::vector<__wake *> _wakes;
  std::vector<int32_t> _ids;
  bool _laid_out = false;
};

// integrate(S, IO, diagnose) called on a __rk4gpu / __rk3gpu (its static
// type) runs __gpu::integrate_on_device.  Called through a pointer or
// reference to __integration, PAWAN's own loop runs instead, with the GPU step
// below and a synchronous download after each step: the same files either way.
class __rk4gpu : public __rk4 {
 public:
  __rk4gpu(const double &t, const size_t &n) : __rk4(t, n) {}
  using __rk4::integrate;
  void integrate(__system *S, __io *IO, bool diagnose = false);
 protected:
  void step(const double &dt, __system *S, gsl_vector *state) override;
};

class __rk3gpu : public __rk3 {
 public:
  __rk3gpu(const double &t, const size_t &n) : __rk3(t, n) {}
  using __rk3::integrate;
  void integrate(__system *S, __io *IO, bool diagnose = false);
 protected:
  void step(const double &dt, __system *S, gsl_vector *state) override;
};

}  // namespace pawan
#endif
