// Drop-in GPU backend for PAWAN's C++ class surface (see pawan_gpu_dropin.h).
#include "pawan_gpu_dropin.h"

#include <string.h>

#include <exception>
#include <stdexcept>
#include <string>
#include <thread>

namespace pawan {

__gpu::__gpu(__wake *W, const pgpu_config &cfg) : __interaction(), _cfg(cfg) {
  _nu = cfg.nu;  // the base constructor hard-codes 1.56e-5 (interaction.cpp:15)
  _cfg.kernel = pawan_kernel();
  check(pgpu_create(&_ctx, &_cfg));
  addWake(W);
}

__gpu::__gpu(__wake *W1, __wake *W2, const pgpu_config &cfg) : __interaction(), _cfg(cfg) {
  _nu = cfg.nu;
  _cfg.kernel = pawan_kernel();
  check(pgpu_create(&_ctx, &_cfg));
  addWake(W1);
  addWake(W2);
}

__gpu::~__gpu() {
  if (_ctx) pgpu_destroy(_ctx);
}

void __gpu::check(int rc) const {
  if (rc != PGPU_OK) {
    std::string msg = "pawan_gpu: ";
    msg += pgpu_last_error(_ctx);  // with no context yet: why pgpu_create failed
    throw std::runtime_error(msg + " (status " + std::to_string(rc) + ")");
  }
}

// __interaction keeps its wake list private (interaction.h:125-126): record
// the wake here as well, after the base class has updated _totalmaxsize.
void __gpu::addWake(__wake *W) {
  if (_laid_out) throw std::logic_error("pawan_gpu: wakes must be added before the first solve");
  __interaction::addWake(W);
  _wakes.push_back(W);
}

// Device slots: every wake but the last holds exactly its current particles
// (the wakes of one system are contiguous on the device); the last wake gets
// PAWAN's capacity so it can grow.
void __gpu::layout() {
  if (_laid_out) return;
  for (size_t k = 0; k < _wakes.size(); ++k) {
    const bool last = k + 1 == _wakes.size();
    const int64_t cap = last ? (int64_t)_wakes[k]->_maxnumParticles : (int64_t)_wakes[k]->_numParticles;
    int32_t id = -1;
    check(pgpu_add_wake(_ctx, 0, cap, &id));
    _ids.push_back(id);
  }
  _laid_out = true;
}

void __gpu::upload() {
  layout();
  for (size_t k = 0; k < _wakes.size(); ++k) {
    __wake *W = _wakes[k];
    check(pgpu_set_particles(_ctx, _ids[k], (int64_t)W->_numParticles, W->_position->data, W->_vorticity->data,
                             W->_radius->data, W->_volume->data));
  }
}

void __gpu::download_state() {
  for (size_t k = 0; k < _wakes.size(); ++k)
    check(pgpu_get_state(_ctx, _ids[k], _wakes[k]->_position->data, _wakes[k]->_vorticity->data));
}

// __interaction::solve (interaction.cpp:54-57): rates of every wake from all
// wakes, written to __wake::_velocity and _retvorcity (zeroed first, as
// interact() does at interaction.cpp:198-201).
void __gpu::solve() {
  upload();
  check(pgpu_solve(_ctx));
  for (size_t k = 0; k < _wakes.size(); ++k) {
    gsl_matrix_set_zero(_wakes[k]->_velocity);
    gsl_matrix_set_zero(_wakes[k]->_retvorcity);
    check(pgpu_get_rates(_ctx, _ids[k], _wakes[k]->_velocity->data, _wakes[k]->_retvorcity->data));
  }
}

// __interaction::diagnose (interaction.cpp:64-194): fills the same members
// writediagnosis() emits.
void __gpu::diagnose() {
  upload();
  diagnose_on_device();
}

void __gpu::diagnose_on_device() {
  double out[15], vbi[3];
  check(pgpu_diagnose(_ctx, 0, out, vbi));
  for (int k = 0; k < 3; ++k) {
    gsl_vector_set(_totalVorticity, k, out[k]);
    gsl_vector_set(_linearImpulse, k, out[3 + k]);
    gsl_vector_set(_angularImpulse, k, out[6 + k]);
  }
  _helicity = out[9];
  _enstrophy = out[10];
  _enstrophyF = out[11];
  _kineticEnergy = out[12];
  _kineticEnergyF = out[13];
  _Zc = out[14];
}

void __gpu::relax(size_t &stepnum) {
  for (__wake *W : _wakes) W->split(stepnum);
  upload();  // split may have appended particles
  for (size_t k = 0; k < _wakes.size(); ++k) {
    __wake *W = _wakes[k];
    // PAWAN's merge loop visits particles while they pass its age test (wake.cpp:115)
    int64_t n_elig = 0;
    while ((size_t)n_elig < W->_numParticles && stepnum - gsl_vector_get(W->_active, n_elig) > 45) ++n_elig;
    int64_t merged = 0;
    check(pgpu_merge(_ctx, _ids[k], n_elig, &merged));
    if (merged)
      check(pgpu_get_particles(_ctx, _ids[k], W->_position->data, W->_vorticity->data, nullptr, W->_volume->data));
  }
}

// __interaction::influence (interaction.cpp:212-260): zeroes every wake's
// _vorticityfield and fills it with the field from all wakes (the particle
// itself included, as SELFINFLUENCE adds it).
void __gpu::influence() {
  upload();
  check(pgpu_influence(_ctx));
  for (size_t k = 0; k < _wakes.size(); ++k) {
    gsl_matrix_set_zero(_wakes[k]->_vorticityfield);
    check(pgpu_get_vorticity_field(_ctx, _ids[k], _wakes[k]->_vorticityfield->data));
  }
}

void __gpu::device_step(int scheme, double dt, int nsteps) {
  upload();
  check(pgpu_step(_ctx, scheme, dt, nsteps));
  check(pgpu_sync(_ctx));
  download_state();
}

void __gpu::write_snapshot(FILE *f, double t, int slot) {
  const double *state = nullptr;
  std::vector<int64_t> off(_wakes.size()), n(_wakes.size());
  check(pgpu_snapshot_wait(_ctx, slot, 0.0, &state, off.data(), n.data(), (int32_t)_wakes.size()));
  for (size_t k = 0; k < _wakes.size(); ++k) {
    __wake *W = _wakes[k];
    const int32_t id = _ids[k];
    if ((size_t)n[id] != W->_numParticles) throw std::logic_error("pawan_gpu: wake size changed during integrate");
    memcpy(W->_position->data, state + 6 * off[id], 3 * (size_t)n[id] * sizeof(double));
    memcpy(W->_vorticity->data, state + 6 * off[id] + 3 * n[id], 3 * (size_t)n[id] * sizeof(double));
  }
  fwrite(&t, sizeof(double), 1, f);
  write(f);  // __interaction::write (interaction.cpp:304-319)
}

// Per step: the device step, then (once the previous record is written, which
// frees the slot used two steps ago) a snapshot into slot i % 2 handed to a
// writer thread, then the diagnostics on the device.  The writer of step i
// writes while step i + 1 computes.
void __gpu::integrate_on_device(int scheme, double dt, size_t nsteps, __io *IO, bool diag) {
  FILE *f = IO->create_binary_file(".wake");
  FILE *fdiag = IO->create_binary_file(".diagnosis");
  if (!f || !fdiag) {
    if (f) fclose(f);
    if (fdiag) fclose(fdiag);
    throw std::runtime_error("pawan_gpu: cannot create the .wake / .diagnosis files");
  }
  std::thread writer;
  std::exception_ptr werr;
  auto join = [&] {
    if (writer.joinable()) writer.join();
    if (werr) {
      std::exception_ptr e = werr;
      werr = nullptr;
      std::rethrow_exception(e);
    }
  };
  try {
    double t = 0.0;
    fwrite(&t, sizeof(double), 1, f);
    write(f);  // the initial particles as they are
    if (diag) {
      writenu(fdiag);
      fwrite(&t, sizeof(double), 1, fdiag);
      diagnose();  // uploads the host wakes
      writediagnosis(fdiag);
    } else {
      upload();
    }
    const double tStart = TIME();
    for (size_t i = 1; i <= nsteps; ++i) {
      OUT("\tStep", i);
      t = i * dt;
      check(pgpu_step(_ctx, scheme, dt, 1));
      join();
      const int slot = (int)(i & 1);
      check(pgpu_snapshot_begin(_ctx, slot));
      writer = std::thread([this, f, t, slot, &werr] {
        try {
          write_snapshot(f, t, slot);
        } catch (...) {
          werr = std::current_exception();
        }
      });
      if (diag) {
        diagnose_on_device();
        fwrite(&t, sizeof(double), 1, fdiag);
        writediagnosis(fdiag);
      }
    }
    join();
    check(pgpu_sync(_ctx));
    OUT("Total Time (s)", TIME() - tStart);
  } catch (...) {
    if (writer.joinable()) writer.join();
    fclose(f);
    fclose(fdiag);
    throw;
  }
  fclose(f);
  fclose(fdiag);
}

void __gpu::probe(const double *pts, long npts, double *vel) {
  upload();
  check(pgpu_probe(_ctx, 0, (int64_t)npts, pts, vel));
}

static __gpu *gpu_system(__system *S) {
  __gpu *G = dynamic_cast<__gpu *>(S);
  if (!G) throw std::invalid_argument("pawan_gpu: a GPU integrator needs a pawan::__gpu system");
  return G;
}

// __rk4::step / __rk3::step (rk4.cpp:12-77, rk3.cpp:12-65): the stage loop
// runs on the device.  On return `state` and the wakes hold the new state, as
// after PAWAN's own step.
static void gpu_step(int scheme, const double &dt, __system *S, gsl_vector *state) {
  __gpu *G = gpu_system(S);
  S->setStates(state);
  G->device_step(scheme, dt, 1);
  S->getStates(state);
}

void __rk4gpu::step(const double &dt, __system *S, gsl_vector *state) { gpu_step(PGPU_RK4, dt, S, state); }
void __rk3gpu::step(const double &dt, __system *S, gsl_vector *state) { gpu_step(PGPU_RK3, dt, S, state); }

void __rk4gpu::integrate(__system *S, __io *IO, bool diagnose) {
  gpu_system(S)->integrate_on_device(PGPU_RK4, _dt, _n, IO, diagnose);
}
void __rk3gpu::integrate(__system *S, __io *IO, bool diagnose) {
  gpu_system(S)->integrate_on_device(PGPU_RK3, _dt, _n, IO, diagnose);
}

}  // namespace pawan
