/*
 * FP64 CPU restatement of PAWAN's vortex-particle hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the second-tier oracle (validated against PAWAN's
 * own compiled sources at small N) and the "port" CPU baseline.  The product
 * never links or calls it.
 *
 * Layout: positions / strengths row-major (n, 3) FP64, radii and volumes (n),
 * as PAWAN's __wake matrices (src/wake/wake.h:49-54).  All particles passed in
 * one call form one system: every particle interacts with every other, as the
 * wakes held by one __interaction do (src/interaction/interaction.cpp:196-210).
 */
#ifndef PAWAN_ORACLE_RESTATE_H_
#define PAWAN_ORACLE_RESTATE_H_
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Selects the regularisation kernel of every later call: 0 = Gaussian
 * (src/interaction/gaussian.h, the default), 1 = high-order algebraic
 * (src/interaction/highorder.h).  Process-wide; not for concurrent callers. */
void rs_set_kernel(int kernel);

/* Rates dx/dt (vel) and dalpha/dt (dalpha) of the targets listed in
 * `targets` (nt entries; NULL means all n particles in order) induced by all n
 * particles, self excluded.  Outputs are (nt, 3) row-major. */
void rs_rates(int64_t n, const double *pos, const double *alpha, const double *sigma,
              const double *vol, double nu, const int64_t *targets, int64_t nt,
              double *vel, double *dalpha);

/* nsteps time steps of size dt; scheme 0 = Euler, 1 = RK3 (Kutta), 2 = RK4.
 * Positions and strengths are advanced in place. */
void rs_step(int scheme, double dt, int nsteps, int64_t n, double *pos, double *alpha,
             const double *sigma, const double *vol, double nu);

/* Diagnostics of one system of nw wakes (wake w = particles
 * [offsets[w], offsets[w+1])).  out[0..14] = total vorticity(3), linear
 * impulse(3), angular impulse(3), helicity, enstrophy, enstrophyF, kinetic
 * energy, kinetic energyF, Zc; vbi[3] = velocity induced at the origin.
 * zc_prev is the Zc reported when no wake has a non-zero weight. */
void rs_diagnose(int nw, const int64_t *offsets, const double *pos, const double *alpha,
                 const double *sigma, double zc_prev, double *out, double *vbi);

/* Velocity induced at point r by all n particles using each particle's own
 * smoothing radius (PAWAN __interaction::getVi). */
void rs_getvi(int64_t n, const double *pos, const double *alpha, const double *sigma,
              const double *r, double *out);

/* Vorticity field k_t = sum_s zeta(rho_ts, sigma_ts) alpha_s of the listed
 * targets (all if NULL), the target itself included (PAWAN's influence()). */
void rs_vorticity_field(int64_t n, const double *pos, const double *alpha, const double *sigma,
                        const int64_t *targets, int64_t nt, double *field);
/* PAWAN's particle merge (__wake::merge, wake.cpp:112-159) over the first
 * n_elig particles (the age-eligible prefix of PAWAN's loop); pos, alpha and
 * vol are updated in place.  Returns the number of merges. */
int64_t rs_merge(int64_t n, int64_t n_elig, double *pos, double *alpha, const double *sigma, double *vol);
int rs_threads(void);

#ifdef __cplusplus
}
#endif
#endif
