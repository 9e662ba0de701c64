/*
 * FP64 CPU restatement of PAWAN's vortex-particle hot path (see restate.h).
 * TEST INFRASTRUCTURE ONLY.
 *
 * Each function cites the PAWAN code it restates.  Differences in structure:
 * PAWAN visits every unordered pair once and applies it to both ends
 * (src/interaction/parallel.cpp:14-49); here every target sums over all
 * sources (ordered pairs), which is the same sum in a different order, with no
 * per-pair heap allocation, parallel over targets with OpenMP.
 */
#include "restate.h"

#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* Kernel of the whole restatement (rs_set_kernel): 0 Gaussian, 1 high-order
 * algebraic.  PAWAN fixes it at compile time (interaction_utils.h:13-20). */
static int g_kernel = 0;

void rs_set_kernel(int kernel) { g_kernel = kernel == 1 ? 1 : 0; }

/* ZETASIG: Gaussian (gaussian.h:20-23) exp(-rb^2/2) / (sigma^3 (2 pi)^(3/2));
 * high-order (highorder.h:20-24) 15 / (8 pi sigma^3 (rb^2 + 1)^(7/2)). */
static inline double zeta_sig(double rho, double sigma) {
  const double rb = rho / sigma;
  const double s3 = sigma * sigma * sigma;
  if (g_kernel == 1) return 1.875 / M_PI / pow(rb * rb + 1.0, 3.5) / s3;
  return exp(-0.5 * rb * rb) / s3 / pow(2.0 * M_PI, 1.5);
}

/* KERNEL, rb = rho/sigma.  Gaussian (gaussian.h:47-60):
 *   phi  = erf(rb / sqrt 2) / (4 pi sigma^3)
 *   q    = (phi/rb - zeta) / rb^2,  eta = zeta.
 * High-order (highorder.h:31-61):
 *   q    = rb^3 (rb^2 + 5/2) / (4 pi (rb^2 + 1)^(5/2) rho^3)
 *   eta  = 105 / (8 pi sigma^3 (rb^2 + 1)^(9/2)).
 * Both: F = (zeta - 3 q) / rho^2; eta is the diffusion kernel. */
static inline void kernel_terms(double rho, double sigma, double *q, double *F, double *Z, double *eta) {
  const double rb = rho / sigma;
  const double s3 = sigma * sigma * sigma;
  const double z = zeta_sig(rho, sigma);
  double qq, n;
  if (g_kernel == 1) {
    const double w = rb * rb + 1.0;
    qq = 0.25 / M_PI * rb * rb * rb * (rb * rb + 2.5) / pow(w, 2.5) / (rho * rho * rho);
    n = 13.125 / M_PI / pow(w, 4.5) / s3;
  } else {
    const double phi = 0.25 / M_PI * erf(rb / sqrt(2.0)) / s3;
    qq = (phi / rb - z) / (rb * rb);
    n = z;
  }
  *q = qq;
  *Z = z;
  *eta = n;
  *F = (z - 3.0 * qq) / (rho * rho);
}

/* Enstrophy pair factors ENST / ENSTF (highorder.h:71-95; zero for the
 * Gaussian kernel, gaussian.h:69-81), s2 = sigma^2, R = rho^2 + s2:
 *   F1  = (2 rho^4 + 7 s2 rho^2 + 20 s2^2) / (8 pi R^(7/2))
 *   F2  = -(6 rho^4 + 27 s2 rho^2 + 21 s2^2) / (8 pi R^(9/2))
 *   F1F = 15 s2^2 / (8 pi R^(7/2)) */
static inline void enst_terms(double r2, double s2, double *F1, double *F2, double *F1F) {
  if (g_kernel != 1) { *F1 = *F2 = *F1F = 0.0; return; }
  const double R = r2 + s2;
  const double f = 0.125 / M_PI / sqrt(pow(R, 7.0));
  *F1 = f * (2.0 * r2 * r2 + 7.0 * s2 * r2 + 20.0 * s2 * s2);
  *F2 = f * (-6.0 * r2 * r2 - 27.0 * s2 * r2 - 21.0 * s2 * s2) / R;
  *F1F = f * 15.0 * s2 * s2;
}

static inline void cross3(const double *a, const double *b, double *c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

/* One target t summed over all sources s != t.  Per ordered pair (target t,
 * source s), with d = x_t - x_s and sigma_ts = sqrt((s_s^2 + s_t^2)/2)
 * (interaction_utils.h:547):
 *   velocity   u_t  += q (alpha_s x d)                 (VELOCITY :55-62)
 *   stretching da_t += q (a_t x a_s) + F [d.(a_t x a_s)] d   (VORSTRETCH :73-105)
 *   diffusion  da_t += nu eta / (sigma^2/2) (vol_t a_s - vol_s a_t)  (DIFFUSION :344-378)
 * The source side of PAWAN's symmetric update (-q(a_t x d), -da) is the same
 * expression with the roles swapped (INTERACT :523-576). */
static void rates_one(int64_t t, int64_t n, const double *pos, const double *alpha,
                      const double *sigma, const double *vol, double nu, double *v, double *da) {
  const double *xt = pos + 3 * t, *at = alpha + 3 * t;
  const double st = sigma[t], vt = vol[t];
  double u0 = 0, u1 = 0, u2 = 0, d0 = 0, d1 = 0, d2 = 0;
  for (int64_t s = 0; s < n; ++s) {
    if (s == t) continue;
    const double *xs = pos + 3 * s, *as = alpha + 3 * s;
    const double d[3] = {xt[0] - xs[0], xt[1] - xs[1], xt[2] - xs[2]};
    const double rho = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    const double sg = sqrt(0.5 * (sigma[s] * sigma[s] + st * st));
    double q, F, Z, eta;
    kernel_terms(rho, sg, &q, &F, &Z, &eta);
    double w[3];
    cross3(as, d, w);
    u0 += q * w[0]; u1 += q * w[1]; u2 += q * w[2];
    double c[3];
    cross3(at, as, c);
    const double dc = d[0] * c[0] + d[1] * c[1] + d[2] * c[2];
    const double k = nu * eta / (0.5 * sg * sg);
    const double vs = vol[s];
    d0 += q * c[0] + F * dc * d[0] + k * (vt * as[0] - vs * at[0]);
    d1 += q * c[1] + F * dc * d[1] + k * (vt * as[1] - vs * at[1]);
    d2 += q * c[2] + F * dc * d[2] + k * (vt * as[2] - vs * at[2]);
  }
  v[0] = u0; v[1] = u1; v[2] = u2;
  da[0] = d0; da[1] = d1; da[2] = d2;
}

void rs_rates(int64_t n, const double *pos, const double *alpha, const double *sigma,
              const double *vol, double nu, const int64_t *targets, int64_t nt,
              double *vel, double *dalpha) {
  if (!targets) nt = n;
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t i = 0; i < nt; ++i) {
    const int64_t t = targets ? targets[i] : i;
    rates_one(t, n, pos, alpha, sigma, vol, nu, vel + 3 * i, dalpha + 3 * i);
  }
}

/* Time stepping on the packed state [x ; alpha] (the flat FP64 vector of
 * __wake::getStates, wake.cpp:882-893).
 *   Euler (integration.cpp:198-208): x += dt k1
 *   RK3   (rk3.cpp:12-65, Kutta):  x1 = x + dt/2 k1, x2 = x - dt k1 + 2 dt k2,
 *                                  x += dt/6 k1 + 2dt/3 k2 + dt/6 k3
 *   RK4   (rk4.cpp:12-77):         x1 = x + dt/2 k1, x2 = x + dt/2 k2,
 *                                  x3 = x + dt k3,
 *                                  x += dt/6 (k1 + k4) + dt/3 (k2 + k3) */
static void eval(int64_t n, const double *st, const double *sigma, const double *vol, double nu,
                 double *k) {
  rs_rates(n, st, st + 3 * n, sigma, vol, nu, NULL, n, k, k + 3 * n);
}

void rs_step(int scheme, double dt, int nsteps, int64_t n, double *pos, double *alpha,
             const double *sigma, const double *vol, double nu) {
  const int64_t m = 6 * n;
  double *x = (double *)malloc(sizeof(double) * m);
  double *y = (double *)malloc(sizeof(double) * m);
  double *k1 = (double *)malloc(sizeof(double) * m);
  double *k2 = (double *)malloc(sizeof(double) * m);
  double *k3 = (double *)malloc(sizeof(double) * m);
  double *k4 = (double *)malloc(sizeof(double) * m);
  memcpy(x, pos, sizeof(double) * 3 * n);
  memcpy(x + 3 * n, alpha, sizeof(double) * 3 * n);
  for (int it = 0; it < nsteps; ++it) {
    eval(n, x, sigma, vol, nu, k1);
    if (scheme == 0) {
      for (int64_t i = 0; i < m; ++i) x[i] += dt * k1[i];
    } else if (scheme == 1) {
      for (int64_t i = 0; i < m; ++i) y[i] = x[i] + 0.5 * dt * k1[i];
      eval(n, y, sigma, vol, nu, k2);
      for (int64_t i = 0; i < m; ++i) y[i] = (x[i] + 2.0 * dt * k2[i]) - dt * k1[i];
      eval(n, y, sigma, vol, nu, k3);
      for (int64_t i = 0; i < m; ++i)
        x[i] += (dt * k1[i] / 6.0 + dt / 6.0 * k3[i]) + dt * 2.0 / 3.0 * k2[i];
    } else {
      for (int64_t i = 0; i < m; ++i) y[i] = x[i] + 0.5 * dt * k1[i];
      eval(n, y, sigma, vol, nu, k2);
      for (int64_t i = 0; i < m; ++i) y[i] = x[i] + 0.5 * dt * k2[i];
      eval(n, y, sigma, vol, nu, k3);
      for (int64_t i = 0; i < m; ++i) y[i] = x[i] + dt * k3[i];
      eval(n, y, sigma, vol, nu, k4);
      for (int64_t i = 0; i < m; ++i)
        x[i] += (k1[i] + k4[i]) * (dt / 6.0) + (k2[i] + k3[i]) * (dt / 3.0);
    }
  }
  memcpy(pos, x, sizeof(double) * 3 * n);
  memcpy(alpha, x + 3 * n, sizeof(double) * 3 * n);
  free(x); free(y); free(k1); free(k2); free(k3); free(k4);
}

/* Diagnostics, src/interaction/interaction.cpp:64-194 with the OpenMP bodies
 * of parallel.cpp:140-401 and the pair terms of interaction_utils.h:214-331:
 *   total vorticity  sum alpha
 *   linear impulse   1/2 sum x x alpha
 *   angular impulse  1/3 sum x x (x x alpha)
 *   helicity         sum_{i != j} q(rho, s_ij) (x_j - x_i).(a_i x a_j)
 *   enstrophy        sum_i ENST(s_i) |a_i|^2
 *                    + sum_{i != j} [F1 (a_i.a_j) + F2 (a_i.d)(a_j.d)]   (ENSTROPHY :107-176)
 *   enstrophyF       sum_i ENSTF(s_i) |a_i|^2 + sum_{i != j} F1F (a_i.a_j)  (:122-201)
 *                    with ENST(s) = 5/(2 pi s^3), ENSTF(s) = 15/(8 pi s^3)
 *                    (highorder.h:101-110); both 0 for the Gaussian kernel
 *                    (gaussian.h:69-92)
 *   KE   = sum_i |a_i|^2/(8 pi s_i)
 *        + sum_{i != j} [(rho^2 + 2 s^2)(a_i.a_j) + (d.a_i)(d.a_j)] / (16 pi (rho^2 + s^2)^(3/2))
 *   KEF  = sum_i 3|a_i|^2/(16 pi s_i)
 *        + sum_{i != j} (rho^2 + 1.5 s^2)(a_i.a_j) / (8 pi (rho^2 + s^2)^(3/2))
 * with s^2 = (s_i^2 + s_j^2)/2.  Zc (interaction.cpp:135-157) takes the last
 * wake with a non-zero weight; vbi is getVi at the origin (:184-193). */
void rs_diagnose(int nw, const int64_t *offsets, const double *pos, const double *alpha,
                 const double *sigma, double zc_prev, double *out, double *vbi) {
  const int64_t n = offsets[nw];
  double O[3] = {0, 0, 0}, I[3] = {0, 0, 0}, A[3] = {0, 0, 0};
  for (int64_t i = 0; i < n; ++i) {
    const double *x = pos + 3 * i, *a = alpha + 3 * i;
    double xa[3], xxa[3];
    cross3(x, a, xa);
    cross3(x, xa, xxa);
    for (int k = 0; k < 3; ++k) { O[k] += a[k]; I[k] += xa[k]; A[k] += xxa[k]; }
  }
  double H = 0, KE = 0, KEF = 0, EN = 0, ENF = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : H, KE, KEF, EN, ENF)
  for (int64_t i = 0; i < n; ++i) {
    const double *xi = pos + 3 * i, *ai = alpha + 3 * i;
    const double si = sigma[i];
    const double a2 = ai[0] * ai[0] + ai[1] * ai[1] + ai[2] * ai[2];
    double h = 0, ke = a2 / si / 8.0 / M_PI, kef = 3.0 * a2 / (si * 16.0) / M_PI;
    double en = 0, enf = 0;
    if (g_kernel == 1) {
      en = 5.0 / M_PI / 2.0 / (si * si * si) * a2;
      enf = 15.0 / M_PI / 8.0 / (si * si * si) * a2;
    }
    for (int64_t j = 0; j < n; ++j) {
      if (j == i) continue;
      const double *xj = pos + 3 * j, *aj = alpha + 3 * j;
      const double d[3] = {xj[0] - xi[0], xj[1] - xi[1], xj[2] - xi[2]};
      const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      const double s2 = 0.5 * (si * si + sigma[j] * sigma[j]);
      double q, F, Z, eta;
      kernel_terms(sqrt(r2), sqrt(s2), &q, &F, &Z, &eta);
      double c[3];
      cross3(ai, aj, c);
      h += q * (d[0] * c[0] + d[1] * c[1] + d[2] * c[2]);
      const double aa = ai[0] * aj[0] + ai[1] * aj[1] + ai[2] * aj[2];
      const double dai = d[0] * ai[0] + d[1] * ai[1] + d[2] * ai[2];
      const double daj = d[0] * aj[0] + d[1] * aj[1] + d[2] * aj[2];
      const double den = pow(r2 + s2, 1.5);
      ke += ((r2 + 2.0 * s2) * aa + dai * daj) / den / 16.0 / M_PI;
      kef += (r2 + 1.5 * s2) * aa / den / 8.0 / M_PI;
      double F1, F2, F1F;
      enst_terms(r2, s2, &F1, &F2, &F1F);
      en += F1 * aa + F2 * dai * daj;
      enf += F1F * aa;
    }
    H += h; KE += ke; KEF += kef; EN += en; ENF += enf;
  }
  double zc = zc_prev;
  for (int w = 0; w < nw; ++w) {
    double num = 0, den = 0;
    for (int64_t i = offsets[w]; i < offsets[w + 1]; ++i) {
      const double *x = pos + 3 * i, *a = alpha + 3 * i;
      const double om = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
      const double rr = x[0] * x[0] + x[1] * x[1];
      num += om * x[2] * rr;
      den += om * rr;
    }
    if (den != 0.0) zc = num / den;
  }
  for (int k = 0; k < 3; ++k) { out[k] = O[k]; out[3 + k] = 0.5 * I[k]; out[6 + k] = A[k] / 3.0; }
  out[9] = H; out[10] = EN; out[11] = ENF; out[12] = KE; out[13] = KEF; out[14] = zc;
  const double origin[3] = {0, 0, 0};
  rs_getvi(n, pos, alpha, sigma, origin, vbi);
}

/* __interaction::getVi (interaction.cpp:453-477): d = r - x_i, the particle's
 * own radius, u += q (alpha_i x d). */
void rs_getvi(int64_t n, const double *pos, const double *alpha, const double *sigma,
              const double *r, double *out) {
  double u[3] = {0, 0, 0};
  for (int64_t i = 0; i < n; ++i) {
    const double d[3] = {r[0] - pos[3 * i], r[1] - pos[3 * i + 1], r[2] - pos[3 * i + 2]};
    const double rho = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    double q, F, Z, eta, w[3];
    kernel_terms(rho, sigma[i], &q, &F, &Z, &eta);
    cross3(alpha + 3 * i, d, w);
    for (int k = 0; k < 3; ++k) u[k] += q * w[k];
  }
  for (int k = 0; k < 3; ++k) out[k] = u[k];
}

/* The sums behind rs_diagnose restricted to the rows [row_lo, row_hi) of the
 * concatenated wakes, per wake, in the field layout of the C ABI's
 * pgpu_diagnose_partial (23 doubles per wake): 0-2 sum alpha, 3-5 sum
 * x x alpha, 6-8 sum x x (x x alpha), 9-10 Zc numerator and denominator,
 * 11-13 velocity at the origin (getVi, interaction.cpp:453-477), 14 helicity,
 * 15-16 KE and KEF pair terms, 17-18 their self terms, 19-20 enstrophy pair
 * terms, 21-22 their self terms.  Pair terms of a row i run over every j != i
 * of the system (ordered pairs, as rs_diagnose), so fields summed over a
 * partition of the rows give rs_diagnose's totals.  Test code for the
 * sharded diagnostics. */
void rs_diagnose_fields(int nw, const int64_t *offsets, const double *pos, const double *alpha,
                        const double *sigma, int64_t row_lo, int64_t row_hi, double *fields) {
  const int64_t n = offsets[nw];
  for (int w = 0; w < nw; ++w) {
    double *f = fields + 23 * w;
    for (int m = 0; m < 23; ++m) f[m] = 0.0;
    const int64_t lo = offsets[w] > row_lo ? offsets[w] : row_lo;
    const int64_t hi = offsets[w + 1] < row_hi ? offsets[w + 1] : row_hi;
    for (int64_t i = lo; i < hi; ++i) {
      const double *x = pos + 3 * i, *a = alpha + 3 * i;
      double xa[3], xxa[3];
      cross3(x, a, xa);
      cross3(x, xa, xxa);
      for (int k = 0; k < 3; ++k) { f[k] += a[k]; f[3 + k] += xa[k]; f[6 + k] += xxa[k]; }
      const double om = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
      const double rr = x[0] * x[0] + x[1] * x[1];
      f[9] += om * x[2] * rr;
      f[10] += om * rr;
      const double d0[3] = {-x[0], -x[1], -x[2]};
      double q0, F0, Z0, eta0, w0[3];
      kernel_terms(sqrt(rr + x[2] * x[2]), sigma[i], &q0, &F0, &Z0, &eta0);
      cross3(a, d0, w0);
      for (int k = 0; k < 3; ++k) f[11 + k] += q0 * w0[k];
      const double si = sigma[i];
      const double a2 = a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
      f[17] += a2 / si / 8.0 / M_PI;
      f[18] += 3.0 * a2 / (si * 16.0) / M_PI;
      if (g_kernel == 1) {
        f[21] += 5.0 / M_PI / 2.0 / (si * si * si) * a2;
        f[22] += 15.0 / M_PI / 8.0 / (si * si * si) * a2;
      }
      double h = 0, ke = 0, kef = 0, en = 0, enf = 0;
#pragma omp parallel for reduction(+ : h, ke, kef, en, enf)
      for (int64_t j = 0; j < n; ++j) {
        if (j == i) continue;
        const double *xj = pos + 3 * j, *aj = alpha + 3 * j;
        const double d[3] = {xj[0] - x[0], xj[1] - x[1], xj[2] - x[2]};
        const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
        const double s2 = 0.5 * (si * si + sigma[j] * sigma[j]);
        double q, F, Z, eta, c[3];
        kernel_terms(sqrt(r2), sqrt(s2), &q, &F, &Z, &eta);
        cross3(a, aj, c);
        h += q * (d[0] * c[0] + d[1] * c[1] + d[2] * c[2]);
        const double aa = a[0] * aj[0] + a[1] * aj[1] + a[2] * aj[2];
        const double dai = d[0] * a[0] + d[1] * a[1] + d[2] * a[2];
        const double daj = d[0] * aj[0] + d[1] * aj[1] + d[2] * aj[2];
        const double den = pow(r2 + s2, 1.5);
        ke += ((r2 + 2.0 * s2) * aa + dai * daj) / den / 16.0 / M_PI;
        kef += (r2 + 1.5 * s2) * aa / den / 8.0 / M_PI;
        double F1, F2, F1F;
        enst_terms(r2, s2, &F1, &F2, &F1F);
        en += F1 * aa + F2 * dai * daj;
        enf += F1F * aa;
      }
      f[14] += h; f[15] += ke; f[16] += kef; f[19] += en; f[20] += enf;
    }
  }
}

/* Vorticity field of the listed targets (all if NULL), PAWAN's influence()
 * (interaction.cpp:212-260; INFLUENCE / SELFINFLUENCE, interaction_utils.h:
 * 626-703): k_t = sum_s ZETASIG(rho_ts, sigma_ts) alpha_s over every particle
 * s, the target itself included (rho = 0, sigma_tt = sigma_t), with
 * sigma_ts = sqrt((sigma_t^2 + sigma_s^2) / 2) and ZETASIG of the selected
 * kernel (zeta_sig above). */
void rs_vorticity_field(int64_t n, const double *pos, const double *alpha, const double *sigma,
                        const int64_t *targets, int64_t nt, double *field) {
  if (!targets) nt = n;
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t i = 0; i < nt; ++i) {
    const int64_t t = targets ? targets[i] : i;
    double k[3] = {0.0, 0.0, 0.0};
    for (int64_t s = 0; s < n; ++s) {
      const double dx = pos[3 * t] - pos[3 * s], dy = pos[3 * t + 1] - pos[3 * s + 1], dz = pos[3 * t + 2] - pos[3 * s + 2];
      const double rho = sqrt(dx * dx + dy * dy + dz * dz);
      const double sg = sqrt(0.5 * (sigma[t] * sigma[t] + sigma[s] * sigma[s]));
      const double z = zeta_sig(rho, sg);
      for (int m = 0; m < 3; ++m) k[m] += z * alpha[3 * s + m];
    }
    for (int m = 0; m < 3; ++m) field[3 * i + m] = k[m];
  }
}

/* Particle merge, __wake::merge (wake.cpp:112-159), sequential as PAWAN's
 * loop: for i < n_elig (the age-eligible prefix) and j = i+1 .. n-1 in order,
 * j merges into i when |x_i - x_j| < 0.125 (r_i + r_j), |a_j| != 0,
 * |a_i| != 0 (|a_i| taken at the start of i's turn) and
 * 1 - a_i.a_j / |a_i| / |a_j| >= 1e-4; then
 * x_i = (x_i |a_i| + x_j |a_j|) (1 / (|a_i| + |a_j|)), a_i += a_j, a_j = 0,
 * vol_j = 0.  Norms by the scaled sum of squares of gsl_blas_dnrm2.
 * Instead of PAWAN's O(n^2) j loop, the js are found in a uniform grid of
 * the positions at entry (cell = 0.25 r_max): only x_i moves during i's turn,
 * and a j > i has not moved yet.  Each time x_i moves, the js after the last
 * merged one are gathered again around the new x_i (within
 * 0.125 (r_i + r_max)) and visited in increasing order, so every merge PAWAN
 * makes is found in PAWAN's order.  Returns the number of merges; pos, alpha,
 * vol are updated in place. */
static double nrm2_3(double a, double b, double c) {
  const double v[3] = {a, b, c};
  double scale = 0.0, ssq = 1.0;
  for (int k = 0; k < 3; ++k) {
    if (v[k] != 0.0) {
      const double ax = fabs(v[k]);
      if (scale < ax) { ssq = 1.0 + ssq * (scale / ax) * (scale / ax); scale = ax; }
      else ssq += (ax / scale) * (ax / scale);
    }
  }
  return scale * sqrt(ssq);
}

static int cmp_i64(const void *a, const void *b) {
  const int64_t x = *(const int64_t *)a, y = *(const int64_t *)b;
  return x < y ? -1 : x > y;
}

typedef struct { int64_t key, idx; } cell_ent;
static int cmp_cell(const void *a, const void *b) {
  const cell_ent *x = (const cell_ent *)a, *y = (const cell_ent *)b;
  if (x->key != y->key) return x->key < y->key ? -1 : 1;
  return x->idx < y->idx ? -1 : x->idx > y->idx;
}

static int64_t cell_key(int64_t cx, int64_t cy, int64_t cz) {
  return ((cx & 0x1fffff) << 42) | ((cy & 0x1fffff) << 21) | (cz & 0x1fffff);
}

int64_t rs_merge(int64_t n, int64_t n_elig, double *pos, double *alpha, const double *sigma, double *vol) {
  if (n_elig > n) n_elig = n;
  if (n < 2 || n_elig <= 0) return 0;
  double rmax = 0.0;
  for (int64_t i = 0; i < n; ++i) rmax = sigma[i] > rmax ? sigma[i] : rmax;
  const double h = rmax > 0.0 ? 0.25 * rmax : 1.0;
  cell_ent *ent = (cell_ent *)malloc(sizeof(cell_ent) * n);
  for (int64_t i = 0; i < n; ++i) {
    ent[i].key = cell_key((int64_t)floor(pos[3 * i] / h), (int64_t)floor(pos[3 * i + 1] / h),
                          (int64_t)floor(pos[3 * i + 2] / h));
    ent[i].idx = i;
  }
  qsort(ent, n, sizeof(cell_ent), cmp_cell);
  int64_t *js = (int64_t *)malloc(sizeof(int64_t) * n);
  int64_t merges = 0;
  for (int64_t i = 0; i < n_elig; ++i) {
    double *xi = pos + 3 * i, *ai = alpha + 3 * i;
    const double ivormag = nrm2_3(ai[0], ai[1], ai[2]);
    if (ivormag == 0.0) continue;
    const double ri = sigma[i];
    int64_t after = i;  /* js > after are still to be visited */
    for (;;) {
      /* gather the js > after within 0.125 (r_i + r_max) of the current x_i */
      const double reach = 0.125 * (ri + rmax);
      const int64_t c0[3] = {(int64_t)floor((xi[0] - reach) / h), (int64_t)floor((xi[1] - reach) / h),
                             (int64_t)floor((xi[2] - reach) / h)};
      const int64_t c1[3] = {(int64_t)floor((xi[0] + reach) / h), (int64_t)floor((xi[1] + reach) / h),
                             (int64_t)floor((xi[2] + reach) / h)};
      int64_t nj = 0;
      for (int64_t cx = c0[0]; cx <= c1[0]; ++cx)
        for (int64_t cy = c0[1]; cy <= c1[1]; ++cy)
          for (int64_t cz = c0[2]; cz <= c1[2]; ++cz) {
            const int64_t key = cell_key(cx, cy, cz);
            int64_t lo = 0, hi = n; /* first entry with this key */
            while (lo < hi) {
              const int64_t mid = (lo + hi) / 2;
              if (ent[mid].key < key) lo = mid + 1; else hi = mid;
            }
            for (int64_t e = lo; e < n && ent[e].key == key; ++e)
              if (ent[e].idx > after) js[nj++] = ent[e].idx;
          }
      qsort(js, nj, sizeof(int64_t), cmp_i64);
      int moved = 0;
      for (int64_t t = 0; t < nj; ++t) {
        const int64_t j = js[t];
        double *xj = pos + 3 * j, *aj = alpha + 3 * j;
        const double jvormag = nrm2_3(aj[0], aj[1], aj[2]);
        const double rho = nrm2_3(xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]);
        if (!(rho < 0.125 * (ri + sigma[j]) && jvormag != 0.0)) continue;
        const double dot = ai[0] * aj[0] + ai[1] * aj[1] + ai[2] * aj[2];
        const double alignment = 1 - dot / ivormag / jvormag;
        if (!(alignment >= 0.0001)) continue;
        const double s = 1 / (ivormag + jvormag);
        for (int m = 0; m < 3; ++m) {
          double p = xi[m] * ivormag;
          p += xj[m] * jvormag;
          xi[m] = p * s;
          ai[m] += aj[m];
          aj[m] = 0.0;
        }
        vol[j] = 0.0;
        ++merges;
        after = j;
        moved = 1;
        break; /* x_i moved: gather again around it */
      }
      if (!moved) break;
    }
  }
  free(js);
  free(ent);
  return merges;
}

int rs_threads(void) { return omp_get_max_threads(); }
