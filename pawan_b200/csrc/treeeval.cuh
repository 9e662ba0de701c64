// Surrogate evaluation on the octree of tree.cuh, FP32 with compensated sums.
//
// Far cells.  Beyond a few cell widths the Gaussian regularisation is below
// FP32 resolution (tests/test_math_fits.py), so a far cell acts through the
// singular kernel, written with phi(d) = 1/|d| (4 pi units, as the pair kernel):
//   velocity    alpha_s x d / rho^3                     = -alpha_s x grad phi(d)
//   stretching  b/rho^3 - 3 (d.b) d / rho^5, b = alpha_t x alpha_s  = -D2(d) b
// Expanding d = r - y about the cell centroid (r = x_t - c, y = x_s - c) in
// powers of y, with A = sum alpha, M_ab = sum alpha_a y_b,
// Q_abc = sum alpha_a y_b y_c, T_abcd = sum alpha_a y_b y_c y_d and Dn the
// n-th derivative tensors of phi at r:
//   u_i = -eps_iab [A_a D1_b - M_ac D2_bc + 1/2 Q_acd D3_bcd - 1/6 T_acde D4_bcde]
//   s_i = -[D2_ik B_k - D3_ikc N_kc + 1/2 D4_ikcd P_kcd - 1/6 D5_ikcde R_kcde],
//         B = alpha_t x A, N_.c = alpha_t x M_.c, P_.cd = alpha_t x Q_.cd,
//         R_.cde = alpha_t x T_.cde.
// `order` 0 keeps the monopole, 1 adds the dipole, 2 the quadrupole, 3 the
// octupole.  The contractions below never form the derivative tensors; the
// order-3 contractions were checked in a CPU restatement against the full
// tensor contraction, and tests/test_surrogate.py checks the result end to
// end (the error falls with the order against the direct sum).
//
// Near leaves.  Exact pair sums with the same three-regime FP32 terms as the
// direct kernel.
#pragma once
#include "kernels.cuh"
#include "mlp.cuh"
#include "tree.cuh"

namespace pgpu {

__device__ __forceinline__ void cross3f(const float *a, const float *b, float *c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}

// Velocity u and stretching s (4 pi units) induced at a target (position x,
// strength at) by a far cell (data v), to the given order.
__device__ __forceinline__ void far_expand(const float *v, const float *x, const float *at, int order, float *u,
                                           float *s) {
  const float r[3] = {x[0] - v[0], x[1] - v[1], x[2] - v[2]};
  const float r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
  const float ir = fast_rsqrt(r2);
  const float ir2 = ir * ir, ir3 = ir * ir2, ir5 = ir3 * ir2, ir7 = ir5 * ir2, ir9 = ir7 * ir2;
  const float A[3] = {v[3], v[4], v[5]};
  float t[3];
  cross3f(A, r, t);
  for (int i = 0; i < 3; ++i) u[i] = ir3 * t[i];
  float B[3];
  cross3f(at, A, B);
  const float rB = r[0] * B[0] + r[1] * B[1] + r[2] * B[2];
  for (int i = 0; i < 3; ++i) s[i] = ir3 * B[i] - 3.f * ir5 * rB * r[i];
  if (order < 1) return;
  // ---- dipole
  const float *M = v + 6;  // M[a*3+b]
  float Mr[3];
  for (int a = 0; a < 3; ++a) Mr[a] = M[3 * a] * r[0] + M[3 * a + 1] * r[1] + M[3 * a + 2] * r[2];
  const float mx[3] = {M[5] - M[7], M[6] - M[2], M[1] - M[3]};
  cross3f(Mr, r, t);
  for (int i = 0; i < 3; ++i) u[i] += 3.f * ir5 * t[i] - ir3 * mx[i];
  float N[3][3];  // N[k][c] = (at x M_.c)_k
  for (int c = 0; c < 3; ++c) {
    const float col[3] = {M[c], M[3 + c], M[6 + c]};
    float n[3];
    cross3f(at, col, n);
    N[0][c] = n[0]; N[1][c] = n[1]; N[2][c] = n[2];
  }
  float Nr[3], NTr[3];
  for (int i = 0; i < 3; ++i) {
    Nr[i] = N[i][0] * r[0] + N[i][1] * r[1] + N[i][2] * r[2];
    NTr[i] = N[0][i] * r[0] + N[1][i] * r[1] + N[2][i] * r[2];
  }
  const float rNr = r[0] * Nr[0] + r[1] * Nr[1] + r[2] * Nr[2];
  const float trN = N[0][0] + N[1][1] + N[2][2];
  for (int i = 0; i < 3; ++i) s[i] += -15.f * ir7 * rNr * r[i] + 3.f * ir5 * (Nr[i] + NTr[i] + r[i] * trN);
  if (order < 2) return;
  // ---- quadrupole; Q_a packed (00,01,02,11,12,22)
  const float *Qp = v + 15;
  float sv[3], tv[3], W[3][3];
  for (int a = 0; a < 3; ++a) {
    const float *q = Qp + 6 * a;
    W[a][0] = q[0] * r[0] + q[1] * r[1] + q[2] * r[2];
    W[a][1] = q[1] * r[0] + q[3] * r[1] + q[4] * r[2];
    W[a][2] = q[2] * r[0] + q[4] * r[1] + q[5] * r[2];
    sv[a] = r[0] * W[a][0] + r[1] * W[a][1] + r[2] * W[a][2];
    tv[a] = q[0] + q[3] + q[5];
  }
  const float wx[3] = {W[1][2] - W[2][1], W[2][0] - W[0][2], W[0][1] - W[1][0]};
  float sr[3], tr[3];
  cross3f(sv, r, sr);
  cross3f(tv, r, tr);
  for (int i = 0; i < 3; ++i) u[i] += 7.5f * ir7 * sr[i] - 1.5f * ir5 * (2.f * wx[i] + tr[i]);
  // P_k (symmetric over cd) = (at x Q_.cd)_k
  float P[3][6];
  for (int e = 0; e < 6; ++e) {
    const float col[3] = {Qp[e], Qp[6 + e], Qp[12 + e]};
    float p[3];
    cross3f(at, col, p);
    P[0][e] = p[0]; P[1][e] = p[1]; P[2][e] = p[2];
  }
  float Pr[3][3], rPr[3], trP[3];
  for (int k = 0; k < 3; ++k) {
    const float *q = P[k];
    Pr[k][0] = q[0] * r[0] + q[1] * r[1] + q[2] * r[2];
    Pr[k][1] = q[1] * r[0] + q[3] * r[1] + q[4] * r[2];
    Pr[k][2] = q[2] * r[0] + q[4] * r[1] + q[5] * r[2];
    rPr[k] = r[0] * Pr[k][0] + r[1] * Pr[k][1] + r[2] * Pr[k][2];
    trP[k] = q[0] + q[3] + q[5];
  }
  const float srPr = r[0] * rPr[0] + r[1] * rPr[1] + r[2] * rPr[2];
  const float sPrk = Pr[0][0] + Pr[1][1] + Pr[2][2];  // sum_k (P_k r)_k
  const float rtr = r[0] * trP[0] + r[1] * trP[1] + r[2] * trP[2];
  // sum_k P_k[i][k]: P_k packed; entry (i,k)
  auto pik = [&](int k, int i) {
    const int a = min(i, k), b = max(i, k);
    const int e = a == 0 ? b : (a == 1 ? 2 + b : 5);
    return P[k][e];
  };
  for (int i = 0; i < 3; ++i) {
    const float sumPk = r[0] * Pr[0][i] + r[1] * Pr[1][i] + r[2] * Pr[2][i];
    const float spik = pik(0, i) + pik(1, i) + pik(2, i);
    const float d4p = 105.f * ir9 * r[i] * srPr -
                      15.f * ir7 * (rPr[i] + 2.f * sumPk + 2.f * r[i] * sPrk + r[i] * rtr) +
                      3.f * ir5 * (trP[i] + 2.f * spik);
    s[i] -= 0.5f * d4p;
  }
  if (order < 3) return;
  // ---- octupole; T_a packed (000,001,002,011,012,022,111,112,122,222).
  // For a symmetric third-order tensor S: Sr[b][d] = S_bde r_e (symmetric),
  // S1 = Sr r, S0 = S1.r, tS_b = S_bdd, and S_ccd r_d = tS.r.
  //   u_i += 1/6 eps_iab [105 S0_a r_b / rho^9 - 45 (S1_ab + r_b (tS_a.r)) / rho^7 + 9 tS_ab / rho^5]
  //   s_i += 1/6 D5_ikcde R_kcde, R_k = (alpha_t x T_.)_k, by the pairings of
  //   D5 = -945 r r r r r / rho^11 + 105 sum_10 (delta r r r) / rho^9 - 15 sum_15 (delta delta r) / rho^7
  const float ir11 = ir9 * ir2;
  auto sym3 = [&](const float *S, float Sr[3][3], float *S1, float &S0, float *tS) {
    // S index of (b, c, d), b <= c <= d sorted
    Sr[0][0] = S[0] * r[0] + S[1] * r[1] + S[2] * r[2];
    Sr[0][1] = S[1] * r[0] + S[3] * r[1] + S[4] * r[2];
    Sr[0][2] = S[2] * r[0] + S[4] * r[1] + S[5] * r[2];
    Sr[1][1] = S[3] * r[0] + S[6] * r[1] + S[7] * r[2];
    Sr[1][2] = S[4] * r[0] + S[7] * r[1] + S[8] * r[2];
    Sr[2][2] = S[5] * r[0] + S[8] * r[1] + S[9] * r[2];
    Sr[1][0] = Sr[0][1]; Sr[2][0] = Sr[0][2]; Sr[2][1] = Sr[1][2];
    for (int b = 0; b < 3; ++b) S1[b] = Sr[b][0] * r[0] + Sr[b][1] * r[1] + Sr[b][2] * r[2];
    S0 = S1[0] * r[0] + S1[1] * r[1] + S1[2] * r[2];
    tS[0] = S[0] + S[3] + S[5];
    tS[1] = S[1] + S[6] + S[8];
    tS[2] = S[2] + S[7] + S[9];
  };
  const float *Tp = v + 40;
  {
    float S0[3], S1[3][3], tS[3][3], Sr[3][3];
    for (int a = 0; a < 3; ++a) sym3(Tp + 10 * a, Sr, S1[a], S0[a], tS[a]);
    for (int i = 0; i < 3; ++i) {
      const int a1 = (i + 1) % 3, b1 = (i + 2) % 3;  // eps_i a1 b1 = +1
      const float x1 = 105.f * ir9 * (S0[a1] * r[b1] - S0[b1] * r[a1]);
      const float sa1 = tS[a1][0] * r[0] + tS[a1][1] * r[1] + tS[a1][2] * r[2];
      const float sb1 = tS[b1][0] * r[0] + tS[b1][1] * r[1] + tS[b1][2] * r[2];
      const float x2 = -45.f * ir7 * ((S1[a1][b1] - S1[b1][a1]) + (sa1 * r[b1] - sb1 * r[a1]));
      const float x3 = 9.f * ir5 * (tS[a1][b1] - tS[b1][a1]);
      u[i] += (x1 + x2 + x3) * (1.f / 6.f);
    }
  }
  {
    // R_k = (alpha_t x T_.)_k, each a symmetric third-order tensor
    float R[3][10];
    for (int e = 0; e < 10; ++e) {
      const float col[3] = {Tp[e], Tp[10 + e], Tp[20 + e]};
      float p[3];
      cross3f(at, col, p);
      R[0][e] = p[0]; R[1][e] = p[1]; R[2][e] = p[2];
    }
    float M[3][3][3], r1[3][3], r0[3], tk[3][3];
    for (int k = 0; k < 3; ++k) sym3(R[k], M[k], r1[k], r0[k], tk[k]);
    float rr0 = 0.f, tr1 = 0.f, rsg = 0.f, trt = 0.f;
    for (int k = 0; k < 3; ++k) {
      rr0 += r[k] * r0[k];
      tr1 += r1[k][k];
      rsg += r[k] * (tk[k][0] * r[0] + tk[k][1] * r[1] + tk[k][2] * r[2]);
      trt += tk[k][k];
    }
    for (int i = 0; i < 3; ++i) {
      float rk1 = 0.f, rkt = 0.f, psi = 0.f;
      for (int k = 0; k < 3; ++k) {
        rk1 += r[k] * r1[k][i];
        rkt += r[k] * tk[k][i];
        psi += M[k][i][k];
      }
      const float ti_r = tk[i][0] * r[0] + tk[i][1] * r[1] + tk[i][2] * r[2];
      const float t1 = -945.f * ir11 * r[i] * rr0;
      const float t2 = 105.f * ir9 * (r0[i] + 3.f * rk1 + 3.f * r[i] * tr1 + 3.f * r[i] * rsg);
      const float t3 = -15.f * ir7 * (3.f * r[i] * trt + 3.f * rkt + 3.f * ti_r + 6.f * psi);
      s[i] += (t1 + t2 + t3) * (1.f / 6.f);
    }
  }
}

// Input features of the far-field correction network for one (target, far
// cell) pair, and the scales of its outputs.  With r = x_t - c (c the cell's
// particle centroid, the expansion origin), rho = |r|, rh = r/rho, w the cube
// width, A = sum alpha, Q_j = sum alpha_j y y^T (y = x_s - c) the second
// moments and C = sum_j (A_j/|A|) Q_j:
//   0-2 rh, 3 4w/rho, 4 4 sigma_c/rho, 5-7 A/|A|,
//   8-10 4 eps_ijk (Q_j rh)_k / (|A| w^2), 11-13 4 rh.Q_j.rh / (|A| w^2),
//   14-16 4 tr Q_j / (|A| w^2), 17-19 16 C rh/(|A| rho^2),
//   20-22 alpha_t/|alpha_t|, 23 16 rh.C.rh/(|A| rho^2)
// The residual of the monopole+dipole expansion is led by the quadrupole
// term, whose velocity is exactly
//   (-3 eps_ijk (Q_j rh)_k + (7.5 rh.Q_j.rh - 1.5 tr Q_j) (e_j x rh)_i) / rho^4
// (4 pi units), a function of slots 0-2 and 8-16 alone; its stretching
// also involves alpha_t, and for strengths close to one direction (Q_j ~
// A_j C / |A|) it depends on C through C rh and rh.C.rh.  sigma_c (the cell's
// mean smoothing radius) carries what is left of the Gaussian regularisation
// for cells only a few radii away.  The network predicts the residual in
// units of the quadrupole scale: velocity / (|A| w^2 / rho^4), stretching /
// (|A| |alpha_t| w^2 / rho^5) (4 pi units).
__device__ __forceinline__ void far_features(const float *v, const float *x, const float *at, float *f, float &sv,
                                             float &ss) {
  const float r[3] = {x[0] - v[0], x[1] - v[1], x[2] - v[2]};
  const float r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
  const float ir = fast_rsqrt(r2);
  const float rh[3] = {r[0] * ir, r[1] * ir, r[2] * ir};
  for (int i = 0; i < 3; ++i) f[i] = rh[i];
  const float w = v[34];
  f[3] = 4.f * w * ir;
  f[4] = 4.f * sqrtf(2.f * v[38]) * ir;
  const float am = sqrtf(v[3] * v[3] + v[4] * v[4] + v[5] * v[5]);
  const float ia = am > 0.f ? 1.f / am : 0.f;
  const float ah[3] = {v[3] * ia, v[4] * ia, v[5] * ia};
  for (int i = 0; i < 3; ++i) f[5 + i] = ah[i];
  const float qs = w > 0.f ? 4.f * ia / (w * w) : 0.f;
  float P[3][3];  // P[j] = Q_j rh
  for (int j = 0; j < 3; ++j) {
    const float *Q = v + 15 + 6 * j;
    P[j][0] = Q[0] * rh[0] + Q[1] * rh[1] + Q[2] * rh[2];
    P[j][1] = Q[1] * rh[0] + Q[3] * rh[1] + Q[4] * rh[2];
    P[j][2] = Q[2] * rh[0] + Q[4] * rh[1] + Q[5] * rh[2];
    f[11 + j] = qs * (rh[0] * P[j][0] + rh[1] * P[j][1] + rh[2] * P[j][2]);
    f[14 + j] = qs * (Q[0] + Q[3] + Q[5]);
  }
  f[8] = qs * (P[1][2] - P[2][1]);
  f[9] = qs * (P[2][0] - P[0][2]);
  f[10] = qs * (P[0][1] - P[1][0]);
  // C = sum_a ah_a Q_a, packed (00,01,02,11,12,22)
  float Cp[6];
  for (int e = 0; e < 6; ++e) Cp[e] = ah[0] * v[15 + e] + ah[1] * v[21 + e] + ah[2] * v[27 + e];
  const float Cr[3] = {Cp[0] * rh[0] + Cp[1] * rh[1] + Cp[2] * rh[2], Cp[1] * rh[0] + Cp[3] * rh[1] + Cp[4] * rh[2],
                       Cp[2] * rh[0] + Cp[4] * rh[1] + Cp[5] * rh[2]};
  const float cs = 16.f * ia * ir * ir;
  for (int i = 0; i < 3; ++i) f[17 + i] = cs * Cr[i];
  const float tm = sqrtf(at[0] * at[0] + at[1] * at[1] + at[2] * at[2]);
  const float it = tm > 0.f ? 1.f / tm : 0.f;
  for (int i = 0; i < 3; ++i) f[20 + i] = at[i] * it;
  f[23] = cs * (rh[0] * Cr[0] + rh[1] * Cr[1] + rh[2] * Cr[2]);
  const float q2 = (w * ir) * (w * ir);
  sv = am * ir * ir * q2;
  ss = am * tm * ir * ir * ir * q2;
}

// One ordered pair with the FP32 three-regime terms of the direct kernel,
// accumulated into CG-group partial sums.  Must be called by all lanes of a
// warp together (it votes).
__device__ __forceinline__ void pair_accum_f32(const float4 p, const float4 q, const float *xt, const float *at,
                                               float hst, float h50, float vt, float *sv, float *sd, float *sp,
                                               float *sdv) {
  const float dx = xt[0] - p.x, dy = xt[1] - p.y, dz = xt[2] - p.z;
  const float r2 = dx * dx + dy * dy + dz * dz;
  const bool near = fmaf(-kFarU, p.w, r2) < h50;
  const float ir = fast_rsqrt(r2);
  const float A = ir * ir;
  float qq = A * ir, FF = -3.0f * qq * A, zd = 0.f;
  bool diffuse = false;
  if (__any_sync(0xffffffffu, near)) {
    if (near) {
      const PairTerms<float> pt = pair_terms_near(r2, hst + p.w);
      qq = pt.q; FF = pt.F; zd = pt.zd;
      diffuse = true;
    }
  }
  const float wx = q.y * dz - q.z * dy, wy = q.z * dx - q.x * dz, wz = q.x * dy - q.y * dx;
  sv[0] += qq * wx; sv[1] += qq * wy; sv[2] += qq * wz;
  const float fd = FF * (at[0] * wx + at[1] * wy + at[2] * wz);
  sd[0] += fd * dx; sd[1] += fd * dy; sd[2] += fd * dz;
  sp[0] += qq * q.x; sp[1] += qq * q.y; sp[2] += qq * q.z;
  if (diffuse) {
    sdv[0] += zd * (vt * q.x - q.w * at[0]);
    sdv[1] += zd * (vt * q.y - q.w * at[1]);
    sdv[2] += zd * (vt * q.z - q.w * at[2]);
  }
}

__device__ __forceinline__ void fold_group(const float *at, float nu2, float *sv, float *sd, float *sp, float *sdv,
                                           float *vh, float *vl, float *dh, float *dl) {
  const float e[3] = {at[1] * sp[2] - at[2] * sp[1] + sd[0] + nu2 * sdv[0],
                      at[2] * sp[0] - at[0] * sp[2] + sd[1] + nu2 * sdv[1],
                      at[0] * sp[1] - at[1] * sp[0] + sd[2] + nu2 * sdv[2]};
  for (int m = 0; m < 3; ++m) {
    two_sum_acc(vh[m], vl[m], sv[m]);
    two_sum_acc(dh[m], dl[m], e[m]);
    sv[m] = sd[m] = sp[m] = sdv[m] = 0.f;
  }
}

struct TreeEvalArgs {
  const CellData *cd;
  const TreeCell *cells;
  const int *leaves;
  int nleaves;
  const int *far_off, *far_cnt, *far_list;
  const int *near_off, *near_cnt;
  const int2 *near_runs;  // sorted-order particle ranges of the near field
  const float4 *Ps, *Qs;  // sorted records
  const int *idx;         // sorted position -> index within the system
  int64_t off;            // slot offset of the system
  double *partial;        // chunk 0 of [nch][6][cap]
  int64_t cap;
  float nu2;
  int order;
  // owned targets [own_lo, own_hi) (indices within the system); a context
  // with a target range evaluates and writes only these
  int own_lo, own_hi;
};

constexpr int kTreeBlock = 256;  // sampled-check kernel


// Warp-independent form: every warp takes work items (target leaf, slice of
// 32 of its targets) from an atomic counter and stages its own source tiles,
// synchronising only within the warp.  Leaves average ~130 particles, so
// whole-leaf CTAs leave most warps idle; independent warps keep ~48 warps per
// SM busy.  items[k] = (leaf index, slice); counter[0] must be 0 at launch.
constexpr int kWarpTile = 64;
constexpr int kWarpCells = 16;
constexpr int kWarpsPerCta = 4;

// Per-warp shared buffers (all carved from dynamic shared memory, after the
// packed network when the correction is on).
struct WarpSmem {
  float sc[kWarpCells][kCellFloats];
  float4 sP[kWarpTile], sQ[kWarpTile];
};
struct WarpSmemMlp {
  __nv_bfloat16 sF[32][kInPad + 8];
  float sO[32][kOutPad];
};
constexpr int kWarpsPerCtaMlp = 12;  // warps sharing one copy of the network
template <bool MLP> constexpr int eval_warps() { return MLP ? kWarpsPerCtaMlp : kWarpsPerCta; }
template <bool MLP> constexpr size_t eval_smem() {
  return (MLP ? sizeof(MlpPacked) : 0) + eval_warps<MLP>() * (sizeof(WarpSmem) + (MLP ? sizeof(WarpSmemMlp) : 0));
}

template <bool MLP>
__global__ void __launch_bounds__(32 * eval_warps<MLP>()) tree_eval_warp_kernel(TreeEvalArgs a, const int2 *items,
                                                                             int nitems, unsigned *counter,
                                                                             const MlpPacked *mlp) {
  extern __shared__ __align__(16) unsigned char dyn_smem[];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const size_t off0 = MLP ? sizeof(MlpPacked) : 0;
  WarpSmem &ws = reinterpret_cast<WarpSmem *>(dyn_smem + off0)[w];
  WarpSmemMlp &wm = reinterpret_cast<WarpSmemMlp *>(dyn_smem + off0 + eval_warps<MLP>() * sizeof(WarpSmem))[w];
  if constexpr (MLP) {
    // the packed network, shared by the CTA's warps
    const uint4 *src = reinterpret_cast<const uint4 *>(mlp);
    uint4 *dst = reinterpret_cast<uint4 *>(dyn_smem);
    for (int i = threadIdx.x; i < (int)(sizeof(MlpPacked) / 16); i += blockDim.x) dst[i] = src[i];
    __syncthreads();
  }
  const MlpPacked &W = *reinterpret_cast<const MlpPacked *>(dyn_smem);
  for (;;) {
    int item = 0;
    if (lane == 0) item = (int)atomicAdd(counter, 1u);
    item = __shfl_sync(0xffffffffu, item, 0);
    if (item >= nitems) break;
    const int2 it = items[item];
    const int li = it.x;
    const TreeCell tc = a.cells[a.leaves[li]];
    const int t0 = tc.start + it.y * 32 + lane;
    const int t = min(t0, tc.end - 1);
    const int ti = a.idx[t];
    const bool mine = t0 < tc.end && ti >= a.own_lo && ti < a.own_hi;
    if (!__any_sync(0xffffffffu, mine)) continue;  // a slice with no owned target
    const float4 pt = a.Ps[t], qt = a.Qs[t];
    const float xt[3] = {pt.x, pt.y, pt.z}, at[3] = {qt.x, qt.y, qt.z};
    const float hst = pt.w, vt = qt.w;
    float vh[3] = {0, 0, 0}, vl[3] = {0, 0, 0}, dh[3] = {0, 0, 0}, dl[3] = {0, 0, 0};
    const int fo = a.far_off[li], fn = a.far_cnt[li];
    for (int c0 = 0; c0 < fn; c0 += kWarpCells) {
      const int cn = min(kWarpCells, fn - c0);
      __syncwarp();
      // the cell data the expansion reads: the third moments only at order 3
      const int nf = a.order >= 3 ? kCellFloats : 40;
      for (int e = lane; e < cn * nf; e += 32)
        ws.sc[e / nf][e % nf] = a.cd[a.far_list[fo + c0 + e / nf]].v[e % nf];
      __syncwarp();
      float su[3] = {0, 0, 0}, ss[3] = {0, 0, 0};
      for (int j = 0; j < cn; ++j) {
        float u[3], s[3];
        far_expand(ws.sc[j], xt, at, a.order, u, s);
        for (int m = 0; m < 3; ++m) { su[m] += u[m]; ss[m] += s[m]; }
        if constexpr (MLP) {
          float f[kIn], scv, scs;
          far_features(ws.sc[j], xt, at, f, scv, scs);
          for (int i = 0; i < kIn; i += 2) *reinterpret_cast<uint32_t *>(&wm.sF[lane][i]) = pack_bf16(f[i], f[i + 1]);
          for (int i = kIn; i < kInPad; i += 2) *reinterpret_cast<uint32_t *>(&wm.sF[lane][i]) = 0u;
          __syncwarp();
          mlp_tile16(W, wm.sF, wm.sO, lane);
          mlp_tile16(W, wm.sF + 16, wm.sO + 16, lane);
          __syncwarp();
          for (int m = 0; m < 3; ++m) {
            su[m] += scv * wm.sO[lane][m];
            ss[m] += scs * wm.sO[lane][3 + m];
          }
          __syncwarp();
        }
      }
      for (int m = 0; m < 3; ++m) {
        two_sum_acc(vh[m], vl[m], su[m]);
        two_sum_acc(dh[m], dl[m], ss[m]);
      }
    }
    // Near field, two sources per packed FP32 instruction (lane .x the even
    // source of a pair, .y the odd one; pair-interleaved staging as in the
    // direct kernel).  A 64-source sub-tile whose box is far from the warp's
    // 32 targets (every pair at u >= 50) takes the far limit; the others take
    // the closed form for every pair, and lanes at u < 1, the self pair among
    // them, the series.  On the 4M coaxial rings the all-far sub-tiles cut
    // the evaluation from 933 to 869 ms; boxes per 32-source half cut fewer
    // pairs than their second reduction cost (877 ms).
    const float2 X2[3] = {dup2(xt[0]), dup2(xt[1]), dup2(xt[2])};
    const float2 AT2[3] = {dup2(at[0]), dup2(at[1]), dup2(at[2])};
    const float2 NAT2[3] = {dup2(-at[0]), dup2(-at[1]), dup2(-at[2])};
    const float2 HS2 = dup2(hst), VT2 = dup2(vt), M1 = dup2(-1.f);
    const float2 AT3[3] = {dup2(-3.f * at[0]), dup2(-3.f * at[1]), dup2(-3.f * at[2])};
    // bounding box of the warp's targets, for the per-sub-tile all-far test
    WarpBox tb;
    tb.init();
    tb.add(xt[0], xt[1], xt[2], hst);
    tb.reduce();
    const int no = a.near_off[li], nn = a.near_cnt[li];
    for (int ni = 0; ni < nn; ++ni) {
      const int2 run = a.near_runs[no + ni];
      for (int sb = run.x; sb < run.y; sb += kWarpTile) {
        __syncwarp();
        WarpBox sbx;
        sbx.init();
        for (int k = lane; k < kWarpTile; k += 32) {
          const int j = sb + k;
          const float4 p = j < run.y ? a.Ps[j] : pad_P<float>();
          const float4 q = j < run.y ? a.Qs[j] : pad_Q<float>();
          if (j < run.y) sbx.add(p.x, p.y, p.z, p.w);
          float *dp = reinterpret_cast<float *>(ws.sP) + (k >> 1) * 8 + (k & 1);
          float *dq = reinterpret_cast<float *>(ws.sQ) + (k >> 1) * 8 + (k & 1);
          dp[0] = p.x; dp[2] = p.y; dp[4] = p.z; dp[6] = p.w;
          dq[0] = q.x; dq[2] = q.y; dq[4] = q.z; dq[6] = q.w;
        }
        sbx.reduce();
        // every pair of the warp's targets with this sub-tile at u >= 50: the
        // far limit (q = 1/rho^3, F = -3/rho^5, no diffusion), as the direct
        // kernel's all-far tiles
        const bool far_tile = all_far(tb, sbx);
        __syncwarp();
        // source pairs; an odd tail pairs with a padding source (zero strength, far away)
        const int npr = (min(kWarpTile, run.y - sb) + 1) >> 1;
        if (far_tile) {
          for (int g = 0; g < npr; g += 16) {
            float2 sv2[3], sd2[3], sp2[3];
            for (int m = 0; m < 3; ++m) { sv2[m] = sd2[m] = sp2[m] = dup2(0.f); }
            const int ge = min(npr, g + 16);
            for (int r = g; r < ge; ++r) {
              const float4 pa = ws.sP[2 * r], pb = ws.sP[2 * r + 1];
              const float4 qa = ws.sQ[2 * r], qb = ws.sQ[2 * r + 1];
              const float2 dx = __ffma2_rn(make_float2(pa.x, pa.y), M1, X2[0]);
              const float2 dy = __ffma2_rn(make_float2(pa.z, pa.w), M1, X2[1]);
              const float2 dz = __ffma2_rn(make_float2(pb.x, pb.y), M1, X2[2]);
              const float2 ax = make_float2(qa.x, qa.y), ay = make_float2(qa.z, qa.w), az = make_float2(qb.x, qb.y);
              float2 r2 = __fmul2_rn(dx, dx);
              r2 = __ffma2_rn(dy, dy, r2);
              r2 = __ffma2_rn(dz, dz, r2);
              const float2 ir = make_float2(fast_rsqrt(r2.x), fast_rsqrt(r2.y));
              const float2 A = __fmul2_rn(ir, ir);
              const float2 qq = __fmul2_rn(A, ir);
              const float2 qA = __fmul2_rn(qq, A);
              const float2 wx = make_float2(ay.x * dz.x - az.x * dy.x, ay.y * dz.y - az.y * dy.y);
              const float2 wy = make_float2(az.x * dx.x - ax.x * dz.x, az.y * dx.y - ax.y * dz.y);
              const float2 wz = make_float2(ax.x * dy.x - ay.x * dx.x, ax.y * dy.y - ay.y * dx.y);
              sv2[0] = __ffma2_rn(qq, wx, sv2[0]);
              sv2[1] = __ffma2_rn(qq, wy, sv2[1]);
              sv2[2] = __ffma2_rn(qq, wz, sv2[2]);
              float2 dot = __fmul2_rn(AT3[0], wx);
              dot = __ffma2_rn(AT3[1], wy, dot);
              dot = __ffma2_rn(AT3[2], wz, dot);
              const float2 fd = __fmul2_rn(qA, dot);
              sd2[0] = __ffma2_rn(fd, dx, sd2[0]);
              sd2[1] = __ffma2_rn(fd, dy, sd2[1]);
              sd2[2] = __ffma2_rn(fd, dz, sd2[2]);
              sp2[0] = __ffma2_rn(qq, ax, sp2[0]);
              sp2[1] = __ffma2_rn(qq, ay, sp2[1]);
              sp2[2] = __ffma2_rn(qq, az, sp2[2]);
            }
            float sv[3], sd[3], sp[3], sdv[3] = {0.f, 0.f, 0.f};
            for (int m = 0; m < 3; ++m) {
              sv[m] = sv2[m].x + sv2[m].y;
              sd[m] = sd2[m].x + sd2[m].y;
              sp[m] = sp2[m].x + sp2[m].y;
            }
            fold_group(at, a.nu2, sv, sd, sp, sdv, vh, vl, dh, dl);
          }
          continue;
        }
        for (int g = 0; g < npr; g += 16) {
          float2 sv2[3], sd2[3], sp2[3], sdv2[3];
          for (int m = 0; m < 3; ++m) { sv2[m] = sd2[m] = sp2[m] = sdv2[m] = dup2(0.f); }
          const int ge = min(npr, g + 16);
          for (int r = g; r < ge; ++r) {
            const float4 pa = ws.sP[2 * r], pb = ws.sP[2 * r + 1];
            const float4 qa = ws.sQ[2 * r], qb = ws.sQ[2 * r + 1];
            const float2 dx = __ffma2_rn(make_float2(pa.x, pa.y), M1, X2[0]);
            const float2 dy = __ffma2_rn(make_float2(pa.z, pa.w), M1, X2[1]);
            const float2 dz = __ffma2_rn(make_float2(pb.x, pb.y), M1, X2[2]);
            const float2 ax = make_float2(qa.x, qa.y), ay = make_float2(qa.z, qa.w), az = make_float2(qb.x, qb.y);
            float2 r2 = __fmul2_rn(dx, dx);
            r2 = __ffma2_rn(dy, dy, r2);
            r2 = __ffma2_rn(dz, dz, r2);
            const float2 s2 = __fadd2_rn(HS2, make_float2(pb.z, pb.w));
            PairTerms2 t = pair_terms_mid2(r2, s2);
            const bool lx = r2.x < s2.x, ly = r2.y < s2.y;  // u < 1
            if (__any_sync(0xffffffffu, lx || ly)) {
              if (lx) { const PairTerms<float> e = pair_terms_near(r2.x, s2.x); t.q.x = e.q; t.F.x = e.F; t.zd.x = e.zd; }
              if (ly) { const PairTerms<float> e = pair_terms_near(r2.y, s2.y); t.q.y = e.q; t.F.y = e.F; t.zd.y = e.zd; }
            }
            // w = alpha_s x d (scalar: the negated operand is free)
            const float2 wx = make_float2(ay.x * dz.x - az.x * dy.x, ay.y * dz.y - az.y * dy.y);
            const float2 wy = make_float2(az.x * dx.x - ax.x * dz.x, az.y * dx.y - ax.y * dz.y);
            const float2 wz = make_float2(ax.x * dy.x - ay.x * dx.x, ax.y * dy.y - ay.y * dx.y);
            sv2[0] = __ffma2_rn(t.q, wx, sv2[0]);
            sv2[1] = __ffma2_rn(t.q, wy, sv2[1]);
            sv2[2] = __ffma2_rn(t.q, wz, sv2[2]);
            float2 dot = __fmul2_rn(AT2[0], wx);
            dot = __ffma2_rn(AT2[1], wy, dot);
            dot = __ffma2_rn(AT2[2], wz, dot);
            const float2 fd = __fmul2_rn(t.F, dot);
            sd2[0] = __ffma2_rn(fd, dx, sd2[0]);
            sd2[1] = __ffma2_rn(fd, dy, sd2[1]);
            sd2[2] = __ffma2_rn(fd, dz, sd2[2]);
            sp2[0] = __ffma2_rn(t.q, ax, sp2[0]);
            sp2[1] = __ffma2_rn(t.q, ay, sp2[1]);
            sp2[2] = __ffma2_rn(t.q, az, sp2[2]);
            // diffusion per pair: zeta (v_t a_s - v_s a_t), as in DIFFUSION (interaction_utils.h:358-369)
            const float2 vs = make_float2(qb.z, qb.w);
            sdv2[0] = __ffma2_rn(t.zd, __ffma2_rn(vs, NAT2[0], __fmul2_rn(VT2, ax)), sdv2[0]);
            sdv2[1] = __ffma2_rn(t.zd, __ffma2_rn(vs, NAT2[1], __fmul2_rn(VT2, ay)), sdv2[1]);
            sdv2[2] = __ffma2_rn(t.zd, __ffma2_rn(vs, NAT2[2], __fmul2_rn(VT2, az)), sdv2[2]);
          }
          float sv[3], sd[3], sp[3], sdv[3];
          for (int m = 0; m < 3; ++m) {
            sv[m] = sv2[m].x + sv2[m].y;
            sd[m] = sd2[m].x + sd2[m].y;
            sp[m] = sp2[m].x + sp2[m].y;
            sdv[m] = sdv2[m].x + sdv2[m].y;
          }
          fold_group(at, a.nu2, sv, sd, sp, sdv, vh, vl, dh, dl);
        }
      }
    }
    if (mine) {
      double *o = a.partial + a.off + ti;
      for (int m = 0; m < 3; ++m) {
        o[m * a.cap] = ((double)vh[m] + (double)vl[m]) * kInv4Pi;
        o[(3 + m) * a.cap] = ((double)dh[m] + (double)dl[m]) * kInv4Pi;
      }
    }
  }
}

// Training samples of the correction network from the current octree: each
// warp draws (leaf, target, far cell) with a hash of (seed, sample), computes
// the features, the exact FP64 contribution of the cell's particles (the
// direct kernel's formula) and the expansion to the surrogate's order
// (a.order), and stores the scaled residual.  Rows whose leaf has no far cell
// after 32 draws are all zero.
__global__ void mlp_sample_kernel(TreeEvalArgs a, const int *far_leaves, int nfar_leaves, int nsamples,
                                  unsigned long long seed, float *X, float *T) {
  const int lane = threadIdx.x & 31;
  const int wg = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (int smp = wg; smp < nsamples; smp += nw) {
    int li = -1, t = 0, fj = 0;
    if (lane == 0) {
      unsigned long long h = seed ^ (0x9E3779B97F4A7C15ULL * (unsigned long long)(smp + 1));
      h ^= h >> 33; h *= 0xFF51AFD7ED558CCDULL; h ^= h >> 33; h *= 0xC4CEB9FE1A85EC53ULL; h ^= h >> 33;
      const int l = far_leaves[(int)(h % (unsigned long long)nfar_leaves)];
      const TreeCell tc = a.cells[a.leaves[l]];
      li = l;
      t = tc.start + (int)((h >> 20) % (unsigned long long)(tc.end - tc.start));
      fj = (int)((h >> 40) % (unsigned long long)a.far_cnt[l]);
    }
    li = __shfl_sync(0xffffffffu, li, 0);
    t = __shfl_sync(0xffffffffu, t, 0);
    fj = __shfl_sync(0xffffffffu, fj, 0);
    float *xo = X + (int64_t)smp * kIn;
    float *to = T + (int64_t)smp * kOut;
    if (li < 0) {
      if (lane < kIn) xo[lane] = 0.f;
      if (lane < kOut) to[lane] = 0.f;
      continue;
    }
    const int ci = a.far_list[a.far_off[li] + fj];
    const TreeCell cc = a.cells[ci];
    const float *v = a.cd[ci].v;
    const float4 pt = a.Ps[t], qt = a.Qs[t];
    const float xt[3] = {pt.x, pt.y, pt.z}, at[3] = {qt.x, qt.y, qt.z};
    double ex[6] = {0, 0, 0, 0, 0, 0};
    for (int j = cc.start + lane; j < cc.end; j += 32) {
      const float4 p = a.Ps[j], q = a.Qs[j];
      const double d[3] = {(double)pt.x - p.x, (double)pt.y - p.y, (double)pt.z - p.z};
      const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      const PairTerms<double> k = pair_terms(r2, (double)pt.w + (double)p.w);
      const double as[3] = {q.x, q.y, q.z}, a_t[3] = {qt.x, qt.y, qt.z};
      const double w3[3] = {as[1] * d[2] - as[2] * d[1], as[2] * d[0] - as[0] * d[2], as[0] * d[1] - as[1] * d[0]};
      const double c3[3] = {a_t[1] * as[2] - a_t[2] * as[1], a_t[2] * as[0] - a_t[0] * as[2], a_t[0] * as[1] - a_t[1] * as[0]};
      const double dc = d[0] * c3[0] + d[1] * c3[1] + d[2] * c3[2];
      for (int m = 0; m < 3; ++m) {
        ex[m] += k.q * w3[m];
        ex[3 + m] += k.q * c3[m] + k.F * dc * d[m];
      }
    }
    for (int m = 0; m < 6; ++m)
      for (int o = 16; o > 0; o >>= 1) ex[m] += __shfl_down_sync(0xffffffffu, ex[m], o);
    if (lane == 0) {
      float f[kIn], scv, scs, u[3], s[3];
      far_features(v, xt, at, f, scv, scs);
      far_expand(v, xt, at, a.order, u, s);
      for (int i = 0; i < kIn; ++i) xo[i] = f[i];
      for (int m = 0; m < 3; ++m) {
        to[m] = scv > 0.f ? (float)((ex[m] - u[m]) / scv) : 0.f;
        to[3 + m] = scs > 0.f ? (float)((ex[3 + m] - s[m]) / scs) : 0.f;
      }
    }
  }
}

// (leaf, slice) work items: count[li] = ceil(size / 32), then written at the
// exclusive-scan offsets.
__global__ void slice_count_kernel(const TreeCell *cells, const int *leaves, int nleaves, int *cnt) {
  const int li = blockIdx.x * blockDim.x + threadIdx.x;
  if (li < nleaves) {
    const TreeCell c = cells[leaves[li]];
    cnt[li] = (c.end - c.start + 31) / 32;
  }
}
__global__ void slice_write_kernel(const int *cnt, const int *off, int nleaves, int2 *items) {
  const int li = blockIdx.x * blockDim.x + threadIdx.x;
  if (li < nleaves)
    for (int k = 0; k < cnt[li]; ++k) items[off[li] + k] = make_int2(li, k);
}

// Exact rates (direct FP32C sum over all n particles of the system) at nt
// sampled targets, split over gridDim.y source chunks:
// out[c][m][t], m = 0..5.
__global__ void __launch_bounds__(kTreeBlock) sample_exact_kernel(const float4 *P, const float4 *Q, int64_t off,
                                                                  int64_t n, const int *targets, int nt, float nu2,
                                                                  double *out) {
  __shared__ float4 sP[kTreeBlock], sQ[kTreeBlock];
  const int tid = threadIdx.x;
  const int ti = blockIdx.x * kTreeBlock + tid;
  const int64_t t = off + targets[min(ti, nt - 1)];
  const float4 pt = P[t], qt = Q[t];
  const float xt[3] = {pt.x, pt.y, pt.z}, at[3] = {qt.x, qt.y, qt.z};
  const float hst = pt.w, h50 = kFarU * pt.w, vt = qt.w;
  float vh[3] = {0, 0, 0}, vl[3] = {0, 0, 0}, dh[3] = {0, 0, 0}, dl[3] = {0, 0, 0};
  const int64_t per = (n + gridDim.y - 1) / gridDim.y;
  const int64_t s0 = off + blockIdx.y * per, s1 = min(off + n, s0 + per);
  for (int64_t sb = s0; sb < s1; sb += kTreeBlock) {
    __syncthreads();
    const int64_t j = sb + tid;
    if (j < s1) { sP[tid] = P[j]; sQ[tid] = Q[j]; }
    else { sP[tid] = pad_P<float>(); sQ[tid] = pad_Q<float>(); }
    __syncthreads();
    for (int g = 0; g < kTreeBlock; g += 32) {
      float sv[3] = {}, sd[3] = {}, sp[3] = {}, sdv[3] = {};
      for (int jj = 0; jj < 32; ++jj) pair_accum_f32(sP[g + jj], sQ[g + jj], xt, at, hst, h50, vt, sv, sd, sp, sdv);
      fold_group(at, nu2, sv, sd, sp, sdv, vh, vl, dh, dl);
    }
  }
  if (ti < nt) {
    double *o = out + (int64_t)blockIdx.y * 6 * nt + ti;
    for (int m = 0; m < 3; ++m) {
      o[m * nt] = ((double)vh[m] + (double)vl[m]) * kInv4Pi;
      o[(3 + m) * nt] = ((double)dh[m] + (double)dl[m]) * kInv4Pi;
    }
  }
}

// Max-norm errors of the surrogate rates (chunk 0 of partial) at the sampled
// targets against the exact sums: res[0] = max |dv|^2, res[1] = max |v|^2,
// res[2] = max |d dalpha|^2, res[3] = max |dalpha|^2 (ordered-float atomics).
__global__ void sample_compare_kernel(const double *exact, int chunks, int nt, const int *targets, int64_t off,
                                      const double *partial, int64_t cap, unsigned *res) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nt) return;
  double ex[6];
  for (int m = 0; m < 6; ++m) {
    double v = 0;
    for (int c = 0; c < chunks; ++c) v += exact[((int64_t)c * 6 + m) * nt + t];
    ex[m] = v;
  }
  const int64_t i = off + targets[t];
  double dv = 0, v2 = 0, da = 0, a2 = 0;
  for (int m = 0; m < 3; ++m) {
    const double s = partial[m * cap + i], sa = partial[(3 + m) * cap + i];
    dv += (s - ex[m]) * (s - ex[m]);
    v2 += ex[m] * ex[m];
    da += (sa - ex[3 + m]) * (sa - ex[3 + m]);
    a2 += ex[3 + m] * ex[3 + m];
  }
  atomicMax(&res[0], f2ord((float)dv));
  atomicMax(&res[1], f2ord((float)v2));
  atomicMax(&res[2], f2ord((float)da));
  atomicMax(&res[3], f2ord((float)a2));
}

}  // namespace pgpu
