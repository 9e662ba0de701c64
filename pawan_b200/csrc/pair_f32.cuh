// FP32 (compensated) body of the direct pair kernel.
//
// Same work decomposition as the generic body in kernels.cuh: persistent
// CTAs take (system, target tile, source chunk) items; each thread holds TPT
// targets; source tiles of TILE = BLOCK records are double-buffered in shared
// memory with cp.async.  What differs is the arithmetic layout:
//
// * Sources are processed in pairs with the packed two-wide FP32 instructions
//   of sm_100 (__ffma2_rn / __fmul2_rn): lane .x of every float2 belongs to
//   the even source of a pair, lane .y to the odd one.  One packed
//   instruction does two pairs' work in one issue slot, which leaves issue
//   slots for the loads, the rsqrt and the loop, so the FP32 pipe, not the
//   issue rate, bounds the kernel.  The per-lane results are the IEEE
//   round-to-nearest results of the scalar operations.
// * The tile is staged pair-interleaved: for source pair r, float4 2r holds
//   (x0, x1, y0, y1) and 2r+1 holds (z0, z1, hs0, hs1); Q likewise with
//   (ax0, ax1, ay0, ay1), (az0, az1, vol0, vol1).  Each source is copied with
//   four 4-byte cp.async per record, so one 16-byte shared load yields two
//   float2 operands.
// * In all-far tiles, positions are taken relative to the tile's first
//   source, which turns the per-pair cross product alpha_s x d into per-source
//   and per-group work (see the far loop): 25 packed FP32 operations per far
//   pair.  In the other tiles the pair terms are packed too for shapes with
//   two or more targets per thread (scalar for one target), and the cross
//   products stay scalar, where a negated operand is free.
#pragma once

namespace pgpu {

__device__ __forceinline__ void cp_async4(float *smem, const float *gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
}

// FP32: about 48 + 32 TPT registers per thread; enough CTAs per SM to hold
// them (e.g. 3 CTAs of 256 threads with one target each).
template <int BLOCK, int TPT>
constexpr int pair_f32_min_blocks() {
  return 65536 / (BLOCK * (48 + 32 * TPT)) > 0 ? 65536 / (BLOCK * (48 + 32 * TPT)) : 1;
}

// Source pairs per unrolled step of the far loop (1, 2 and 4 time within 3%
// of each other on B200; 2 is best with the autotuner's usual 128x2 shape).
constexpr int kF32Unroll = 2;

template <int BLOCK, int TPT, int CG, bool SPLIT>
__device__ __forceinline__ void pair_body_f32(const PairArgs<float> &a) {
  constexpr int TILE = BLOCK;
  constexpr int TT = BLOCK * TPT;
  constexpr int NPR = TILE / 2;  // source pairs per tile
  static_assert(TILE % CG == 0 && CG % 2 == 0, "compensation group must divide the tile into source pairs");
  __shared__ __align__(16) float4 sP[2][TILE];
  __shared__ __align__(16) float4 sQ[2][TILE];
  // split positions: the sources' FP32 residuals, pair-interleaved like sP
  // (float4 2r = (xl0, xl1, yl0, yl1), 2r+1 = (zl0, zl1, -, -))
  __shared__ __align__(16) float4 sL[SPLIT ? 2 : 1][SPLIT ? TILE : 1];
  __shared__ __align__(16) float4 sN[TILE];  // n_s = (x_s - ref) x alpha_s, pair-interleaved like sP
  __shared__ int s_item;
  const int tid = threadIdx.x;
  const int lane = tid & 31;
  const float2 M1 = make_float2(-1.f, -1.f);
  const int64_t total = a.plan[a.nsys].item_start;
  int64_t item;
  while (next_item(a.counters, total, item, &s_item)) {
    const int si = find_plan(a.plan, a.nsys, item);
    const PlanEntry pe = a.plan[si];
    const int64_t local = item - pe.item_start;
    const int64_t tile = local / a.nch;
    const int c = (int)(local - tile * a.nch);
    const int64_t t0 = pe.off + pe.toff + tile * TT;
    const int64_t tend = pe.off + pe.toff + pe.tn;  // end of the targets
    const int64_t s0 = pe.off + (int64_t)c * pe.chunk;
    const int64_t s1 = min(s0 + pe.chunk, pe.off + pe.n);

    // targets: positions duplicated into both float2 lanes (lane .x serves
    // the scalar code); scalar strength, sigma^2/2 and volume
    float at[TPT][3], hst[TPT], vt[TPT], h50[TPT];
    float xl[SPLIT ? TPT : 1][3];  // targets' position residuals (split positions)
    float2 X[TPT][3], AT3[TPT][3];
    float vh[TPT][3], vl[TPT][3], dh[TPT][3], dl[TPT][3];
    unsigned nfull = 0;  // pairs evaluated with the full (non-far) formula, self pairs included
#pragma unroll
    for (int k = 0; k < TPT; ++k) {
      int64_t ti = t0 + tid + k * BLOCK;
      ti = ti < tend ? ti : tend - 1;
      const float4 p = a.P[ti];
      const float4 q = a.Q[ti];
      if constexpr (SPLIT) {
        const float4 l = a.L[ti];
        xl[k][0] = l.x; xl[k][1] = l.y; xl[k][2] = l.z;
      }
      hst[k] = p.w;
      h50[k] = kFarU * p.w;
      at[k][0] = q.x; at[k][1] = q.y; at[k][2] = q.z; vt[k] = q.w;
#pragma unroll
      for (int m = 0; m < 3; ++m) {
        X[k][m] = dup2(m == 0 ? p.x : m == 1 ? p.y : p.z);
        // -3 alpha_t: the far limit's F' = -3 r^5 with the constant folded in
        AT3[k][m] = make_float2(-3.f * at[k][m], -3.f * at[k][m]);
        vh[k][m] = 0.f; vl[k][m] = 0.f; dh[k][m] = 0.f; dl[k][m] = 0.f;
      }
    }
    // bounding box of this warp's targets and their largest sigma^2/2, for
    // the per-tile all-far test
    WarpBox tb;
    tb.init();
#pragma unroll
    for (int k = 0; k < TPT; ++k) tb.add(X[k][0].x, X[k][1].x, X[k][2].x, hst[k]);
    tb.reduce();

    // Stage source j into buffer b at its pair-interleaved place.
    auto stage = [&](int b, int64_t j) {
      float *dp = reinterpret_cast<float *>(&sP[b][0]) + (tid >> 1) * 8 + (tid & 1);
      float *dq = reinterpret_cast<float *>(&sQ[b][0]) + (tid >> 1) * 8 + (tid & 1);
      if (j < s1) {
        const float *gp = reinterpret_cast<const float *>(a.P + j);
        const float *gq = reinterpret_cast<const float *>(a.Q + j);
#pragma unroll
        for (int m = 0; m < 4; ++m) { cp_async4(dp + 2 * m, gp + m); cp_async4(dq + 2 * m, gq + m); }
      } else {
        // padding source: far away, zero strength and volume (pad_P / pad_Q)
        dp[0] = 1e18f; dp[2] = 1e18f; dp[4] = 1e18f; dp[6] = 1.f;
        dq[0] = 0.f; dq[2] = 0.f; dq[4] = 0.f; dq[6] = 0.f;
      }
      if constexpr (SPLIT) {
        float *dl = reinterpret_cast<float *>(&sL[b][0]) + (tid >> 1) * 8 + (tid & 1);
        if (j < s1) {
          const float *gl = reinterpret_cast<const float *>(a.L + j);
#pragma unroll
          for (int m = 0; m < 3; ++m) cp_async4(dl + 2 * m, gl + m);
        } else {
          dl[0] = 0.f; dl[2] = 0.f; dl[4] = 0.f;
        }
      }
    };

    int buf = 0;
    if (s0 < s1) stage(0, s0 + tid);
    cp_async_commit();

    for (int64_t sb = s0; sb < s1; sb += TILE) {
      if (sb + TILE < s1) stage(buf ^ 1, sb + TILE + tid);
      cp_async_commit();
      cp_async_wait<1>();
      __syncthreads();

      // Positions relative to the tile's first source, ref: with n_s =
      // (x_s - ref) x alpha_s and X' = x_t - ref, alpha_s x d = alpha_s x X' +
      // n_s, so the far loop sums q alpha_s and q n_s and forms the velocity
      // (sum q alpha_s) x X' + sum q n_s once per group; the stretching's
      // alpha_t . w becomes alpha_s . (X' x alpha_t) + n_s . alpha_t.  Keeping
      // ref inside the tile bounds the cancellation by the tile's extent.
      const float *fp = reinterpret_cast<const float *>(&sP[buf][0]);
      const float rx = fp[0], ry = fp[2], rz = fp[4];
      {
        const float *fq = reinterpret_cast<const float *>(&sQ[buf][0]);
        const int e = (tid >> 1) * 8 + (tid & 1);
        const float px = fp[e] - rx, py = fp[e + 2] - ry, pz = fp[e + 4] - rz;
        const float ax = fq[e], ay = fq[e + 2], az = fq[e + 4];
        float *fn = reinterpret_cast<float *>(sN);
        fn[e] = py * az - pz * ay;
        fn[e + 2] = pz * ax - px * az;
        fn[e + 4] = px * ay - py * ax;
      }
      __syncthreads();

      // Every pair of this warp's targets with this tile's sources is far
      // (u >= 50) when the boxes are at least sqrt(50 (hs_t + hs_s)) apart;
      // such tiles take the far limit with no per-pair test.  The boxes'
      // distance is a lower bound of every pair's, so a far pair is never
      // misclassified near; a pair within rounding of u = 50 may take the far
      // limit, whose dropped terms are below 2e-9 there.
      WarpBox sbox;
      sbox.init();
      if (a.box) {
        // the tile's blocks of precomputed boxes (the same address in every
        // lane: one broadcast load each)
#pragma unroll
        for (int k = 0; k < TILE / kBoxGran; ++k) {
          const int64_t b = sb / kBoxGran + k;
          const float4 lo = __ldg(a.box + 2 * b), hi = __ldg(a.box + 2 * b + 1);
          sbox.lo[0] = fminf(sbox.lo[0], lo.x); sbox.lo[1] = fminf(sbox.lo[1], lo.y);
          sbox.lo[2] = fminf(sbox.lo[2], lo.z); sbox.hs = fmaxf(sbox.hs, lo.w);
          sbox.hi[0] = fmaxf(sbox.hi[0], hi.x); sbox.hi[1] = fmaxf(sbox.hi[1], hi.y);
          sbox.hi[2] = fmaxf(sbox.hi[2], hi.z);
        }
      } else {
        // the tile's real sources only (not the padding), as the precomputed boxes
        const int nvalid = (int)min((int64_t)TILE, s1 - sb);
        for (int r = lane; r < NPR; r += 32) {
          const float4 u = sP[buf][2 * r], v = sP[buf][2 * r + 1];
          if (2 * r < nvalid) sbox.add(u.x, u.z, v.x, v.z);
          if (2 * r + 1 < nvalid) sbox.add(u.y, u.w, v.y, v.w);
        }
        sbox.reduce();
      }
      const bool far_tile = all_far(tb, sbox);

#pragma unroll 1
      for (int g = 0; g < NPR; g += CG / 2) {
        // per-lane partial sums over the group: .x even sources, .y odd
        float2 sv[TPT][3], sd[TPT][3], sp[TPT][3];
        float sdv[TPT][3];
#pragma unroll
        for (int k = 0; k < TPT; ++k) {
#pragma unroll
          for (int m = 0; m < 3; ++m) {
            sv[k][m] = make_float2(0.f, 0.f); sd[k][m] = make_float2(0.f, 0.f); sp[k][m] = make_float2(0.f, 0.f);
            sdv[k][m] = 0.f;
          }
        }
        if (far_tile) {
          // B3 = X' x (-3 alpha_t), duplicated into both lanes (per group, so
          // that it is live only in this loop)
          float2 B3[TPT][3];
#pragma unroll
          for (int k = 0; k < TPT; ++k) {
            const float xr0 = X[k][0].x - rx, xr1 = X[k][1].x - ry, xr2 = X[k][2].x - rz;
            const float c0 = AT3[k][0].x, c1 = AT3[k][1].x, c2 = AT3[k][2].x;
            B3[k][0] = dup2(xr1 * c2 - xr2 * c1);
            B3[k][1] = dup2(xr2 * c0 - xr0 * c2);
            B3[k][2] = dup2(xr0 * c1 - xr1 * c0);
          }
#pragma unroll kF32Unroll
          for (int r = g; r < g + CG / 2; ++r) {
            const float4 pa = sP[buf][2 * r], pb = sP[buf][2 * r + 1];
            const float4 qa = sQ[buf][2 * r], qb = sQ[buf][2 * r + 1];
            const float4 na = sN[2 * r], nb = sN[2 * r + 1];
            const float2 px = make_float2(pa.x, pa.y), py = make_float2(pa.z, pa.w), pz = make_float2(pb.x, pb.y);
            const float2 ax = make_float2(qa.x, qa.y), ay = make_float2(qa.z, qa.w), az = make_float2(qb.x, qb.y);
            const float2 nx = make_float2(na.x, na.y), ny = make_float2(na.z, na.w), nz = make_float2(nb.x, nb.y);
#pragma unroll
            for (int k = 0; k < TPT; ++k) {
              // d = x_t - x_s (exact-rounded, as a subtraction)
              const float2 dx = __ffma2_rn(px, M1, X[k][0]);
              const float2 dy = __ffma2_rn(py, M1, X[k][1]);
              const float2 dz = __ffma2_rn(pz, M1, X[k][2]);
              float2 r2 = __fmul2_rn(dx, dx);
              r2 = __ffma2_rn(dy, dy, r2);
              r2 = __ffma2_rn(dz, dz, r2);
              // far limit: q' = r^3, F' = -3 r^5 (the -3 is in AT3 and B3), no diffusion
              const float2 ir = make_float2(fast_rsqrt(r2.x), fast_rsqrt(r2.y));
              const float2 A = __fmul2_rn(ir, ir);
              const float2 qq = __fmul2_rn(A, ir);
              const float2 qA = __fmul2_rn(qq, A);
              // sum q alpha_s and sum q n_s (the velocity is formed at the fold)
              sp[k][0] = __ffma2_rn(qq, ax, sp[k][0]);
              sp[k][1] = __ffma2_rn(qq, ay, sp[k][1]);
              sp[k][2] = __ffma2_rn(qq, az, sp[k][2]);
              sv[k][0] = __ffma2_rn(qq, nx, sv[k][0]);
              sv[k][1] = __ffma2_rn(qq, ny, sv[k][1]);
              sv[k][2] = __ffma2_rn(qq, nz, sv[k][2]);
              // F (alpha_t . w) d, alpha_t . w = alpha_s . (X' x alpha_t) + n_s . alpha_t
              float2 dot = __fmul2_rn(ax, B3[k][0]);
              dot = __ffma2_rn(ay, B3[k][1], dot);
              dot = __ffma2_rn(az, B3[k][2], dot);
              dot = __ffma2_rn(nx, AT3[k][0], dot);
              dot = __ffma2_rn(ny, AT3[k][1], dot);
              dot = __ffma2_rn(nz, AT3[k][2], dot);
              const float2 fd = __fmul2_rn(qA, dot);
              sd[k][0] = __ffma2_rn(fd, dx, sd[k][0]);
              sd[k][1] = __ffma2_rn(fd, dy, sd[k][1]);
              sd[k][2] = __ffma2_rn(fd, dz, sd[k][2]);
            }
          }
        } else if constexpr (TPT >= 2) {
          // Tiles with possible near pairs, shapes with two or more targets
          // per thread: every pair takes the closed form, two sources per
          // packed instruction (pair_terms_mid2: the mid formula, which beyond
          // u = 50 equals the far limit to within e^{-u/2}); lanes at u < 1,
          // the self pair among them, take the series.  Per pair: q (alpha_t x
          // alpha_s) for the stretching (nearly parallel neighbours along a
          // filament) and the diffusion v_t a_s - v_s a_t.  On the 1M ring
          // this is 1% faster than the scalar path below at 128 x 2 and
          // 256 x 2, and 2% slower at 256 x 1, which keeps the scalar path.
          float2 sdv2[TPT][3];
#pragma unroll
          for (int k = 0; k < TPT; ++k) {
#pragma unroll
            for (int m = 0; m < 3; ++m) sdv2[k][m] = make_float2(0.f, 0.f);
          }
#pragma unroll 1
          for (int r = g; r < g + CG / 2; ++r) {
            const float4 pa = sP[buf][2 * r], pb = sP[buf][2 * r + 1];
            const float4 qa = sQ[buf][2 * r], qb = sQ[buf][2 * r + 1];
            const float2 px = make_float2(pa.x, pa.y), py = make_float2(pa.z, pa.w), pz = make_float2(pb.x, pb.y);
            const float2 ph = make_float2(pb.z, pb.w);
            const float2 ax = make_float2(qa.x, qa.y), ay = make_float2(qa.z, qa.w), az = make_float2(qb.x, qb.y);
            const float2 av = make_float2(qb.z, qb.w);
            float2 lx = make_float2(0.f, 0.f), ly = lx, lz = lx;
            if constexpr (SPLIT) {
              const float4 la = sL[buf][2 * r], lb = sL[buf][2 * r + 1];
              lx = make_float2(la.x, la.y); ly = make_float2(la.z, la.w); lz = make_float2(lb.x, lb.y);
            }
#pragma unroll
            for (int k = 0; k < TPT; ++k) {
              float2 dx = __ffma2_rn(px, M1, X[k][0]);
              float2 dy = __ffma2_rn(py, M1, X[k][1]);
              float2 dz = __ffma2_rn(pz, M1, X[k][2]);
              if constexpr (SPLIT) {
                // the FP32 difference of nearby positions is exact; adding the
                // difference of the residuals restores the FP64 difference
                dx = __fadd2_rn(dx, __ffma2_rn(lx, M1, dup2(xl[k][0])));
                dy = __fadd2_rn(dy, __ffma2_rn(ly, M1, dup2(xl[k][1])));
                dz = __fadd2_rn(dz, __ffma2_rn(lz, M1, dup2(xl[k][2])));
              }
              float2 r2 = __fmul2_rn(dx, dx);
              r2 = __ffma2_rn(dy, dy, r2);
              r2 = __ffma2_rn(dz, dz, r2);
              const float2 s2 = __fadd2_rn(dup2(hst[k]), ph);
              PairTerms2 t = pair_terms_mid2(r2, s2);
              const bool nx = r2.x < s2.x, ny = r2.y < s2.y;  // u < 1
              if (__any_sync(0xffffffffu, nx || ny)) {
                if (nx) { const PairTerms<float> e = pair_terms_near(r2.x, s2.x); t.q.x = e.q; t.F.x = e.F; t.zd.x = e.zd; }
                if (ny) { const PairTerms<float> e = pair_terms_near(r2.y, s2.y); t.q.y = e.q; t.F.y = e.F; t.zd.y = e.zd; }
              }
              // pairs inside the far regime's bound count as full-formula pairs
              nfull += (fmaf(-kFarU, ph.x, r2.x) < h50[k]) + (fmaf(-kFarU, ph.y, r2.y) < h50[k]);
              // w = alpha_s x d (scalar: the negated operand is free)
              const float2 wx = make_float2(ay.x * dz.x - az.x * dy.x, ay.y * dz.y - az.y * dy.y);
              const float2 wy = make_float2(az.x * dx.x - ax.x * dz.x, az.y * dx.y - ax.y * dz.y);
              const float2 wz = make_float2(ax.x * dy.x - ay.x * dx.x, ax.y * dy.y - ay.y * dx.y);
              sv[k][0] = __ffma2_rn(t.q, wx, sv[k][0]);
              sv[k][1] = __ffma2_rn(t.q, wy, sv[k][1]);
              sv[k][2] = __ffma2_rn(t.q, wz, sv[k][2]);
              float2 dot = __fmul2_rn(dup2(at[k][0]), wx);
              dot = __ffma2_rn(dup2(at[k][1]), wy, dot);
              dot = __ffma2_rn(dup2(at[k][2]), wz, dot);
              const float2 fd = __fmul2_rn(t.F, dot);
              sd[k][0] = __ffma2_rn(fd, dx, sd[k][0]);
              sd[k][1] = __ffma2_rn(fd, dy, sd[k][1]);
              sd[k][2] = __ffma2_rn(fd, dz, sd[k][2]);
              const float2 cx = __ffma2_rn(dup2(at[k][1]), az, __fmul2_rn(dup2(-at[k][2]), ay));
              const float2 cy = __ffma2_rn(dup2(at[k][2]), ax, __fmul2_rn(dup2(-at[k][0]), az));
              const float2 cz = __ffma2_rn(dup2(at[k][0]), ay, __fmul2_rn(dup2(-at[k][1]), ax));
              sp[k][0] = __ffma2_rn(t.q, cx, sp[k][0]);
              sp[k][1] = __ffma2_rn(t.q, cy, sp[k][1]);
              sp[k][2] = __ffma2_rn(t.q, cz, sp[k][2]);
              const float2 VT = dup2(vt[k]);
              sdv2[k][0] = __ffma2_rn(t.zd, __ffma2_rn(av, dup2(-at[k][0]), __fmul2_rn(VT, ax)), sdv2[k][0]);
              sdv2[k][1] = __ffma2_rn(t.zd, __ffma2_rn(av, dup2(-at[k][1]), __fmul2_rn(VT, ay)), sdv2[k][1]);
              sdv2[k][2] = __ffma2_rn(t.zd, __ffma2_rn(av, dup2(-at[k][2]), __fmul2_rn(VT, az)), sdv2[k][2]);
            }
          }
#pragma unroll
          for (int k = 0; k < TPT; ++k) {
#pragma unroll
            for (int m = 0; m < 3; ++m) sdv[k][m] += sdv2[k][m].x + sdv2[k][m].y;
          }
        } else {
          // Tiles with possible near pairs: scalar, one source at a time,
          // accumulated into lane .x.
          auto one = [&](float sx, float sy, float sz, float shs, float qx, float qy, float qz, float qv, float lx,
                         float ly, float lz) {
#pragma unroll
            for (int k = 0; k < TPT; ++k) {
              float dx = X[k][0].x - sx, dy = X[k][1].x - sy, dz = X[k][2].x - sz;
              if constexpr (SPLIT) {
                // the FP32 difference of nearby positions is exact; adding the
                // difference of the residuals restores the FP64 difference
                dx += xl[k][0] - lx; dy += xl[k][1] - ly; dz += xl[k][2] - lz;
              }
              const float r2 = dx * dx + dy * dy + dz * dz;
              // far test r^2 >= 50 (hs_t + hs_s) as one FMA against the
              // target's precomputed 50 hs_t
              const bool near = fmaf(-kFarU, shs, r2) < h50[k];
              const float ir = fast_rsqrt(r2);
              const float A = ir * ir;
              float qq = A * ir;
              float FF = -3.0f * qq * A;
              // the full formula only when some lane of the warp needs it:
              // the vote keeps the common all-far case free of divergence
              if (__any_sync(0xffffffffu, near)) {
                if (near) {
                  const PairTerms<float> pt = pair_terms_near(r2, hst[k] + shs);
                  qq = pt.q; FF = pt.F;
                  // v_t a_s - v_s a_t per pair, so nearly equal strengths cancel
                  // before they are summed (as in DIFFUSION, interaction_utils.h:358-369)
                  sdv[k][0] += pt.zd * (vt[k] * qx - qv * at[k][0]);
                  sdv[k][1] += pt.zd * (vt[k] * qy - qv * at[k][1]);
                  sdv[k][2] += pt.zd * (vt[k] * qz - qv * at[k][2]);
                  ++nfull;
                }
              }
              const float wx = qy * dz - qz * dy;
              const float wy = qz * dx - qx * dz;
              const float wz = qx * dy - qy * dx;
              sv[k][0].x += qq * wx; sv[k][1].x += qq * wy; sv[k][2].x += qq * wz;
              const float fd = FF * (at[k][0] * wx + at[k][1] * wy + at[k][2] * wz);
              sd[k][0].x += fd * dx; sd[k][1].x += fd * dy; sd[k][2].x += fd * dz;
              // near tiles: q (alpha_t x alpha_s) per pair.  Along a filament the
              // neighbours' strengths are nearly parallel to alpha_t, and
              // alpha_t x (sum q alpha_s) would keep only the FP32 rounding of
              // the parallel part (2.3e-5 of max |dalpha| on a rotor tip vortex)
              sp[k][0].x += qq * (at[k][1] * qz - at[k][2] * qy);
              sp[k][1].x += qq * (at[k][2] * qx - at[k][0] * qz);
              sp[k][2].x += qq * (at[k][0] * qy - at[k][1] * qx);
            }
          };
#pragma unroll 1
          for (int r = g; r < g + CG / 2; ++r) {
            const float4 pa = sP[buf][2 * r], pb = sP[buf][2 * r + 1];
            const float4 qa = sQ[buf][2 * r], qb = sQ[buf][2 * r + 1];
            float4 la = make_float4(0.f, 0.f, 0.f, 0.f), lb = la;
            if constexpr (SPLIT) { la = sL[buf][2 * r]; lb = sL[buf][2 * r + 1]; }
            one(pa.x, pa.z, pb.x, pb.z, qa.x, qa.z, qb.x, qb.z, la.x, la.z, lb.x);
            one(pa.y, pa.w, pb.y, pb.w, qa.y, qa.w, qb.y, qb.w, la.y, la.w, lb.y);
          }
        }
#pragma unroll
        for (int k = 0; k < TPT; ++k) {
          float svs[3], sds[3], sps[3];
#pragma unroll
          for (int m = 0; m < 3; ++m) {
            svs[m] = sv[k][m].x + sv[k][m].y;
            sds[m] = sd[k][m].x + sd[k][m].y;
            sps[m] = sp[k][m].x + sp[k][m].y;
          }
          if (far_tile) {
            // velocity = (sum q alpha_s) x X' + sum q n_s
            const float xr0 = X[k][0].x - rx, xr1 = X[k][1].x - ry, xr2 = X[k][2].x - rz;
            const float n0 = svs[0], n1 = svs[1], n2 = svs[2];
            svs[0] = sps[1] * xr2 - sps[2] * xr1 + n0;
            svs[1] = sps[2] * xr0 - sps[0] * xr2 + n1;
            svs[2] = sps[0] * xr1 - sps[1] * xr0 + n2;
          }
          // da = sum q (alpha_t x alpha_s) + sum F (d.c) d + 2 nu sum z (v_t a_s - v_s a_t);
          // far tiles summed q alpha_s, near tiles q (alpha_t x alpha_s) itself
          float c0 = sps[0], c1 = sps[1], c2 = sps[2];
          if (far_tile) {
            c0 = at[k][1] * sps[2] - at[k][2] * sps[1];
            c1 = at[k][2] * sps[0] - at[k][0] * sps[2];
            c2 = at[k][0] * sps[1] - at[k][1] * sps[0];
          }
          const float ex = c0 + sds[0] + a.nu2 * sdv[k][0];
          const float ey = c1 + sds[1] + a.nu2 * sdv[k][1];
          const float ez = c2 + sds[2] + a.nu2 * sdv[k][2];
          two_sum_acc(vh[k][0], vl[k][0], svs[0]);
          two_sum_acc(vh[k][1], vl[k][1], svs[1]);
          two_sum_acc(vh[k][2], vl[k][2], svs[2]);
          two_sum_acc(dh[k][0], dl[k][0], ex);
          two_sum_acc(dh[k][1], dl[k][1], ey);
          two_sum_acc(dh[k][2], dl[k][2], ez);
        }
      }
      __syncthreads();
      buf ^= 1;
    }
    cp_async_wait<0>();
    const unsigned wsum = __reduce_add_sync(0xffffffffu, nfull);
    if (lane == 0 && wsum) atomicAdd(a.nfull, (unsigned long long)wsum);

#pragma unroll
    for (int k = 0; k < TPT; ++k) {
      const int64_t ti = t0 + tid + k * BLOCK;
      if (ti < tend) {
        double *o = a.partial + (int64_t)c * 6 * a.cap + ti;
#pragma unroll
        for (int m = 0; m < 3; ++m) {
          o[m * a.cap] = ((double)vh[k][m] + (double)vl[k][m]) * kInv4Pi;
          o[(3 + m) * a.cap] = ((double)dh[k][m] + (double)dl[k][m]) * kInv4Pi;
        }
      }
    }
  }
}

}  // namespace pgpu
