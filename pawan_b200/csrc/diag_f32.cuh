// FP32 body of the quadratic diagnostics (helicity, KE, KEF) for the Gaussian
// kernel: the terms and work decomposition of diag_pair_kernel (kernels.cuh),
// with the arithmetic layout of the FP32 rate kernel (pair_f32.cuh):
//
// * Sources are staged pair-interleaved and processed two at a time with the
//   packed FP32 instructions of sm_100 (lane .x even source, .y odd source).
// * A tile whose source box is at least sqrt(50 (hs_t + hs_s)) from the warp's
//   target box (all_far) takes the helicity's far limit q' = 1/rho^3 with no
//   per-pair test; other tiles run the scalar per-pair code of the generic
//   body, with its warp vote for the mid/series terms.
// * In far tiles the helicity's d . (a_t x a_s) is formed from positions
//   relative to the tile's first source, ref: with X' = x_t - ref,
//   p' = x_s - ref, B = X' x a_t (per target) and m_s = a_s x p' (per
//   source, staged once per tile), d . (a_t x a_s) = a_s . B - a_t . m_s:
//   6 operations instead of 9.
// Per unordered pair in a far tile: 35 FP32 operations (packed over two
// sources) and two reciprocal square roots.
#pragma once

namespace pgpu {

template <int BLOCK>
__device__ __forceinline__ void diag_body_f32(const DiagArgs<float> &a) {
  constexpr int NPR = BLOCK / 2;  // source pairs per tile
  __shared__ __align__(16) float4 sP[BLOCK];
  __shared__ __align__(16) float4 sQ[BLOCK];
  __shared__ __align__(16) float4 sM[BLOCK];  // m_s = a_s x (x_s - ref), pair-interleaved like sP
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
    const int64_t tend = pe.off + pe.toff + pe.tn;   // end of the (owned) targets
    const int64_t tlo = pe.off + pe.toff + tile * BLOCK;  // first target of the tile
    const int64_t t = min(tlo + tid, tend - 1);
    const bool valid = tlo + tid < tend;
    // sources above the tile's first target only (s > t is tested per pair
    // while a tile can still hold s <= t), up to the end of the system
    const int64_t s0 = max(pe.off + (int64_t)c * pe.chunk, tlo);
    const int64_t s1 = min(pe.off + (int64_t)c * pe.chunk + pe.chunk, pe.off + pe.n);
    const float4 pt = a.P[t], qt = a.Q[t];
    const float h50 = kFarU * pt.w;
    const float2 X0 = dup2(pt.x), X1 = dup2(pt.y), X2 = dup2(pt.z), HT = dup2(pt.w);
    const float2 A0 = dup2(qt.x), A1 = dup2(qt.y), A2 = dup2(qt.z);
    const float2 NA0 = dup2(-qt.x), NA1 = dup2(-qt.y), NA2 = dup2(-qt.z);
    WarpBox tb;
    tb.init();
    tb.add(pt.x, pt.y, pt.z, pt.w);
    tb.reduce();
    double h = 0, ke = 0, kef = 0;
    for (int64_t sb = s0; sb < s1; sb += BLOCK) {
      __syncthreads();
      {
        const int64_t j = sb + tid;
        const float4 p = j < s1 ? a.P[j] : pad_P<float>();
        const float4 q = j < s1 ? a.Q[j] : pad_Q<float>();
        float *dp = reinterpret_cast<float *>(sP) + (tid >> 1) * 8 + (tid & 1);
        float *dq = reinterpret_cast<float *>(sQ) + (tid >> 1) * 8 + (tid & 1);
        dp[0] = p.x; dp[2] = p.y; dp[4] = p.z; dp[6] = p.w;
        dq[0] = q.x; dq[2] = q.y; dq[4] = q.z; dq[6] = q.w;
      }
      __syncthreads();
      const float *fp = reinterpret_cast<const float *>(sP);
      const float rx = fp[0], ry = fp[2], rz = fp[4];
      {
        const float *fq = reinterpret_cast<const float *>(sQ);
        const int e = (tid >> 1) * 8 + (tid & 1);
        const float px = fp[e] - rx, py = fp[e + 2] - ry, pz = fp[e + 4] - rz;
        const float ax = fq[e], ay = fq[e + 2], az = fq[e + 4];
        float *fm = reinterpret_cast<float *>(sM);
        fm[e] = ay * pz - az * py;
        fm[e + 2] = az * px - ax * pz;
        fm[e + 4] = ax * py - ay * px;
      }
      __syncthreads();
      const int cnt = (int)min((int64_t)BLOCK, s1 - sb);
      const bool diag = sb <= tlo + BLOCK - 1;  // the tile may still see s <= t
      WarpBox sbox;
      sbox.init();
      for (int r = lane; r < NPR; r += 32) {
        const float4 u = sP[2 * r], v = sP[2 * r + 1];
        sbox.add(u.x, u.z, v.x, v.z);
        sbox.add(u.y, u.w, v.y, v.w);
      }
      sbox.reduce();
      const bool far_tile = !diag && all_far(tb, sbox);
      float2 hh = make_float2(0.f, 0.f), kk = make_float2(0.f, 0.f), kf = make_float2(0.f, 0.f);
      if (far_tile) {
        // B = X' x a_t, duplicated into both lanes
        const float xr0 = pt.x - rx, xr1 = pt.y - ry, xr2 = pt.z - rz;
        const float2 B0 = dup2(xr1 * qt.z - xr2 * qt.y);
        const float2 B1 = dup2(xr2 * qt.x - xr0 * qt.z);
        const float2 B2 = dup2(xr0 * qt.y - xr1 * qt.x);
        // pad sources have zero strength: every term they add is zero
#pragma unroll 2
        for (int r = 0; r < NPR; ++r) {
          const float4 pa = sP[2 * r], pb = sP[2 * r + 1];
          const float4 qa = sQ[2 * r], qb = sQ[2 * r + 1];
          const float4 ma = sM[2 * r], mb = sM[2 * r + 1];
          const float2 px = make_float2(pa.x, pa.y), py = make_float2(pa.z, pa.w), pz = make_float2(pb.x, pb.y);
          const float2 hs = make_float2(pb.z, pb.w);
          const float2 ax = make_float2(qa.x, qa.y), ay = make_float2(qa.z, qa.w), az = make_float2(qb.x, qb.y);
          const float2 mx = make_float2(ma.x, ma.y), my = make_float2(ma.z, ma.w), mz = make_float2(mb.x, mb.y);
          const float2 dx = __ffma2_rn(px, M1, X0);
          const float2 dy = __ffma2_rn(py, M1, X1);
          const float2 dz = __ffma2_rn(pz, M1, X2);
          float2 r2 = __fmul2_rn(dx, dx);
          r2 = __ffma2_rn(dy, dy, r2);
          r2 = __ffma2_rn(dz, dz, r2);
          const float2 s2 = __fadd2_rn(HT, hs);
          const float2 rs = __fadd2_rn(r2, s2);
          // helicity: far-limit q' = 1/rho^3, d . (a_t x a_s) = a_s . B - a_t . m_s
          const float2 irr = make_float2(fast_rsqrt(r2.x), fast_rsqrt(r2.y));
          const float2 kq = __fmul2_rn(__fmul2_rn(irr, irr), irr);
          float2 dc = __fmul2_rn(ax, B0);
          dc = __ffma2_rn(ay, B1, dc);
          dc = __ffma2_rn(az, B2, dc);
          dc = __ffma2_rn(mx, NA0, dc);
          dc = __ffma2_rn(my, NA1, dc);
          dc = __ffma2_rn(mz, NA2, dc);
          hh = __ffma2_rn(kq, dc, hh);
          // KE and KEF with (rho^2 + s^2)^-1.5
          const float2 ir = make_float2(fast_rsqrt(rs.x), fast_rsqrt(rs.y));
          const float2 ir3 = __fmul2_rn(__fmul2_rn(ir, ir), ir);
          float2 aa = __fmul2_rn(ax, A0);
          aa = __ffma2_rn(ay, A1, aa);
          aa = __ffma2_rn(az, A2, aa);
          float2 dat = __fmul2_rn(dx, A0);
          dat = __ffma2_rn(dy, A1, dat);
          dat = __ffma2_rn(dz, A2, dat);
          float2 das = __fmul2_rn(dx, ax);
          das = __ffma2_rn(dy, ay, das);
          das = __ffma2_rn(dz, az, das);
          const float2 e = __ffma2_rn(__ffma2_rn(s2, dup2(2.f), r2), aa, __fmul2_rn(dat, das));
          kk = __ffma2_rn(e, ir3, kk);
          kf = __ffma2_rn(__fmul2_rn(__ffma2_rn(s2, dup2(1.5f), r2), aa), ir3, kf);
        }
        hh = __fmul2_rn(hh, M1);  // the generic body subtracts q d.(a_t x a_s)
      } else {
        // scalar per-pair code of the generic body, into lane .x
        for (int jj = 0; jj < cnt; ++jj) {
          const bool use = !diag || sb + jj > t;
          const int e = (jj >> 1) * 8 + (jj & 1);
          const float *fq = reinterpret_cast<const float *>(sQ);
          const float sx = fp[e], sy = fp[e + 2], sz = fp[e + 4], shs = fp[e + 6];
          const float qx = fq[e], qy = fq[e + 2], qz = fq[e + 4];
          const float dx = pt.x - sx, dy = pt.y - sy, dz = pt.z - sz;
          const float r2 = dx * dx + dy * dy + dz * dz;
          const float s2 = pt.w + shs;
          const bool near = fmaf(-kFarU, shs, r2) < h50;
          const float irr = fast_rsqrt(r2);
          float kq = irr * irr * irr;
          if (__any_sync(0xffffffffu, near && use)) {
            if (near && use) kq = pair_terms_near(r2, s2).q;
          }
          const float cx = qt.y * qz - qt.z * qy, cy = qt.z * qx - qt.x * qz, cz = qt.x * qy - qt.y * qx;
          const float aa = qt.x * qx + qt.y * qy + qt.z * qz;
          const float dat = dx * qt.x + dy * qt.y + dz * qt.z;
          const float das = dx * qx + dy * qy + dz * qz;
          const float ir = fast_rsqrt(r2 + s2);
          const float ir3 = ir * ir * ir;
          if (use) {
            hh.x -= kq * (dx * cx + dy * cy + dz * cz);
            kk.x += ((r2 + 2.f * s2) * aa + dat * das) * ir3;
            kf.x += (r2 + 1.5f * s2) * aa * ir3;
          }
        }
      }
      h += (double)hh.x + (double)hh.y;
      ke += (double)kk.x + (double)kk.y;
      kef += (double)kf.x + (double)kf.y;
    }
    if (valid) {
      // doubled: each unordered pair was summed once
      double *o = a.partial + (int64_t)c * 6 * a.cap + t;
      o[0] = h * (2.0 * kInv4Pi);
      o[a.cap] = ke * (2.0 * kInv4Pi * 0.25);      // 1/(16 pi)
      o[2 * a.cap] = kef * (2.0 * kInv4Pi * 0.5);  // 1/(8 pi)
    }
  }
}

}  // namespace pgpu
