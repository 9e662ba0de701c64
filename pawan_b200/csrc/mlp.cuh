// Far-field correction network: 24 -> 128 -> 128 -> 128 -> 6, GELU (tanh
// form, Hendrycks & Gimpel 2016), BF16 tensor-core products with FP32
// accumulation, FP32 master weights, Adam.
//
// Training and the batch forward use one generic GEMM on the tcgen05 tensor
// cores (C = op(A) op(B), 128-row CTA tiles, accumulator in TMEM;
// mlp_tc.cuh) with fused epilogues (bias + GELU forward, GELU' backward,
// split-K accumulation for weight gradients).  Inference inside the
// far-field evaluation runs the whole network per warp on 16-row tiles with
// activations kept in registers: the FP32 accumulator fragment of one layer is
// the BF16 A fragment of the next (same thread-to-element map), so hidden
// activations never touch shared memory.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace pgpu {

constexpr int kIn = 24, kInPad = 32, kHid = 128, kOut = 6, kOutPad = 8;
// Parameter layout (FP32): W1[32][128] (rows >= 24 zero), b1[128], W2[128][128],
// b2[128], W3[128][128], b3[128], W4[128][8] (cols >= 6 zero), b4[8].
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kInPad * kHid, kOffW2 = kOffB1 + kHid, kOffB2 = kOffW2 + kHid * kHid,
              kOffW3 = kOffB2 + kHid, kOffB3 = kOffW3 + kHid * kHid, kOffW4 = kOffB3 + kHid,
              kOffB4 = kOffW4 + kHid * kOutPad, kNumParams = kOffB4 + kOutPad;

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
  return *reinterpret_cast<const uint32_t *>(&v);
}

// D = A (16x16 bf16, row) * B (16x8 bf16, col) + C, FP32 accumulate.
__device__ __forceinline__ void mma_16816(float *d, const uint32_t *a, const uint32_t *b) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

__device__ __forceinline__ float gelu_f(float z) {
  const float t = tanhf(0.7978845608028654f * (z + 0.044715f * z * z * z));
  return 0.5f * z * (1.f + t);
}
__device__ __forceinline__ float gelu_grad(float z) {
  const float u = 0.7978845608028654f * (z + 0.044715f * z * z * z);
  const float t = tanhf(u);
  return 0.5f * (1.f + t) + 0.5f * z * (1.f - t * t) * 0.7978845608028654f * (1.f + 3.f * 0.044715f * z * z);
}
__device__ __forceinline__ float tanh_fast(float x) {
  float y;
  asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float gelu_fast(float z) {
  return 0.5f * z * (1.f + tanh_fast(0.7978845608028654f * (z + 0.044715f * z * z * z)));
}

// ---------------------------------------------------------------- generic GEMM
enum GemmEpi { kEpiStore = 0, kEpiBiasGelu = 1, kEpiGeluGrad = 2, kEpiAtomic = 3, kEpiBias = 4 };

struct GemmArgs {
  const float *A;  // element (m,k) = transA ? A[k*lda + m] : A[m*lda + k]
  const float *B;  // element (k,n) = transB ? B[n*ldb + k] : B[k*ldb + n]
  float *C;        // C[m*ldc + n]
  float *H;        // kEpiBiasGelu: GELU(C) also stored here (same ld)
  const float *bias;  // [N]
  const float *Z;     // kEpiGeluGrad: C = acc * GELU'(Z[m*ldc + n])
  int M, N, K, lda, ldb, ldc;
  int transA, transB, epi;
  int ksplit;  // K range per blockIdx.z
};

__global__ void colsum_kernel(const float *X, int M, int N, int ld, float *out) {
  const int n = blockIdx.x;
  float s = 0.f;
  for (int m = threadIdx.x; m < M; m += blockDim.x) s += X[(int64_t)m * ld + n];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  __shared__ float red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += red[k];
    out[n] += t;
  }
}

// Mean-squared error over the kOut outputs and its gradient dY (padded ld 8):
// loss = sum (y - t)^2 / (rows * kOut).  loss_acc (double) accumulates the sum.
__global__ void mse_kernel(const float *Y, const float *T, int rows, float *dY, double *loss_acc) {
  double s = 0.0;
  const float scale = 2.f / ((float)rows * kOut);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < rows * kOutPad; i += gridDim.x * blockDim.x) {
    const int r = i / kOutPad, c = i % kOutPad;
    float d = 0.f;
    if (c < kOut) {
      d = Y[i] - T[(int64_t)r * kOut + c];
      s += (double)d * d;
    }
    dY[i] = scale * d;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss_acc, s);
}

// Adam (Kingma & Ba) with bias correction; padded rows/cols of W1/W4/b4 stay 0.
__global__ void adam_kernel(float *p, const float *g, float *m, float *v, int n, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const bool pad = (i < kOffB1 && (i / kHid) >= kIn) || (i >= kOffW4 && i < kOffB4 && (i - kOffW4) % kOutPad >= kOut) ||
                     (i >= kOffB4 && i - kOffB4 >= kOut);
    if (pad) continue;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// ---------------------------------------------------------------- warp inference
// Weights for inference, BF16 and transposed (WT[n][k]) so that a B fragment
// (two consecutive k of one n) is one 32-bit shared-memory load; rows padded by
// 8 elements against bank conflicts.  Built once by mlp_pack_kernel.
struct MlpPacked {
  __nv_bfloat16 w1t[kHid][kInPad + 8];
  __nv_bfloat16 w2t[kHid][kHid + 8];
  __nv_bfloat16 w3t[kHid][kHid + 8];
  __nv_bfloat16 w4t[kOutPad][kHid + 8];
  float b1[kHid], b2[kHid], b3[kHid], b4[kOutPad];
};

__global__ void mlp_pack_kernel(const float *p, MlpPacked *out) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kHid * kHid; i += gridDim.x * blockDim.x) {
    const int k = i / kHid, n = i % kHid;  // W[k][n]
    out->w2t[n][k] = __float2bfloat16_rn(p[kOffW2 + i]);
    out->w3t[n][k] = __float2bfloat16_rn(p[kOffW3 + i]);
    if (k < kInPad) out->w1t[n][k] = __float2bfloat16_rn(p[kOffW1 + k * kHid + n]);
    if (n < kOutPad) out->w4t[n][k] = __float2bfloat16_rn(p[kOffW4 + k * kOutPad + n]);
    if (k == 0) {
      out->b1[n] = p[kOffB1 + n];
      out->b2[n] = p[kOffB2 + n];
      out->b3[n] = p[kOffB3 + n];
      if (n < kOutPad) out->b4[n] = p[kOffB4 + n];
    }
  }
}

__device__ __forceinline__ void gelu_pack(const float (*c)[4], uint32_t (*a)[4]) {
  // accumulator n-tiles 2kk, 2kk+1 are exactly the A fragment of k-step kk
#pragma unroll
  for (int kk = 0; kk < kHid / 16; ++kk) {
    a[kk][0] = pack_bf16(gelu_fast(c[2 * kk][0]), gelu_fast(c[2 * kk][1]));
    a[kk][1] = pack_bf16(gelu_fast(c[2 * kk][2]), gelu_fast(c[2 * kk][3]));
    a[kk][2] = pack_bf16(gelu_fast(c[2 * kk + 1][0]), gelu_fast(c[2 * kk + 1][1]));
    a[kk][3] = pack_bf16(gelu_fast(c[2 * kk + 1][2]), gelu_fast(c[2 * kk + 1][3]));
  }
}

template <int LD>
__device__ __forceinline__ void dense_layer(const __nv_bfloat16 (*wt)[LD], const float *bias, const uint32_t (*a)[4],
                                            float (*c)[4], int gid, int tig) {
#pragma unroll
  for (int nt = 0; nt < kHid / 8; ++nt) {
    const float b0 = bias[nt * 8 + tig * 2], b1 = bias[nt * 8 + tig * 2 + 1];
    c[nt][0] = b0; c[nt][1] = b1; c[nt][2] = b0; c[nt][3] = b1;
#pragma unroll
    for (int kk = 0; kk < kHid / 16; ++kk) {
      uint32_t b[2];
      b[0] = *reinterpret_cast<const uint32_t *>(&wt[nt * 8 + gid][kk * 16 + tig * 2]);
      b[1] = *reinterpret_cast<const uint32_t *>(&wt[nt * 8 + gid][kk * 16 + tig * 2 + 8]);
      mma_16816(c[nt], a[kk], b);
    }
  }
}

// The network on 16 rows: F[16][kInPad + 8] BF16 features in shared memory ->
// O[16][kOutPad] FP32 outputs in shared memory.  Called by a full warp.
__device__ __forceinline__ void mlp_tile16(const MlpPacked &W, const __nv_bfloat16 (*F)[kInPad + 8],
                                           float (*O)[kOutPad], int lane) {
  const int gid = lane >> 2, tig = lane & 3;
  uint32_t a[kHid / 16][4];
  float c[kHid / 8][4];
  // layer 1 (K = 32)
  uint32_t a1[2][4];
#pragma unroll
  for (int ks = 0; ks < 2; ++ks) {
    a1[ks][0] = *reinterpret_cast<const uint32_t *>(&F[gid][ks * 16 + tig * 2]);
    a1[ks][1] = *reinterpret_cast<const uint32_t *>(&F[gid + 8][ks * 16 + tig * 2]);
    a1[ks][2] = *reinterpret_cast<const uint32_t *>(&F[gid][ks * 16 + tig * 2 + 8]);
    a1[ks][3] = *reinterpret_cast<const uint32_t *>(&F[gid + 8][ks * 16 + tig * 2 + 8]);
  }
#pragma unroll
  for (int nt = 0; nt < kHid / 8; ++nt) {
    const float b0 = W.b1[nt * 8 + tig * 2], b1 = W.b1[nt * 8 + tig * 2 + 1];
    c[nt][0] = b0; c[nt][1] = b1; c[nt][2] = b0; c[nt][3] = b1;
#pragma unroll
    for (int ks = 0; ks < 2; ++ks) {
      uint32_t b[2];
      b[0] = *reinterpret_cast<const uint32_t *>(&W.w1t[nt * 8 + gid][ks * 16 + tig * 2]);
      b[1] = *reinterpret_cast<const uint32_t *>(&W.w1t[nt * 8 + gid][ks * 16 + tig * 2 + 8]);
      mma_16816(c[nt], a1[ks], b);
    }
  }
  gelu_pack(c, a);
  dense_layer<kHid + 8>(W.w2t, W.b2, a, c, gid, tig);
  gelu_pack(c, a);
  dense_layer<kHid + 8>(W.w3t, W.b3, a, c, gid, tig);
  gelu_pack(c, a);
  // output layer (N = 8)
  float o[4] = {W.b4[tig * 2], W.b4[tig * 2 + 1], W.b4[tig * 2], W.b4[tig * 2 + 1]};
#pragma unroll
  for (int kk = 0; kk < kHid / 16; ++kk) {
    uint32_t b[2];
    b[0] = *reinterpret_cast<const uint32_t *>(&W.w4t[gid][kk * 16 + tig * 2]);
    b[1] = *reinterpret_cast<const uint32_t *>(&W.w4t[gid][kk * 16 + tig * 2 + 8]);
    mma_16816(o, a[kk], b);
  }
  O[gid][tig * 2] = o[0];
  O[gid][tig * 2 + 1] = o[1];
  O[gid + 8][tig * 2] = o[2];
  O[gid + 8][tig * 2 + 1] = o[3];
}

// The fused inference path on given rows (one warp per 16-row tile): X[rows][24] -> Y[rows][6].
__global__ void __launch_bounds__(128) mlp_infer_kernel(const MlpPacked *Wg, const float *X, int rows, float *Y) {
  extern __shared__ __align__(16) unsigned char dyn[];
  MlpPacked &W = *reinterpret_cast<MlpPacked *>(dyn);
  __nv_bfloat16 (*F)[kInPad + 8] = reinterpret_cast<__nv_bfloat16 (*)[kInPad + 8]>(dyn + sizeof(MlpPacked));
  float (*O)[kOutPad] = reinterpret_cast<float (*)[kOutPad]>(dyn + sizeof(MlpPacked) + 4 * 16 * (kInPad + 8) * 2);
  const uint4 *src = reinterpret_cast<const uint4 *>(Wg);
  uint4 *dst = reinterpret_cast<uint4 *>(dyn);
  for (int i = threadIdx.x; i < (int)(sizeof(MlpPacked) / 16); i += blockDim.x) dst[i] = src[i];
  __syncthreads();
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  auto Fw = F + 16 * w;
  auto Ow = O + 16 * w;
  for (int t0 = (blockIdx.x * 4 + w) * 16; t0 < rows; t0 += gridDim.x * 4 * 16) {
    for (int e = lane; e < 16 * kInPad; e += 32) {
      const int r = e / kInPad, c = e % kInPad;
      const int row = t0 + r;
      Fw[r][c] = __float2bfloat16_rn(c < kIn && row < rows ? X[(int64_t)row * kIn + c] : 0.f);
    }
    __syncwarp();
    mlp_tile16(W, Fw, Ow, lane);
    __syncwarp();
    for (int e = lane; e < 16 * kOut; e += 32) {
      const int r = e / kOut, c = e % kOut;
      if (t0 + r < rows) Y[(int64_t)(t0 + r) * kOut + c] = Ow[r][c];
    }
    __syncwarp();
  }
}

// Gathers batch rows of the dataset: X[b][0..31] (features, zero padded), T[b][0..5].
__global__ void gather_batch_kernel(const float *Xd, const float *Td, const int *rows, int batch, float *X, float *T) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < batch * kInPad; i += gridDim.x * blockDim.x) {
    const int b = i / kInPad, c = i % kInPad;
    const int r = rows[b];
    X[i] = c < kIn ? Xd[(int64_t)r * kIn + c] : 0.f;
    if (c < kOut) T[(int64_t)b * kOut + c] = Td[(int64_t)r * kOut + c];
  }
}

}  // namespace pgpu

#include "mlp_tc.cuh"
