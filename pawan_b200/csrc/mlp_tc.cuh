// Tensor-core GEMM of the far-field network's training and batch forward on
// the fifth-generation tensor cores of sm_100a: tcgen05.mma (kind::f16, BF16
// operands, FP32 accumulation) with the accumulator in tensor memory (TMEM).
//
// C = op(A) op(B) with the operand and epilogue conventions of GemmArgs
// (mlp.cuh).  One CTA of 128 threads computes a 128 x BN tile of C over its
// K range (blockIdx.z splits K for the weight gradients):
//
//   * per K chunk of 64, all threads convert their share of op(A) (128 x 64)
//     and op(B) (BN x 64) from FP32 to BF16 into shared memory, in the
//     no-swizzle K-major layout of the tensor cores: 8 x 8 element core
//     matrices of 128 contiguous bytes, stacked along M (or N) every 128 B
//     and along K every 16 MN-rows' worth;
//   * one thread issues the chunk's four 128 x BN x 16 MMAs and commits them
//     to an mbarrier, which every thread waits on (a bounded wait) before the
//     buffers are refilled;
//   * the epilogue reads the accumulator from TMEM (each warp the 32 lanes =
//     rows it may access, 16 columns per tcgen05.ld), applies the fused
//     epilogue and stores FP32 to global memory.
//
// The MLP's products are small (K, N <= 128; 2 GFLOP per 65536-row layer),
// so these launches are bound by the FP32 operand traffic, not by the tensor
// cores.  No cluster, no TMA and no multicast.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace pgpu {

constexpr int kTcBM = 128;  // rows of C per CTA (the MMA's M)
constexpr int kTcBK = 64;   // K per shared-memory chunk (four MMAs of K = 16)
constexpr unsigned kTcSpinLimit = 1u << 26;  // polls of the MMA mbarrier before giving up

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor of a no-swizzle K-major operand: start
// address, leading byte offset (between core matrices adjacent in K), stride
// byte offset (between core matrices adjacent in M / N), all in 16-byte
// units, and the descriptor version of sm_100 (bit 46).
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

// Instruction descriptor of kind::f16: FP32 accumulator (bits 4-5 = 1), BF16
// A and B (bits 7-9 = 1, 10-12 = 1), both K-major, N / 8 at bits 17-22, M / 16
// at bits 24-28.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int m, int n) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(m >> 4) << 24);
}

__device__ __forceinline__ void tc_mma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void tc_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(mbar), "r"(count) : "memory");
}

// Waits for the phase `parity` of the mbarrier to complete, at most
// kTcSpinLimit polls; false if the limit was reached.
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (unsigned i = 0; i < kTcSpinLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 32 lanes x 16 columns of FP32 from TMEM: thread `lane` of the warp gets row
// (lane quadrant of the warp) + lane, columns taddr.col .. +15.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
  for (int j = 0; j < 16; ++j) v[j] = __uint_as_float(r[j]);
}

// Byte offset of element (r, k) of a no-swizzle tile with `rows` rows (a
// multiple of 8) and 64 columns of BF16, in core matrices of 8 x 8 elements
// (128 contiguous bytes) stacked along the rows every 128 B and along K every
// rows x 16 B.  K-major: a core matrix row holds 8 consecutive k of one r;
// MN-major: 8 consecutive r of one k.  The descriptors of both take the same
// offsets (LBO = rows x 16 B between K groups, SBO = 128 B between row groups).
__device__ __forceinline__ int kmajor_off(int r, int k, int rows) {
  return (r & 7) * 16 + (r >> 3) * 128 + (k >> 3) * (rows * 16) + (k & 7) * 2;
}
__device__ __forceinline__ int mnmajor_off(int r, int k, int rows) {
  return (k & 7) * 16 + (r >> 3) * 128 + (k >> 3) * (rows * 16) + (r & 7) * 2;
}

// Eight consecutive FP32 values of a row of `src` (leading dimension ld)
// starting at column c, zero where the row or a column is out of range
// (vector loads when the run is whole and 16-byte aligned), as BF16.
__device__ __forceinline__ uint4 load8_bf16(const float *src, int64_t ld, int row, int nrows, int c, int ncols) {
  float v[8];
  const float *p = src + (int64_t)row * ld + c;
  if (row < nrows && c + 8 <= ncols && ((reinterpret_cast<uintptr_t>(p) & 15) == 0)) {
    const float4 a = *reinterpret_cast<const float4 *>(p), b = *reinterpret_cast<const float4 *>(p + 4);
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w; v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
  } else {
#pragma unroll
    for (int j = 0; j < 8; ++j) v[j] = (row < nrows && c + j < ncols) ? p[j] : 0.f;
  }
  uint4 o;
  o.x = pack_bf16(v[0], v[1]);
  o.y = pack_bf16(v[2], v[3]);
  o.z = pack_bf16(v[4], v[5]);
  o.w = pack_bf16(v[6], v[7]);
  return o;
}

// Dynamic shared memory of a CTA: the two operand tiles, padded so that at
// most four CTAs share an SM and their TMEM allocations (128 columns each)
// always fit the SM's 512 columns.
template <int BN> constexpr size_t gemm_tc_smem() { return 56 * 1024; }

template <int BN>
__global__ void __launch_bounds__(128) gemm_tc_kernel(GemmArgs g, int *err) {
  static_assert(BN % 16 == 0 && BN >= 16 && BN <= 128, "MMA N for M = 128");
  static_assert((kTcBM + BN) * kTcBK * 2 <= gemm_tc_smem<BN>(), "operand tiles fit the shared memory");
  constexpr int kCols = BN < 32 ? 32 : BN;  // TMEM allocation: a power of two >= 32 columns
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  unsigned char *sA = tc_smem;                       // 128 x 64 BF16
  unsigned char *sB = tc_smem + kTcBM * kTcBK * 2;   // BN x 64 BF16
  __shared__ __align__(8) unsigned long long s_mbar;
  __shared__ uint32_t s_tmem;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * kTcBM, n0 = blockIdx.x * BN;
  const int kz0 = blockIdx.z * g.ksplit, kz1 = min(g.K, kz0 + g.ksplit);
  const uint32_t mbar = smem_u32(&s_mbar);
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(&s_tmem)),
                 "r"(kCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  if (tid == 0) mbar_init(mbar, 1);
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  const uint32_t tmem = s_tmem;
  // Each operand is staged in the major order of its global layout, 16 bytes
  // (8 BF16) per store: op(A) is K-major unless A is transposed (then its M
  // run is contiguous: MN-major, idesc bit 15); op(B) is K-major when B is
  // transposed, else N-major (idesc bit 16).
  const uint32_t idesc =
      umma_idesc_bf16(kTcBM, BN) | ((g.transA ? 1u : 0u) << 15) | ((g.transB ? 0u : 1u) << 16);
  uint32_t phase = 0;
  bool ok = true;
  int issued = 0;
  for (int k0 = kz0; k0 < kz1; k0 += kTcBK) {
    const int kc = min(kTcBK, kz1 - k0);
    // op(A) tile, 1024 runs of 8: consecutive threads take consecutive runs
    // along the contiguous global dimension
    for (int i = tid; i < kTcBM * kTcBK / 8; i += 128) {
      if (!g.transA) {
        const int m = i >> 3, kg = i & 7;  // A[m][k], k contiguous
        *reinterpret_cast<uint4 *>(sA + kmajor_off(m, 8 * kg, kTcBM)) =
            load8_bf16(g.A, g.lda, m0 + m, g.M, k0 + 8 * kg, kz1);
      } else {
        const int k = i >> 4, mg = i & 15;  // A[k][m], m contiguous
        *reinterpret_cast<uint4 *>(sA + mnmajor_off(8 * mg, k, kTcBM)) =
            load8_bf16(g.A, g.lda, k0 + k, kz1, m0 + 8 * mg, g.M);
      }
    }
    for (int i = tid; i < BN * kTcBK / 8; i += 128) {
      if (g.transB) {
        const int n = i >> 3, kg = i & 7;  // B[n][k], k contiguous
        *reinterpret_cast<uint4 *>(sB + kmajor_off(n, 8 * kg, BN)) =
            load8_bf16(g.B, g.ldb, n0 + n, g.N, k0 + 8 * kg, kz1);
      } else {
        const int k = i / (BN / 8), ng = i % (BN / 8);  // B[k][n], n contiguous
        *reinterpret_cast<uint4 *>(sB + mnmajor_off(8 * ng, k, BN)) =
            load8_bf16(g.B, g.ldb, k0 + k, kz1, n0 + 8 * ng, g.N);
      }
    }
    // the generic-proxy stores must be visible to the tensor cores' async proxy
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
      const int steps = (kc + 15) / 16;
      for (int s = 0; s < steps; ++s) {
        const uint64_t ad = umma_desc(smem_u32(sA) + s * 2 * (kTcBM * 16), kTcBM * 16, 128);
        const uint64_t bd = umma_desc(smem_u32(sB) + s * 2 * (BN * 16), BN * 16, 128);
        tc_mma(tmem, ad, bd, idesc, issued > 0 ? 1u : 0u);
        ++issued;
      }
      tc_commit(mbar);
    }
    // every thread waits for the chunk's MMAs before the buffers are refilled
    // (and before the accumulator is read); a wait that gives up stops the
    // whole CTA (the decision is uniform)
    if (!mbar_wait(mbar, phase)) ok = false;
    phase ^= 1u;
    if (__syncthreads_or(!ok)) {
      ok = false;
      break;
    }
  }
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
  } else {
    // warp w reads TMEM lanes 32 w .. 32 w + 31 = rows of C
    const int m = m0 + warp * 32 + lane;
    const bool any_k = kz1 > kz0;
#pragma unroll 1
    for (int c = 0; c < BN; c += 16) {
      float v[16];
      if (any_k) {
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c, v);
      } else {
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] = 0.f;
      }
      if (m < g.M) {
        const int nb = n0 + c;
        const int64_t o0 = (int64_t)m * g.ldc + nb;
        if (g.epi == kEpiAtomic) {
#pragma unroll
          for (int j = 0; j < 16; ++j)
            if (nb + j < g.N) atomicAdd(g.C + o0 + j, v[j]);
        } else {
          float h[16];
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int n = nb + j < g.N ? nb + j : g.N - 1;  // clamped: columns past N are not stored
            if (g.epi == kEpiBias || g.epi == kEpiBiasGelu) v[j] += g.bias[n];
            if (g.epi == kEpiBiasGelu) h[j] = gelu_f(v[j]);
            if (g.epi == kEpiGeluGrad) v[j] *= gelu_grad(g.Z[(int64_t)m * g.ldc + n]);
          }
          const bool vec = nb + 16 <= g.N && ((reinterpret_cast<uintptr_t>(g.C + o0) & 15) == 0) &&
                           (g.epi != kEpiBiasGelu || ((reinterpret_cast<uintptr_t>(g.H + o0) & 15) == 0));
          if (vec) {
#pragma unroll
            for (int j = 0; j < 16; j += 4) {
              *reinterpret_cast<float4 *>(g.C + o0 + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
              if (g.epi == kEpiBiasGelu)
                *reinterpret_cast<float4 *>(g.H + o0 + j) = make_float4(h[j], h[j + 1], h[j + 2], h[j + 3]);
            }
          } else {
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              if (nb + j >= g.N) continue;
              g.C[o0 + j] = v[j];
              if (g.epi == kEpiBiasGelu) g.H[o0 + j] = h[j];
            }
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem), "r"(kCols) : "memory");
}

}  // namespace pgpu
