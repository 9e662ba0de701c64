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

// Byte offset of element (r, k) of a no-swizzle K-major tile with `rows` rows
// (a multiple of 8) and 64 columns of BF16.
__device__ __forceinline__ int kmajor_off(int r, int k, int rows) {
  return (r & 7) * 16 + (r >> 3) * 128 + (k >> 3) * (rows * 16) + (k & 7) * 2;
}

// op(A) element (m, k) and op(B) element (k, n) as GemmArgs defines them.
__device__ __forceinline__ float tc_a(const GemmArgs &g, int m, int k) {
  return g.transA ? g.A[(int64_t)k * g.lda + m] : g.A[(int64_t)m * g.lda + k];
}
__device__ __forceinline__ float tc_b(const GemmArgs &g, int k, int n) {
  return g.transB ? g.B[(int64_t)n * g.ldb + k] : g.B[(int64_t)k * g.ldb + n];
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
  constexpr uint32_t idesc = umma_idesc_bf16(kTcBM, BN);
  uint32_t phase = 0;
  bool ok = true;
  int issued = 0;
  for (int k0 = kz0; k0 < kz1; k0 += kTcBK) {
    const int kc = min(kTcBK, kz1 - k0);
    // op(A) tile: consecutive threads take consecutive elements of the
    // contiguous global dimension (k, or m when A is transposed)
    for (int i = tid; i < kTcBM * kTcBK; i += 128) {
      const int m = g.transA ? (i & (kTcBM - 1)) : (i >> 6);
      const int k = g.transA ? (i >> 7) : (i & (kTcBK - 1));
      const float v = (m0 + m < g.M && k < kc) ? tc_a(g, m0 + m, k0 + k) : 0.f;
      *reinterpret_cast<__nv_bfloat16 *>(sA + kmajor_off(m, k, kTcBM)) = __float2bfloat16_rn(v);
    }
    for (int i = tid; i < BN * kTcBK; i += 128) {
      const int n = g.transB ? (i >> 6) : (i % BN);
      const int k = g.transB ? (i & (kTcBK - 1)) : (i / BN);
      const float v = (n0 + n < g.N && k < kc) ? tc_b(g, k0 + k, n0 + n) : 0.f;
      *reinterpret_cast<__nv_bfloat16 *>(sB + kmajor_off(n, k, BN)) = __float2bfloat16_rn(v);
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
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int n = n0 + c + j;
          if (n >= g.N) continue;
          const int64_t o = (int64_t)m * g.ldc + n;
          const float a = v[j];
          switch (g.epi) {
            case kEpiStore: g.C[o] = a; break;
            case kEpiBias: g.C[o] = a + g.bias[n]; break;
            case kEpiBiasGelu: {
              const float z = a + g.bias[n];
              g.C[o] = z;
              g.H[o] = gelu_f(z);
              break;
            }
            case kEpiGeluGrad: g.C[o] = a * gelu_grad(g.Z[o]); break;
            default: atomicAdd(g.C + o, a); break;
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
