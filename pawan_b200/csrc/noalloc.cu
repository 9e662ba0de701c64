// Rate evaluation that allocates no memory (pgpu_rates_noalloc).
//
// Some callers cannot call cudaMalloc at all.  Examples: code running inside
// another framework's memory pool, or inside a real-time loop, where an
// allocation would synchronise the device or could fail under memory
// pressure; and plugin hosts that only hand out buffers they allocated
// themselves.  For them this entry point takes device input and output
// buffers and does all of its intermediate work in one file-scope device
// array of fixed size.  It never calls cudaMalloc, cudaFree or any
// allocating library routine.
//
// The intermediate work is the packed FP32 source records and the per-chunk
// partial rates of the direct pair kernel.  The array has a fixed capacity of
// kNoAllocMaxN particles, ~13.6 MB, and every GPU that loads this library
// holds it until the process exits.
//
// In host code the array's name is only a host-side stand-in, not a device
// address.  So, once per device and with that device current, the first call
// asks the runtime for the array's device address (cudaGetSymbolAddress) and
// clears the work counters with an asynchronous memset on the caller's
// stream, ordered before that call's kernels.  That first call should
// therefore come before any stream capture on the device.
//
// All calls share the one array and it keeps the last call's contents: every
// call rewrites all it reads.  Calls that overlap on the GPU (on different
// streams, or from different host threads without ordering) race on it and
// must not be issued.
#include <cuda_runtime.h>

#include <cstdio>
#include <mutex>

#include "../../include/pawan_gpu.h"
#include "kernels.cuh"

using namespace pgpu;

namespace {

constexpr int64_t kNoAllocMaxN = PGPU_NOALLOC_MAX_N;
constexpr int kNoAllocChunks = 8;
constexpr int kNoAllocBlock = 256;  // one target per thread, 256-source tiles
constexpr int kNoAllocCG = kPairCG;  // sources per compensation group, as in the context path

// Carve-up of the scratch array (byte offsets, each 256-aligned).
constexpr size_t kOffP = 0;
constexpr size_t kOffQ = kOffP + kNoAllocMaxN * sizeof(float4);
constexpr size_t kOffPartial = kOffQ + kNoAllocMaxN * sizeof(float4);
constexpr size_t kOffPlan = kOffPartial + (size_t)kNoAllocChunks * 6 * kNoAllocMaxN * sizeof(double);
constexpr size_t kOffCounters = kOffPlan + 256;
constexpr size_t kOffNfull = kOffCounters + 256;
constexpr size_t kScratchBytes = kOffNfull + 256;
static_assert(kNoAllocMaxN % 16 == 0, "every region of the scratch array starts 256-byte aligned");
static_assert(2 * sizeof(PlanEntry) <= 256, "the plan fits its region");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char *g_scratch[kMaxDevices] = {nullptr};
int g_grid[kMaxDevices] = {0};
thread_local char g_err[256] = "";

int noalloc_fail(int code, const char *msg, long long v = 0, long long lim = 0) {
  snprintf(g_err, sizeof(g_err), msg, v, lim);
  return code;
}

// Row-major (n, 3) FP64 inputs -> source records, and the one-system work plan.
__global__ void noalloc_pack_kernel(const double *pos, const double *alpha, const double *sigma, const double *vol,
                                    int64_t n, float4 *P, float4 *Q, PlanEntry *plan, int nch) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const double s = sigma[i];
    P[i] = make_float4((float)pos[3 * i], (float)pos[3 * i + 1], (float)pos[3 * i + 2], (float)(0.5 * s * s));
    Q[i] = make_float4((float)alpha[3 * i], (float)alpha[3 * i + 1], (float)alpha[3 * i + 2], (float)vol[i]);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    const int64_t tiles = (n + kNoAllocBlock - 1) / kNoAllocBlock;
    const int64_t per = (n + nch - 1) / nch;
    plan[0].off = 0;
    plan[0].n = n;
    plan[0].item_start = 0;
    plan[0].tiles = tiles;
    plan[0].chunk = (per + kNoAllocBlock - 1) / kNoAllocBlock * kNoAllocBlock;
    plan[0].toff = 0;
    plan[0].tn = n;
    plan[1].off = 0;
    plan[1].n = 0;
    plan[1].item_start = tiles * nch;
    plan[1].tiles = 0;
    plan[1].chunk = 0;
    plan[1].toff = 0;
    plan[1].tn = 0;
  }
}

// Sum of the chunk partials -> row-major (n, 3) outputs.
__global__ void noalloc_reduce_kernel(const double *partial, int nch, int64_t n, double *vel, double *dalpha) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    for (int m = 0; m < 6; ++m) {
      double v = 0.0;
      for (int c = 0; c < nch; ++c) v += partial[((int64_t)c * 6 + m) * kNoAllocMaxN + i];
      if (m < 3) vel[3 * i + m] = v;
      else dalpha[3 * i + m - 3] = v;
    }
  }
}

// Device address of the scratch array for the current device (set up on the
// first call for that device).
int scratch_for_current_device(cudaStream_t st, unsigned char **out, int *grid) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return noalloc_fail(PGPU_ECUDA, "cudaGetDevice failed");
  if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(PGPU_EINVAL, "device %lld is beyond the %lld supported", dev, kMaxDevices);
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch[dev]) {
    void *ptr = nullptr;
    if (cudaGetSymbolAddress(&ptr, g_noalloc_scratch) != cudaSuccess || !ptr)
      return noalloc_fail(PGPU_ECUDA, "cudaGetSymbolAddress of the scratch array failed");
    unsigned char *base = static_cast<unsigned char *>(ptr);
    // The pair kernel's work counters must start at zero; after that it resets
    // them itself at the end of every launch.  Nothing else needs clearing:
    // each call rewrites the records, the plan and every partial it reads.
    // The clear goes on the caller's stream, so it is ordered before this
    // call's pair kernel even on a non-blocking stream.
    if (cudaMemsetAsync(base + kOffCounters, 0, 256, st) != cudaSuccess)
      return noalloc_fail(PGPU_ECUDA, "clearing the work counters failed");
    int sms = 0, nb = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, pair_kernel<float, kNoAllocBlock, 1, kNoAllocCG>, kNoAllocBlock,
                                                      0) != cudaSuccess)
      return noalloc_fail(PGPU_ECUDA, "querying the device for the launch size failed");
    g_grid[dev] = (nb > 0 ? nb : 1) * sms;
    g_scratch[dev] = base;
  }
  *out = g_scratch[dev];
  *grid = g_grid[dev];
  return PGPU_OK;
}

}  // namespace

extern "C" int pgpu_rates_noalloc(const double *pos, const double *alpha, const double *sigma, const double *vol,
                                  int64_t n, double nu, double *vel, double *dalpha, void *stream) {
  g_err[0] = '\0';
  if (n < 0 || n > kNoAllocMaxN)
    return noalloc_fail(PGPU_EINVAL, "n=%lld is outside [0, %lld], the capacity of the fixed scratch array", (long long)n,
                        (long long)kNoAllocMaxN);
  if (n == 0) return PGPU_OK;
  if (!pos || !alpha || !sigma || !vol || !vel || !dalpha) return noalloc_fail(PGPU_EINVAL, "null device array");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  unsigned char *base = nullptr;
  int grid = 0;
  int r = scratch_for_current_device(st, &base, &grid);
  if (r) return r;
  float4 *P = reinterpret_cast<float4 *>(base + kOffP);
  float4 *Q = reinterpret_cast<float4 *>(base + kOffQ);
  double *partial = reinterpret_cast<double *>(base + kOffPartial);
  PlanEntry *plan = reinterpret_cast<PlanEntry *>(base + kOffPlan);
  const int64_t tiles = (n + kNoAllocBlock - 1) / kNoAllocBlock;
  int nch = (int)((4LL * grid + tiles - 1) / tiles);
  nch = nch < 1 ? 1 : (nch > kNoAllocChunks ? kNoAllocChunks : nch);
  const int pg = (int)((n + 255) / 256 < 1024 ? (n + 255) / 256 : 1024);
  noalloc_pack_kernel<<<pg, 256, 0, st>>>(pos, alpha, sigma, vol, n, P, Q, plan, nch);
  PairArgs<float> a;
  a.P = P;
  a.Q = Q;
  a.partial = partial;
  a.plan = plan;
  a.nsys = 1;
  a.nch = nch;
  a.cap = kNoAllocMaxN;
  a.nu2 = (float)(2.0 * nu);
  a.counters = reinterpret_cast<unsigned int *>(base + kOffCounters);
  a.nfull = reinterpret_cast<unsigned long long *>(base + kOffNfull);
  pair_kernel<float, kNoAllocBlock, 1, kNoAllocCG><<<grid, kNoAllocBlock, 0, st>>>(a);
  noalloc_reduce_kernel<<<pg, 256, 0, st>>>(partial, nch, n, vel, dalpha);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    snprintf(g_err, sizeof(g_err), "kernel launch failed: %s", cudaGetErrorString(e));
    return PGPU_ECUDA;
  }
  return PGPU_OK;
}

extern "C" const char *pgpu_noalloc_last_error(void) { return g_err; }
