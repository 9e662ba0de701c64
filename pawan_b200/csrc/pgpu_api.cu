// C-ABI implementation of the B200 vortex-particle backend (include/pawan_gpu.h).
//
// Device memory of a context (cap = total particle slots of all wakes):
//   x0     [6][cap] FP64   state at the step start (x, y, z, alpha_x, alpha_y, alpha_z), SoA
//   acc    [6][cap] FP64   RK accumulator
//   rates  [6][cap] FP64   rates of the last evaluation
//   sig, vol [cap]  FP64   smoothing radius, volume
//   P, Q   [cap]    float4 (FP32C) or double4 (FP64) source records (x, y, z, sigma^2/2), (alpha, vol)
//   partial [nch][6][cap] FP64 per-chunk partial rates written by the pair kernel
//   stage  [8][cap] FP64   staging for host row-major <-> SoA transfers
// Systems occupy contiguous slot ranges; inside a system its wakes are laid out
// in the order they were added.
#include <cuda_runtime.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "../../include/pawan_gpu.h"
#include "kernels.cuh"
#include "treeeval.cuh"

#include <cub/cub.cuh>

using namespace pgpu;

namespace {

constexpr int kCG = kPairCG;
static_assert(kDiagFields == PGPU_DIAG_FIELDS, "the diagnostic field layout of the header");

struct Shape { int block, tpt; };
// Compiled pair-kernel shapes (the autotuner chooses among these).
constexpr Shape kShapes[] = {{128, 1}, {128, 2}, {256, 1}, {256, 2}, {64, 2}, {128, 4}};
constexpr int kNumShapes = sizeof(kShapes) / sizeof(kShapes[0]);

template <typename T> using PairFn = void (*)(PairArgs<T>);

template <typename T, int KER, bool SPLIT = false> PairFn<T> pair_fn_k(int s) {
  switch (s) {
    case 0: return pair_kernel<T, 128, 1, kCG, KER, SPLIT>;
    case 1: return pair_kernel<T, 128, 2, kCG, KER, SPLIT>;
    case 2: return pair_kernel<T, 256, 1, kCG, KER, SPLIT>;
    case 3: return pair_kernel<T, 256, 2, kCG, KER, SPLIT>;
    case 4: return pair_kernel<T, 64, 2, kCG, KER, SPLIT>;
    default: return pair_kernel<T, 128, 4, kCG, KER, SPLIT>;
  }
}
// Pair kernel of shape s for regularisation kernel `ker` (PGPU_KERNEL_*);
// split: the FP32C Gaussian body with split positions.
template <typename T> PairFn<T> pair_fn(int s, int ker, bool split) {
  if (ker == PGPU_KERNEL_HIGHORDER) return pair_fn_k<T, kHighOrder>(s);
  if constexpr (sizeof(T) == 4) {
    if (split) return pair_fn_k<T, kGaussian, true>(s);
  }
  return pair_fn_k<T, kGaussian>(s);
}

struct WakeRec {
  int sys;
  int64_t cap, n, off;
};
struct SysRec {
  std::vector<int> wakes;
  int64_t off = 0, cap = 0;
  double zc = 0.0;  // last reported Zc (PAWAN keeps _Zc across calls)
  int64_t t_first = 0, t_count = -1;  // owned targets (pgpu_set_target_range); count < 0: all
};

}  // namespace

struct SurrogateState;

struct pgpu_ctx {
  pgpu_config cfg;
  cudaStream_t st = nullptr;
  int sms = 0;
  std::vector<WakeRec> wakes;
  std::vector<SysRec> sys;
  bool frozen = false;
  int64_t cap = 0;
  double *x0 = nullptr, *acc = nullptr, *rates = nullptr, *sig = nullptr, *vol = nullptr;
  double *partial = nullptr, *stage = nullptr, *d_diag = nullptr;
  void *P = nullptr, *Q = nullptr;
  int64_t *d_sysoff = nullptr, *d_sysn = nullptr, *d_syst = nullptr;
  PlanEntry *d_plan = nullptr, *d_plan_diag = nullptr, *d_plan_field = nullptr;
  double *d_field = nullptr;  // [6][cap] vorticity field (components 0..2), allocated by pgpu_influence
  unsigned long long *d_merge = nullptr;  // merge candidate keys (pgpu_merge): d_merge_cap, a counter, d_merge_cap sorted
  int64_t d_merge_cap = 0;
  void *d_merge_tmp = nullptr;  // radix-sort space of the candidate keys
  size_t d_merge_tmp_bytes = 0;
  unsigned int *d_counters = nullptr;
  unsigned long long *d_nfull = nullptr;
  float4 *d_box = nullptr;  // FP32 source boxes per kBoxGran slots (box_kernel), FP32C Gaussian contexts
  float4 *d_L = nullptr;    // [cap] split-position residuals (pgpu_config.split_positions)
  int64_t pairs_acc = 0, selfs_acc = 0;  // ordered pairs and self pairs of the pair launches so far
  int *d_flag = nullptr;
  int diag_blocks = 0;
  int shape = 2;  // (256, 1) before autotuning: the high-order kernel's default (pgpu_create picks the Gaussian's)
  // Shapes per system chosen by pgpu_autotune_classes (empty: `shape` for
  // every system).  Each distinct shape in `groups` (ascending) is one pair
  // launch per evaluation over the systems that use it, with its own plan at
  // d_plan + g (nsys + 1).
  std::vector<int> sys_shape;
  std::vector<int> groups;
  int grid[kNumShapes] = {0};
  int nch = 1;
  bool plan_dirty = true;
  bool timing = true;
  bool capturing = false;
  cudaEvent_t ev[8][2] = {};
  double pair_ms = 0.0;
  int64_t pair_launches = 0;
  int64_t launches = 0;
  std::map<std::tuple<int, double, int, int, bool>, cudaGraphExec_t> graphs;  // (scheme, dt, launch layout, nch, timing)
  std::vector<cudaGraph_t> graph_defs;
  // last error message: a fixed buffer under a mutex, since pgpu_snapshot_wait
  // may fail on a writer thread while the owning thread queues work
  char err[512] = {0};
  std::mutex err_mu;
  SurrogateState *sur = nullptr;  // far-field surrogate of the single system, when enabled
  // State snapshots (pgpu_snapshot_begin / _wait): per slot a device buffer,
  // a pinned host buffer, the gather's and the copy's events, and the wake
  // rows the snapshot holds.
  cudaStream_t st_copy = nullptr;
  double *d_snap[2] = {nullptr, nullptr};
  double *h_snap[2] = {nullptr, nullptr};
  cudaEvent_t snap_gathered[2] = {nullptr, nullptr};
  cudaEvent_t snap_copied[2] = {nullptr, nullptr};
  bool snap_begun[2] = {false, false};
  std::vector<int64_t> snap_off[2], snap_n[2];
};

namespace {

// NVTX range over an entry point (header-only NVTX3: a no-op unless a
// profiler is attached), so profiler timelines show the library's phases.
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
};

// Makes a context's (or network's) device current for one entry point that
// works on the device, and restores the caller's device on return, so that
// contexts on different GPUs can be driven from one host thread.  pgpu_create
// leaves the new context's device current (as cudaSetDevice would), so a
// thread that creates a context and then uses it never switches: it calls
// nothing but cudaGetDevice.  Host-only calls and pgpu_snapshot_wait (which
// writer threads call; events need no current device) do not switch.
struct DeviceScope {
  int prev = -1;
  explicit DeviceScope(int dev) {
    int cur = -1;
    if (cudaGetDevice(&cur) == cudaSuccess && cur != dev && cudaSetDevice(dev) == cudaSuccess) prev = cur;
  }
  ~DeviceScope() {
    if (prev >= 0) cudaSetDevice(prev);
  }
  DeviceScope(const DeviceScope &) = delete;
  DeviceScope &operator=(const DeviceScope &) = delete;
};

int fail(pgpu_ctx *c, int code, const char *fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  if (c) {
    std::lock_guard<std::mutex> lock(c->err_mu);
    memcpy(c->err, buf, sizeof(buf));
  }
  return code;
}

// On failure the per-thread last error is reset (cudaGetLastError), so a
// non-sticky error such as a failed allocation is reported once, by the call
// that met it, and not again by the next healthy launch.
#define CK(call)                                                                                    \
  do {                                                                                              \
    cudaError_t e_ = (call);                                                                        \
    if (e_ != cudaSuccess) {                                                                        \
      cudaGetLastError();                                                                           \
      return fail(c, PGPU_ECUDA, "%s failed: %s", #call, cudaGetErrorString(e_));                   \
    }                                                                                               \
  } while (0)

// Why the calling thread's last pgpu_create failed ("" after a success);
// pgpu_last_error(NULL) returns it.
thread_local char g_create_err[512] = "";

// Releases what pgpu_create made before it failed, and records why.
int create_fail(pgpu_ctx *c, int code, const char *fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_create_err, sizeof(g_create_err), fmt, ap);
  va_end(ap);
  if (c) {
    for (auto &pair : c->ev)
      for (cudaEvent_t e : pair)
        if (e) cudaEventDestroy(e);
    if (c->st) cudaStreamDestroy(c->st);
    delete c;
  }
  return code;
}

bool fp64(const pgpu_ctx *c) { return c->cfg.precision == PGPU_FP64; }
// The FP32C Gaussian pair kernel tests whole source tiles against boxes
// precomputed per kBoxGran slots (box_kernel) before each launch.
bool uses_boxes(const pgpu_ctx *c) { return !fp64(c) && c->cfg.kernel == PGPU_KERNEL_GAUSSIAN; }
// Split positions: FP32C Gaussian contexts with pgpu_config.split_positions.
bool uses_split(const pgpu_ctx *c) { return uses_boxes(c) && c->cfg.split_positions != 0; }
// Boxes cover every slot plus one largest tile (256 slots) past the last:
// the last tile of the last system may end beyond `cap`, and those blocks
// hold empty boxes.
int64_t box_blocks(const pgpu_ctx *c) { return (c->cap + kBoxGran - 1) / kBoxGran + 256 / kBoxGran; }
size_t rec_bytes(const pgpu_ctx *c) { return fp64(c) ? sizeof(double4) : sizeof(float4); }

int64_t sys_n(const pgpu_ctx *c, int s) {
  const SysRec &S = c->sys[s];
  if (S.wakes.empty()) return 0;
  const WakeRec &L = c->wakes[S.wakes.back()];
  return (L.off - S.off) + L.n;
}

int check_contiguous(pgpu_ctx *c) {
  for (size_t s = 0; s < c->sys.size(); ++s) {
    const SysRec &S = c->sys[s];
    for (size_t k = 0; k + 1 < S.wakes.size(); ++k) {
      const WakeRec &W = c->wakes[S.wakes[k]];
      if (W.n != W.cap)
        return fail(c, PGPU_EINVAL,
                    "wake %d of system %zu holds %lld of %lld particles; every wake but the last of a system must be full",
                    S.wakes[k], s, (long long)W.n, (long long)W.cap);
    }
  }
  return PGPU_OK;
}

template <typename T> int occupancy(pgpu_ctx *c, int s) {
  int nb = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, pair_fn<T>(s, c->cfg.kernel, uses_split(c)), kShapes[s].block, 0);
  if (e != cudaSuccess || nb < 1) nb = 1;
  return nb * c->sms;
}

// Freeze the slot layout and allocate device memory (first upload).
int freeze(pgpu_ctx *c) {
  if (c->frozen) return PGPU_OK;
  if (c->wakes.empty()) return fail(c, PGPU_EINVAL, "no wakes were added");
  int64_t off = 0;
  for (auto &S : c->sys) {
    // systems start at multiples of kBoxGran slots, so every source tile of
    // the pair kernel is a run of whole precomputed boxes
    off = (off + kBoxGran - 1) / kBoxGran * kBoxGran;
    S.off = off;
    for (int w : S.wakes) {
      c->wakes[w].off = off;
      off += c->wakes[w].cap;
    }
    S.cap = off - S.off;
  }
  c->cap = std::max<int64_t>(off, 1);
  const int64_t cap = c->cap;
  auto alloc = [&](void **p, size_t bytes) -> int {
    cudaError_t e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();  // a failed allocation must not surface again at the next launch
      return fail(c, PGPU_ENOMEM, "cudaMalloc(%zu) failed: %s", bytes, cudaGetErrorString(e));
    }
    return PGPU_OK;
  };
  int r;
  if ((r = alloc((void **)&c->x0, 6 * cap * sizeof(double)))) return r;
  if ((r = alloc((void **)&c->acc, 6 * cap * sizeof(double)))) return r;
  if ((r = alloc((void **)&c->rates, 6 * cap * sizeof(double)))) return r;
  if ((r = alloc((void **)&c->sig, cap * sizeof(double)))) return r;
  if ((r = alloc((void **)&c->vol, cap * sizeof(double)))) return r;
  if ((r = alloc((void **)&c->stage, 8 * cap * sizeof(double)))) return r;
  if ((r = alloc((void **)&c->partial, (size_t)kMaxChunks * 6 * cap * sizeof(double)))) return r;
  if ((r = alloc(&c->P, cap * rec_bytes(c)))) return r;
  if ((r = alloc(&c->Q, cap * rec_bytes(c)))) return r;
  const size_t ns = c->sys.size();
  if ((r = alloc((void **)&c->d_sysoff, (ns + 1) * sizeof(int64_t)))) return r;
  if ((r = alloc((void **)&c->d_sysn, ns * sizeof(int64_t)))) return r;
  if ((r = alloc((void **)&c->d_syst, 2 * ns * sizeof(int64_t)))) return r;
  if ((r = alloc((void **)&c->d_plan, (size_t)kNumShapes * (ns + 1) * sizeof(PlanEntry)))) return r;
  if ((r = alloc((void **)&c->d_plan_diag, 2 * sizeof(PlanEntry)))) return r;
  if ((r = alloc((void **)&c->d_plan_field, (ns + 1) * sizeof(PlanEntry)))) return r;
  if ((r = alloc((void **)&c->d_counters, 4 * sizeof(unsigned int)))) return r;
  if ((r = alloc((void **)&c->d_nfull, sizeof(unsigned long long)))) return r;
  if (uses_boxes(c) && (r = alloc((void **)&c->d_box, 2 * box_blocks(c) * sizeof(float4)))) return r;
  if (uses_split(c)) {
    if ((r = alloc((void **)&c->d_L, cap * sizeof(float4)))) return r;
    CK(cudaMemsetAsync(c->d_L, 0, cap * sizeof(float4), c->st));
  }
  if ((r = alloc((void **)&c->d_flag, sizeof(int)))) return r;
  c->diag_blocks = 2 * c->sms;
  if ((r = alloc((void **)&c->d_diag, (size_t)c->diag_blocks * kDiagFields * sizeof(double)))) return r;
  CK(cudaMemsetAsync(c->x0, 0, 6 * cap * sizeof(double), c->st));
  CK(cudaMemsetAsync(c->acc, 0, 6 * cap * sizeof(double), c->st));
  CK(cudaMemsetAsync(c->rates, 0, 6 * cap * sizeof(double), c->st));
  CK(cudaMemsetAsync(c->sig, 0, cap * sizeof(double), c->st));
  CK(cudaMemsetAsync(c->vol, 0, cap * sizeof(double), c->st));
  CK(cudaMemsetAsync(c->partial, 0, (size_t)kMaxChunks * 6 * cap * sizeof(double), c->st));
  CK(cudaMemsetAsync(c->d_counters, 0, 4 * sizeof(unsigned int), c->st));
  CK(cudaMemsetAsync(c->d_nfull, 0, sizeof(unsigned long long), c->st));
  CK(cudaMemsetAsync(c->d_flag, 0, sizeof(int), c->st));
  for (int s = 0; s < kNumShapes; ++s) c->grid[s] = fp64(c) ? occupancy<double>(c, s) : occupancy<float>(c, s);
  c->frozen = true;
  c->plan_dirty = true;
  return PGPU_OK;
}

int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

// Owned targets [first, first + count) of system s (all of them unless
// pgpu_set_target_range restricted it), clamped to its particles.
std::pair<int64_t, int64_t> owned(const pgpu_ctx *c, int s) {
  const int64_t n = sys_n(c, s);
  const SysRec &S = c->sys[s];
  if (S.t_count < 0) return {0, n};
  const int64_t lo = std::min(S.t_first, n);
  return {lo, std::min(S.t_count, n - lo)};
}

bool restricted(const pgpu_ctx *c) {
  for (const SysRec &S : c->sys)
    if (S.t_count >= 0) return true;
  return false;
}

// Work list: systems by decreasing work, target tiles x source chunks each.
// With own_targets, only each system's owned targets are listed (all
// particles stay sources); otherwise every particle is a target.
std::vector<PlanEntry> build_plan(const pgpu_ctx *c, const std::vector<int> &systems, int shape, int nch,
                                  bool own_targets = true) {
  const int64_t TT = (int64_t)kShapes[shape].block * kShapes[shape].tpt;
  const int64_t TILE = kShapes[shape].block;
  std::vector<std::pair<int64_t, int>> order;
  for (int s : systems) {
    const int64_t tn = own_targets ? owned(c, s).second : sys_n(c, s);
    order.push_back({tn * sys_n(c, s), s});
  }
  std::stable_sort(order.begin(), order.end(), [](auto &a, auto &b) { return a.first > b.first; });
  std::vector<PlanEntry> plan;
  int64_t item = 0;
  for (auto &o : order) {
    const int64_t n = sys_n(c, o.second);
    const auto t = own_targets ? owned(c, o.second) : std::make_pair<int64_t, int64_t>(0, sys_n(c, o.second));
    if (n <= 0 || t.second <= 0) continue;
    PlanEntry e;
    e.off = c->sys[o.second].off;
    e.n = n;
    e.item_start = item;
    e.tiles = ceil_div(t.second, TT);
    e.chunk = ceil_div(ceil_div(n, nch), TILE) * TILE;
    e.toff = t.first;
    e.tn = t.second;
    item += e.tiles * nch;
    plan.push_back(e);
  }
  PlanEntry sentinel{};
  sentinel.item_start = item;
  plan.push_back(sentinel);
  return plan;
}

// Source chunks per system for one pair launch of `shape` over `systems`:
// enough work items for >= 24 per resident CTA, which keeps the tail of the
// persistent launch below ~2%.
int choose_nch_for(const pgpu_ctx *c, int shape, const std::vector<int> &systems) {
  if (c->cfg.chunks > 0) return std::min(c->cfg.chunks, kMaxChunks);
  const int64_t TT = (int64_t)kShapes[shape].block * kShapes[shape].tpt;
  int64_t tiles = 0;
  for (int s : systems) tiles += ceil_div(owned(c, s).second, TT);
  if (tiles <= 0) return 1;
  const int64_t want = 24LL * c->grid[shape];
  return (int)std::max<int64_t>(1, std::min<int64_t>(kMaxChunks, ceil_div(want, tiles)));
}

std::vector<int> all_systems(const pgpu_ctx *c) {
  std::vector<int> all(c->sys.size());
  for (size_t s = 0; s < all.size(); ++s) all[s] = (int)s;
  return all;
}

int choose_nch(const pgpu_ctx *c, int shape) { return choose_nch_for(c, shape, all_systems(c)); }

// Systems that launch with the g-th group's shape.
std::vector<int> group_systems(const pgpu_ctx *c, int g) {
  std::vector<int> out;
  for (size_t s = 0; s < c->sys.size(); ++s)
    if (c->sys_shape[s] == c->groups[g]) out.push_back((int)s);
  return out;
}

// Graph key part that fixes the launch sequence of one evaluation: the single
// shape, or the set of group shapes.
int launch_layout(const pgpu_ctx *c) {
  if (c->groups.empty()) return c->shape;
  int mask = 0;
  for (int g : c->groups) mask |= 1 << g;
  return 1000 + mask;
}

int upload_plan(pgpu_ctx *c) {
  if (!c->plan_dirty) return PGPU_OK;
  int r = check_contiguous(c);
  if (r) return r;
  const size_t ns = c->sys.size();
  c->groups.clear();
  if (!c->sur && c->sys_shape.size() == ns) {
    for (int sh : c->sys_shape)
      if (std::find(c->groups.begin(), c->groups.end(), sh) == c->groups.end()) c->groups.push_back(sh);
    std::sort(c->groups.begin(), c->groups.end());
    if (c->groups.size() == 1) {  // one shape after all: the single-launch path
      c->shape = c->groups[0];
      c->groups.clear();
    }
  }
  std::vector<PlanEntry> plan;
  if (c->groups.empty()) {
    // the surrogate writes one chunk of rates per evaluation
    c->nch = c->sur ? 1 : choose_nch(c, c->shape);
    plan = build_plan(c, all_systems(c), c->shape, c->nch);
    // Unused tail entries keep the sentinel item_start so the device search is bounded.
    plan.resize(ns + 1, plan.back());
  } else {
    // one chunk count for every group (the stage kernel sums nch chunks of
    // every particle): the largest any group's launch wants
    c->nch = 1;
    for (size_t g = 0; g < c->groups.size(); ++g)
      c->nch = std::max(c->nch, choose_nch_for(c, c->groups[g], group_systems(c, (int)g)));
    for (size_t g = 0; g < c->groups.size(); ++g) {
      std::vector<PlanEntry> p = build_plan(c, group_systems(c, (int)g), c->groups[g], c->nch);
      p.resize(ns + 1, p.back());
      plan.insert(plan.end(), p.begin(), p.end());
    }
  }
  std::vector<int64_t> off(c->sys.size() + 1), n(c->sys.size());
  for (size_t s = 0; s < c->sys.size(); ++s) { off[s] = c->sys[s].off; n[s] = sys_n(c, (int)s); }
  off[c->sys.size()] = c->cap;
  CK(cudaMemcpyAsync(c->d_plan, plan.data(), plan.size() * sizeof(PlanEntry), cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_sysoff, off.data(), off.size() * sizeof(int64_t), cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->d_sysn, n.data(), n.size() * sizeof(int64_t), cudaMemcpyHostToDevice, c->st));
  std::vector<int64_t> t(2 * c->sys.size());
  for (size_t k = 0; k < c->sys.size(); ++k) {
    // an unrestricted system owns every slot, including particles appended later
    const auto o = owned(c, (int)k);
    t[2 * k] = c->sys[k].t_count < 0 ? 0 : o.first;
    t[2 * k + 1] = c->sys[k].t_count < 0 ? INT64_MAX : o.first + o.second;
  }
  CK(cudaMemcpyAsync(c->d_syst, t.data(), t.size() * sizeof(int64_t), cudaMemcpyHostToDevice, c->st));
  // Pageable host sources: make sure the copies are done before the vectors go away.
  CK(cudaStreamSynchronize(c->st));
  c->plan_dirty = false;
  return PGPU_OK;
}

void account_pairs(pgpu_ctx *c, int launches) {
  for (size_t s = 0; s < c->sys.size(); ++s) {
    const int64_t n = sys_n(c, (int)s), tn = owned(c, (int)s).second;
    c->pairs_acc += launches * tn * (n > 0 ? n - 1 : 0);
    c->selfs_acc += launches * tn;
  }
}

int launch_boxes(pgpu_ctx *c) {
  const int64_t nb = box_blocks(c);
  const int grid = (int)std::min<int64_t>(ceil_div(nb, 8), 16LL * c->sms);  // 8 warps per CTA, one per block
  box_kernel<<<grid, 256, 0, c->st>>>(static_cast<const float4 *>(c->P), c->d_sysoff, c->d_sysn, (int)c->sys.size(),
                                      c->cap, nb, c->d_box);
  CK(cudaGetLastError());
  c->launches++;
  return PGPU_OK;
}

// Kernel launches of one rate evaluation by the direct sum.
int64_t eval_launches(const pgpu_ctx *c) {
  return (int64_t)std::max<size_t>(1, c->groups.size()) + (uses_boxes(c) ? 1 : 0);
}

template <typename T> int launch_pair(pgpu_ctx *c, int slot) {
  PairArgs<T> a;
  a.P = static_cast<const v4_t<T> *>(c->P);
  a.Q = static_cast<const v4_t<T> *>(c->Q);
  a.partial = c->partial;
  a.plan = c->d_plan;
  a.nsys = (int)c->sys.size();
  a.nch = c->nch;
  a.cap = c->cap;
  a.nu2 = (T)(2.0 * c->cfg.nu);
  a.counters = c->d_counters;
  a.nfull = c->d_nfull;
  if (uses_boxes(c)) {
    // source boxes of the current records, ahead of (and outside the timing of) the pair launch
    int r = launch_boxes(c);
    if (r) return r;
    a.box = c->d_box;
  }
  a.L = c->d_L;
  // Inside stream capture an event record only becomes a timestamp node of
  // the graph when it is marked external.
  const unsigned flags = c->capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
  if (c->timing && slot >= 0) CK(cudaEventRecordWithFlags(c->ev[slot][0], c->st, flags));
  if (c->groups.empty()) {
    pair_fn<T>(c->shape, c->cfg.kernel, uses_split(c))<<<c->grid[c->shape], kShapes[c->shape].block, 0, c->st>>>(a);
    CK(cudaGetLastError());
    c->launches++;
  } else {
    // one launch per group shape, each over its own plan; the launches share
    // the work counters, which each resets when its last CTA leaves
    for (size_t g = 0; g < c->groups.size(); ++g) {
      const int sh = c->groups[g];
      a.plan = c->d_plan + g * (c->sys.size() + 1);
      pair_fn<T>(sh, c->cfg.kernel, uses_split(c))<<<c->grid[sh], kShapes[sh].block, 0, c->st>>>(a);
      CK(cudaGetLastError());
      c->launches++;
    }
  }
  if (c->timing && slot >= 0) CK(cudaEventRecordWithFlags(c->ev[slot][1], c->st, flags));
  if (!c->capturing) account_pairs(c, 1);
  return PGPU_OK;
}

int launch_stage(pgpu_ctx *c, int scheme, int stage, double dt) {
  StageArgs s;
  s.x0 = c->x0; s.acc = c->acc; s.rates = c->rates; s.sig = c->sig; s.vol = c->vol; s.L = c->d_L;
  s.partial = c->partial; s.P = c->P; s.Q = c->Q;
  s.sys_off = c->d_sysoff; s.sys_n = c->d_sysn; s.sys_t = c->d_syst; s.nsys = (int)c->sys.size();
  s.nch = c->nch; s.cap = c->cap; s.scheme = scheme; s.stage = stage; s.dt = dt;
  for (int m = 0; m < 3; ++m) s.vinf[m] = c->cfg.vinf[m];
  s.flag = c->d_flag;
  const int block = 256;
  const int grid = (int)std::min<int64_t>(ceil_div(c->cap, block), 16LL * c->sms);
  if (fp64(c)) stage_kernel<double><<<grid, block, 0, c->st>>>(s);
  else stage_kernel<float><<<grid, block, 0, c->st>>>(s);
  CK(cudaGetLastError());
  c->launches++;
  return PGPU_OK;
}

int launch_pack(pgpu_ctx *c, int64_t lo, int64_t hi) {
  if (hi <= lo) return PGPU_OK;
  const int block = 256;
  const int grid = (int)std::min<int64_t>(ceil_div(hi - lo, block), 16LL * c->sms);
  if (fp64(c)) pack_kernel<double><<<grid, block, 0, c->st>>>(c->x0, c->sig, c->vol, c->P, c->Q, nullptr, lo, hi, c->cap);
  else pack_kernel<float><<<grid, block, 0, c->st>>>(c->x0, c->sig, c->vol, c->P, c->Q, c->d_L, lo, hi, c->cap);
  CK(cudaGetLastError());
  c->launches++;
  return PGPU_OK;
}

int surrogate_eval(pgpu_ctx *c);
void surrogate_free(pgpu_ctx *c);
int surrogate_pick_targets(pgpu_ctx *c, SurrogateState *s);

int launch_eval(pgpu_ctx *c, int slot) {
  if (c->sur) return surrogate_eval(c);
  return fp64(c) ? launch_pair<double>(c, slot) : launch_pair<float>(c, slot);
}

int collect_timing(pgpu_ctx *c, int nslots) {
  if (!c->timing || c->sur) return PGPU_OK;  // surrogate evaluations keep their own phase times
  for (int k = 0; k < nslots; ++k) {
    CK(cudaEventSynchronize(c->ev[k][1]));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c->ev[k][0], c->ev[k][1]));
    c->pair_ms += ms;
    c->pair_launches++;
  }
  return PGPU_OK;
}

int stages_of(int scheme) { return scheme == PGPU_RK4 ? 4 : scheme == PGPU_RK3 ? 3 : 1; }

int record_step(pgpu_ctx *c, int scheme, double dt) {
  const int ns = stages_of(scheme);
  for (int k = 0; k < ns; ++k) {
    int r = launch_eval(c, k);
    if (r) return r;
    if ((r = launch_stage(c, scheme, k, dt))) return r;
  }
  return PGPU_OK;
}

int wake_ok(pgpu_ctx *c, int32_t wake) {
  if (!c) return PGPU_EINVAL;
  if (wake < 0 || wake >= (int32_t)c->wakes.size()) return fail(c, PGPU_EINVAL, "invalid wake id %d", wake);
  return PGPU_OK;
}

int upload_rows(pgpu_ctx *c, const WakeRec &W, int64_t first, int64_t m, const double *pos, const double *alpha,
                const double *sigma, const double *vol) {
  if (m <= 0) return PGPU_OK;
  if (!pos || !alpha || !sigma || !vol) return fail(c, PGPU_EINVAL, "null particle array");
  CK(cudaMemcpyAsync(c->stage, pos, 3 * m * sizeof(double), cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->stage + 3 * m, alpha, 3 * m * sizeof(double), cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->stage + 6 * m, sigma, m * sizeof(double), cudaMemcpyHostToDevice, c->st));
  CK(cudaMemcpyAsync(c->stage + 7 * m, vol, m * sizeof(double), cudaMemcpyHostToDevice, c->st));
  const int grid = (int)std::min<int64_t>(ceil_div(m, 256), 16LL * c->sms);
  scatter_kernel<<<grid, 256, 0, c->st>>>(c->stage, m, W.off + first, c->cap, c->x0, c->sig, c->vol);
  CK(cudaGetLastError());
  c->launches++;
  return launch_pack(c, W.off + first, W.off + first + m);
}

}  // namespace

extern "C" {

void pgpu_config_default(pgpu_config *cfg) {
  memset(cfg, 0, sizeof(*cfg));
  cfg->precision = PGPU_FP32C;
  cfg->device = 0;
  cfg->nu = 1.56e-5;
  cfg->use_graphs = 1;
}

const char *pgpu_version(void) { return "pawan_b200 0.1 (sm_100a)"; }

int pgpu_create(pgpu_ctx **out, const pgpu_config *cfg) {
  if (!out) return create_fail(nullptr, PGPU_EINVAL, "no output pointer for the context");
  *out = nullptr;
  pgpu_ctx *c = new pgpu_ctx;
  if (cfg) c->cfg = *cfg;
  else pgpu_config_default(&c->cfg);
  if (c->cfg.precision != PGPU_FP32C && c->cfg.precision != PGPU_FP64)
    return create_fail(c, PGPU_EINVAL, "unknown precision %d", c->cfg.precision);
  if (c->cfg.kernel != PGPU_KERNEL_GAUSSIAN && c->cfg.kernel != PGPU_KERNEL_HIGHORDER)
    return create_fail(c, PGPU_EINVAL, "unknown regularisation kernel %d", c->cfg.kernel);
  if (c->cfg.block > 0 || c->cfg.tpt > 0) {
    int found = -1;
    for (int s = 0; s < kNumShapes; ++s)
      if ((c->cfg.block <= 0 || kShapes[s].block == c->cfg.block) && (c->cfg.tpt <= 0 || kShapes[s].tpt == c->cfg.tpt)) {
        found = s;
        break;
      }
    if (found < 0)
      return create_fail(c, PGPU_EINVAL, "no compiled pair-kernel shape with block %d and %d targets per thread",
                         c->cfg.block, c->cfg.tpt);
    c->shape = found;
  } else if (c->cfg.kernel == PGPU_KERNEL_GAUSSIAN) {
    // untuned defaults: the fastest Gaussian shapes on the 1M ring, FP32C
    // 128 x 2 (1075 ms per evaluation against 1163 ms for 256 x 1) and FP64
    // 128 x 1 (3.09 s against 3.22 s)
    c->shape = c->cfg.precision == PGPU_FP32C ? 1 : 0;
  }
  cudaError_t e = cudaSetDevice(c->cfg.device);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&c->sms, cudaDevAttrMultiProcessorCount, c->cfg.device);
  for (int k = 0; k < 8 && e == cudaSuccess; ++k) {
    e = cudaEventCreate(&c->ev[k][0]);
    if (e == cudaSuccess) e = cudaEventCreate(&c->ev[k][1]);
  }
  if (e != cudaSuccess) {
    cudaGetLastError();
    return create_fail(c, PGPU_ECUDA, "device %d: %s", c->cfg.device, cudaGetErrorString(e));
  }
  g_create_err[0] = '\0';
  *out = c;
  return PGPU_OK;
}

int pgpu_destroy(pgpu_ctx *c) {
  if (!c) return PGPU_EINVAL;
  DeviceScope device_scope(c->cfg.device);
  cudaStreamSynchronize(c->st);
  surrogate_free(c);
  for (auto &g : c->graphs) cudaGraphExecDestroy(g.second);
  for (auto g : c->graph_defs) cudaGraphDestroy(g);
  void *ptrs[] = {c->x0, c->acc, c->rates, c->sig, c->vol, c->partial, c->stage, c->d_diag, c->P, c->Q,
                  c->d_sysoff, c->d_sysn, c->d_syst, c->d_plan, c->d_plan_diag, c->d_plan_field, c->d_field,
                  c->d_counters, c->d_nfull, c->d_flag, c->d_merge, c->d_merge_tmp, c->d_box, c->d_L};
  for (void *p : ptrs)
    if (p) cudaFree(p);
  for (int k = 0; k < 8; ++k) { cudaEventDestroy(c->ev[k][0]); cudaEventDestroy(c->ev[k][1]); }
  if (c->st_copy) cudaStreamSynchronize(c->st_copy);
  for (int s = 0; s < 2; ++s) {
    if (c->d_snap[s]) cudaFree(c->d_snap[s]);
    if (c->h_snap[s]) cudaFreeHost(c->h_snap[s]);
    if (c->snap_gathered[s]) cudaEventDestroy(c->snap_gathered[s]);
    if (c->snap_copied[s]) cudaEventDestroy(c->snap_copied[s]);
  }
  if (c->st_copy) cudaStreamDestroy(c->st_copy);
  cudaStreamDestroy(c->st);
  delete c;
  return PGPU_OK;
}

int pgpu_add_wake(pgpu_ctx *c, int32_t system, int64_t capacity, int32_t *wake_id) {
  if (!c) return PGPU_EINVAL;
  if (c->frozen) return fail(c, PGPU_EINVAL, "wakes must be added before the first particle upload");
  if (system < 0 || system > 1 << 20) return fail(c, PGPU_EINVAL, "invalid system id %d", system);
  if (capacity < 0 || capacity > (int64_t)1 << 31) return fail(c, PGPU_EINVAL, "invalid capacity %lld", (long long)capacity);
  if ((int)c->sys.size() <= system) c->sys.resize(system + 1);
  WakeRec w{system, capacity, 0, 0};
  c->wakes.push_back(w);
  c->sys[system].wakes.push_back((int)c->wakes.size() - 1);
  if (wake_id) *wake_id = (int32_t)c->wakes.size() - 1;
  return PGPU_OK;
}

int pgpu_set_particles(pgpu_ctx *c, int32_t wake, int64_t n, const double *pos, const double *alpha,
                       const double *sigma, const double *vol) {
  int r = wake_ok(c, wake);
  if (r) return r;
  DeviceScope device_scope(c->cfg.device);
  if ((r = freeze(c))) return r;
  WakeRec &W = c->wakes[wake];
  if (n < 0 || n > W.cap) return fail(c, PGPU_EINVAL, "n=%lld exceeds the capacity %lld of wake %d", (long long)n, (long long)W.cap, wake);
  if ((r = upload_rows(c, W, 0, n, pos, alpha, sigma, vol))) return r;
  W.n = n;
  c->plan_dirty = true;
  return PGPU_OK;
}

int pgpu_append_particles(pgpu_ctx *c, int32_t wake, int64_t m, const double *pos, const double *alpha,
                          const double *sigma, const double *vol) {
  int r = wake_ok(c, wake);
  if (r) return r;
  DeviceScope device_scope(c->cfg.device);
  if ((r = freeze(c))) return r;
  WakeRec &W = c->wakes[wake];
  if (c->sys[W.sys].wakes.back() != wake) return fail(c, PGPU_EINVAL, "only the last wake of a system can grow");
  if (m < 0 || W.n + m > W.cap) return fail(c, PGPU_EINVAL, "appending %lld particles exceeds the capacity of wake %d", (long long)m, wake);
  if ((r = upload_rows(c, W, W.n, m, pos, alpha, sigma, vol))) return r;
  // Appended particles start a step with a zero RK accumulator.
  W.n += m;
  c->plan_dirty = true;
  return PGPU_OK;
}

int pgpu_get_num_particles(pgpu_ctx *c, int32_t wake, int64_t *n) {
  int r = wake_ok(c, wake);
  if (r) return r;
  if (n) *n = c->wakes[wake].n;
  return PGPU_OK;
}

static int download_rows(pgpu_ctx *c, const double *src, const WakeRec &W, double *a, double *b) {
  if (W.n == 0) return PGPU_OK;
  const int grid = (int)std::min<int64_t>(ceil_div(W.n, 256), 16LL * c->sms);
  gather_kernel<<<grid, 256, 0, c->st>>>(src, W.n, W.off, c->cap, c->stage);
  CK(cudaGetLastError());
  c->launches++;
  CK(cudaMemcpyAsync(a, c->stage, 3 * W.n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaMemcpyAsync(b, c->stage + 3 * W.n, 3 * W.n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaStreamSynchronize(c->st));
  return PGPU_OK;
}

int pgpu_get_state(pgpu_ctx *c, int32_t wake, double *pos, double *alpha) {
  int r = wake_ok(c, wake);
  if (r) return r;
  DeviceScope device_scope(c->cfg.device);
  if (!c->frozen) return fail(c, PGPU_EINVAL, "no particles were uploaded");
  if (!pos || !alpha) return fail(c, PGPU_EINVAL, "null output array");
  return download_rows(c, c->x0, c->wakes[wake], pos, alpha);
}

int pgpu_get_rates(pgpu_ctx *c, int32_t wake, double *vel, double *dalpha) {
  int r = wake_ok(c, wake);
  if (r) return r;
  DeviceScope device_scope(c->cfg.device);
  if (!c->frozen) return fail(c, PGPU_EINVAL, "no particles were uploaded");
  if (!vel || !dalpha) return fail(c, PGPU_EINVAL, "null output array");
  return download_rows(c, c->rates, c->wakes[wake], vel, dalpha);
}

static int flat_io(pgpu_ctx *c, double *flat, const int64_t *maxn, int32_t nwakes, int dir, const double *soa_src) {
  if (!c) return PGPU_EINVAL;
  DeviceScope device_scope(c->cfg.device);
  if (!c->frozen) return fail(c, PGPU_EINVAL, "no particles were uploaded");
  if (!flat || !maxn || nwakes != (int32_t)c->wakes.size()) return fail(c, PGPU_EINVAL, "flat state needs one capacity per wake");
  int64_t off = 0;
  for (int w = 0; w < nwakes; ++w) {
    const WakeRec &W = c->wakes[w];
    if (maxn[w] < W.n) return fail(c, PGPU_EINVAL, "maxn[%d] is smaller than the wake size", w);
    const int64_t sz = 6 * maxn[w];
    if (W.n > 0) {
      const int grid = (int)std::min<int64_t>(ceil_div(W.n, 256), 16LL * c->sms);
      if (dir == 0) {
        CK(cudaMemcpyAsync(c->stage, flat + off, 3 * W.n * sizeof(double), cudaMemcpyHostToDevice, c->st));
        CK(cudaMemcpyAsync(c->stage + 3 * W.n, flat + off + 3 * maxn[w], 3 * W.n * sizeof(double), cudaMemcpyHostToDevice, c->st));
        flat_kernel<<<grid, 256, 0, c->st>>>(c->stage, W.n, W.n, W.off, c->cap, c->x0, 0);
        CK(cudaGetLastError());
        c->launches++;
        int r = launch_pack(c, W.off, W.off + W.n);
        if (r) return r;
        CK(cudaStreamSynchronize(c->st));
      } else {
        flat_kernel<<<grid, 256, 0, c->st>>>(c->stage, W.n, W.n, W.off, c->cap, const_cast<double *>(soa_src), 1);
        CK(cudaGetLastError());
        c->launches++;
        CK(cudaMemcpyAsync(flat + off, c->stage, 3 * W.n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
        CK(cudaMemcpyAsync(flat + off + 3 * maxn[w], c->stage + 3 * W.n, 3 * W.n * sizeof(double), cudaMemcpyDeviceToHost, c->st));
        CK(cudaStreamSynchronize(c->st));
      }
    }
    off += sz;
  }
  return PGPU_OK;
}

int pgpu_set_states_flat(pgpu_ctx *c, const double *state, const int64_t *maxn, int32_t nwakes) {
  return flat_io(c, const_cast<double *>(state), maxn, nwakes, 0, nullptr);
}
int pgpu_get_states_flat(pgpu_ctx *c, double *state, const int64_t *maxn, int32_t nwakes) {
  return flat_io(c, state, maxn, nwakes, 1, c ? c->x0 : nullptr);
}
int pgpu_get_rates_flat(pgpu_ctx *c, double *rate, const int64_t *maxn, int32_t nwakes) {
  return flat_io(c, rate, maxn, nwakes, 1, c ? c->rates : nullptr);
}

int pgpu_solve(pgpu_ctx *c) {
  NvtxRange nvtx("pgpu_solve");
  if (!c) return PGPU_EINVAL;
  DeviceScope device_scope(c->cfg.device);
  if (!c->frozen) return fail(c, PGPU_EINVAL, "no particles were uploaded");
  int r = upload_plan(c);
  if (r) return r;
  if ((r = launch_eval(c, 0))) return r;
  if ((r = launch_stage(c, -1, 0, 0.0))) return r;
  return collect_timing(c, 1);
}

int pgpu_set_target_range(pgpu_ctx *c, int32_t system, int64_t first, int64_t count) {
  if (!c) return PGPU_EINVAL;
  DeviceScope device_scope(c->cfg.device);
  if (system < 0 || system >= (int32_t)c->sys.size()) return fail(c, PGPU_EINVAL, "invalid system id %d", system);
  if (uses_split(c) && count >= 0)
    return fail(c, PGPU_EINVAL, "split positions are not exchanged between contexts: use one context per system");
  if (count >= 0 && first < 0) return fail(c, PGPU_EINVAL, "negative first target %lld", (long long)first);
  SysRec &S = c->sys[system];
  S.t_first = count < 0 ? 0 : first;
  S.t_count = count < 0 ? -1 : count;
  c->plan_dirty = true;
  // the surrogate's sampled check draws from the owned targets
  if (c->sur) return surrogate_pick_targets(c, c->sur);
  return PGPU_OK;
}

int pgpu_stage(pgpu_ctx *c, int scheme, int stage, double dt) {
  NvtxRange nvtx("pgpu_stage");
  if (!c) return PGPU_EINVAL;
  DeviceScope device_scope(c->cfg.device);
  if (scheme != PGPU_EULER && scheme != PGPU_RK3 && scheme != PGPU_RK4) return fail(c, PGPU_EINVAL, "unknown scheme %d", scheme);
  if (stage < 0 || stage >= stages_of(scheme)) return fail(c, PGPU_EINVAL, "stage %d out of range for scheme %d", stage, scheme);
  if (!c->frozen) return fail(c, PGPU_EINVAL, "no particles were uploaded");
  int r = upload_plan(c);
  if (r) return r;
  if ((r = launch_eval(c, 0))) return r;
  if ((r = launch_stage(c, scheme, stage, dt))) return r;
  return collect_timing(c, 1);
}

int pgpu_records(pgpu_ctx *c, int32_t system, void **P, void **Q) {
  if (!c || !P || !Q) return PGPU_EINVAL;
  if (!c->frozen) return fail(c, PGPU_EINVAL, "no particles were uploaded");
  if (system < 0 || system >= (int32_t)c->sys.size()) return fail(c, PGPU_EINVAL, "invalid system id %d", system);
  const size_t rb = rec_bytes(c);
  *P = static_cast<char *>(c->P) + (size_t)c->sys[system].off * rb;
  *Q = static_cast<char *>(c->Q) + (size_t)c->sys[system].off * rb;
  return PGPU_OK;
}

int pgpu_step(pgpu_ctx *c, int scheme, double dt, int32_t nsteps) {
  NvtxRange nvtx("pgpu_step");
  if (!c) return PGPU_EINVAL;
  DeviceScope device_scope(c->cfg.device);
  if (scheme != PGPU_EULER && scheme != PGPU_RK3 && scheme != PGPU_RK4) return fail(c, PGPU_EINVAL, "unknown scheme %d", scheme);
  if (nsteps < 0) return fail(c, PGPU_EINVAL, "negative step count");
  if (!c->frozen) return fail(c, PGPU_EINVAL, "no particles were uploaded");
  if (restricted(c))
    return fail(c, PGPU_EINVAL, "a context with target ranges steps stage by stage (pgpu_stage), with the source "
                                "records of the other targets exchanged between stages");
  int r = upload_plan(c);
  if (r) return r;
  const int ns = stages_of(scheme);
  if (!c->cfg.use_graphs || c->sur) {  // the surrogate's tree build synchronises with the host
    for (int i = 0; i < nsteps; ++i) {
      if ((r = record_step(c, scheme, dt))) return r;
      if ((r = collect_timing(c, ns))) return r;
    }
    return PGPU_OK;
  }
  auto key = std::make_tuple(scheme, dt, launch_layout(c), c->nch, c->timing);
  auto it = c->graphs.find(key);
  if (it == c->graphs.end()) {
    cudaGraph_t g;
    CK(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
    const int64_t before = c->launches;
    c->capturing = true;
    r = record_step(c, scheme, dt);
    c->capturing = false;
    cudaError_t e = cudaStreamEndCapture(c->st, &g);
    if (r) return r;
    if (e != cudaSuccess) return fail(c, PGPU_ECUDA, "stream capture failed: %s", cudaGetErrorString(e));
    c->launches = before;  // counted at replay
    cudaGraphExec_t ex;
    CK(cudaGraphInstantiate(&ex, g, 0));
    c->graph_defs.push_back(g);
    it = c->graphs.emplace(key, ex).first;
  }
  for (int i = 0; i < nsteps; ++i) {
    CK(cudaGraphLaunch(it->second, c->st));
    c->launches += (1 + eval_launches(c)) * ns;
    account_pairs(c, ns);
    if ((r = collect_timing(c, ns))) return r;
  }
  return PGPU_OK;
}

int pgpu_diagnose_partial(pgpu_ctx *c, int32_t system, double *fields) {
  NvtxRange nvtx("pgpu_diagnose_partial");
  if (!c || !fields) return PGPU_EINVAL;
  DeviceScope device_scope(c->cfg.device);
  if (!c->frozen) return fail(c, PGPU_EINVAL, "no particles were uploaded");
  if (system < 0 || system >= (int32_t)c->sys.size()) return fail(c, PGPU_EINVAL, "invalid system id %d", system);
  int r = check_contiguous(c);
  if (r) return r;
  const int shape = 2;  // 256-thread tiles for the diagnostic pair sums
  const int block = 256;
  const auto own = owned(c, system);
  const int64_t row_lo = c->sys[system].off + own.first, row_hi = row_lo + own.second;
  const int nch = std::max(1, std::min(kMaxChunks, (int)ceil_div(8LL * c->sms, std::max<int64_t>(1, ceil_div(own.second, block)))));
  // rows: the owned targets (all of them without a target range); each
  // unordered pair is summed from its lower index, so the ranks' row ranges
  // together cover every pair once
  std::vector<PlanEntry> plan = build_plan(c, {system}, shape, nch, true);
  CK(cudaMemcpyAsync(c->d_plan_diag, plan.data(), plan.size() * sizeof(PlanEntry), cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  const bool quad = plan.size() > 1;
  if (quad) {
    int grid = 0;
    const bool ho = c->cfg.kernel == PGPU_KERNEL_HIGHORDER;
    if (fp64(c)) {
      DiagArgs<double> a{static_cast<const double4 *>(c->P), static_cast<const double4 *>(c->Q), c->partial,
                         c->d_plan_diag, 1, nch, c->cap, c->d_counters};
      auto fn = ho ? diag_pair_kernel<double, 256, kHighOrder> : diag_pair_kernel<double, 256, kGaussian>;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&grid, fn, block, 0);
      fn<<<std::max(1, grid) * c->sms, block, 0, c->st>>>(a);
    } else {
      DiagArgs<float> a{static_cast<const float4 *>(c->P), static_cast<const float4 *>(c->Q), c->partial,
                        c->d_plan_diag, 1, nch, c->cap, c->d_counters};
      auto fn = ho ? diag_pair_kernel<float, 256, kHighOrder> : diag_pair_kernel<float, 256, kGaussian>;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&grid, fn, block, 0);
      fn<<<std::max(1, grid) * c->sms, block, 0, c->st>>>(a);
    }
    CK(cudaGetLastError());
    c->launches++;
  }
  std::vector<double> h((size_t)c->diag_blocks * kDiagFields);
  const std::vector<int> &ws = c->sys[system].wakes;
  for (size_t k = 0; k < ws.size(); ++k) {
    const WakeRec &W = c->wakes[ws[k]];
    double *g = fields + k * PGPU_DIAG_FIELDS;
    for (int m = 0; m < PGPU_DIAG_FIELDS; ++m) g[m] = 0.0;
    const int64_t lo = std::max(W.off, row_lo), hi = std::min(W.off + W.n, row_hi);
    if (hi <= lo) continue;
    const int grid = (int)std::min<int64_t>(ceil_div(hi - lo, 256), c->diag_blocks);
    diag_wake_kernel<<<grid, 256, 0, c->st>>>(c->x0, c->sig, c->partial, nch, c->cap, lo, hi, quad ? 1 : 0,
                                              c->cfg.kernel, c->d_diag);
    CK(cudaGetLastError());
    c->launches++;
    CK(cudaMemcpyAsync(h.data(), c->d_diag, (size_t)grid * kDiagFields * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    CK(cudaStreamSynchronize(c->st));
    // per-CTA partials summed in CTA order: deterministic
    for (int b = 0; b < grid; ++b)
      for (int m = 0; m < kDiagFields; ++m) g[m] += h[(size_t)b * kDiagFields + m];
  }
  return PGPU_OK;
}

int pgpu_diagnose_combine(const double *fields, int32_t nwakes, double zc_prev, double *out, double *vbi,
                          double *zc_out) {
  if (!fields || !out || nwakes < 0) return PGPU_EINVAL;
  double f[PGPU_DIAG_FIELDS] = {0};
  double zc = zc_prev;
  for (int k = 0; k < nwakes; ++k) {
    const double *g = fields + (size_t)k * PGPU_DIAG_FIELDS;
    for (int m = 0; m < PGPU_DIAG_FIELDS; ++m) f[m] += g[m];
    // PAWAN's Zc: the last wake with non-zero weight wins (interaction.cpp:135-157)
    if (g[10] != 0.0) zc = g[9] / g[10];
  }
  for (int m = 0; m < 3; ++m) {
    out[m] = f[m];
    out[3 + m] = 0.5 * f[3 + m];
    out[6 + m] = f[6 + m] / 3.0;
  }
  out[9] = f[14];
  out[10] = f[21] + f[19];
  out[11] = f[22] + f[20];
  out[12] = f[17] + f[15];
  out[13] = f[18] + f[16];
  out[14] = zc;
  if (vbi)
    for (int m = 0; m < 3; ++m) vbi[m] = f[11 + m];
  if (zc_out) *zc_out = zc;
  return PGPU_OK;
}

int pgpu_diagnose(pgpu_ctx *c, int32_t system, double *out, double *vbi) {
  NvtxRange nvtx("pgpu_diagnose");
  if (!c || !out) return PGPU_EINVAL;
  DeviceScope device_scope(c->cfg.device);
  if (!c->frozen) return fail(c, PGPU_EINVAL, "no particles were uploaded");
  if (restricted(c))
    return fail(c, PGPU_EINVAL, "with target ranges each context holds a part of the diagnostics: sum "
                                "pgpu_diagnose_partial over the contexts and finish with pgpu_diagnose_combine");
  if (system < 0 || system >= (int32_t)c->sys.size()) return fail(c, PGPU_EINVAL, "invalid system id %d", system);
  std::vector<double> fields(c->sys[system].wakes.size() * PGPU_DIAG_FIELDS);
  int r = pgpu_diagnose_partial(c, system, fields.data());
  if (r) return r;
  double zc = c->sys[system].zc;
  pgpu_diagnose_combine(fields.data(), (int32_t)c->sys[system].wakes.size(), zc, out, vbi, &zc);
  c->sys[system].zc = zc;
  return PGPU_OK;
}

int pgpu_probe(pgpu_ctx *c, int32_t system, int64_t npts, const double *pts, double *vel) {
  if (!c) return PGPU_EINVAL;
  DeviceScope device_scope(c->cfg.device);
  if (!c->frozen) return fail(c, PGPU_EINVAL, "no particles were uploaded");
  if (system < 0 || system >= (int32_t)c->sys.size()) return fail(c, PGPU_EINVAL, "invalid system id %d", system);
  if (npts < 0 || (npts > 0 && (!pts || !vel))) return fail(c, PGPU_EINVAL, "bad probe arrays");
  if (npts == 0) return PGPU_OK;
  double *d = nullptr;
  CK(cudaMallocAsync((void **)&d, 6 * npts * sizeof(double), c->st));
  CK(cudaMemcpyAsync(d, pts, 3 * npts * sizeof(double), cudaMemcpyHostToDevice, c->st));
  CK(cudaMemsetAsync(d + 3 * npts, 0, 3 * npts * sizeof(double), c->st));
  const int64_t lo = c->sys[system].off, hi = lo + sys_n(c, system);
  if (hi > lo) {
    auto fn = c->cfg.kernel == PGPU_KERNEL_HIGHORDER ? probe_kernel<128, kHighOrder> : probe_kernel<128, kGaussian>;
    fn<<<(unsigned)ceil_div(npts, 128), 128, 0, c->st>>>(c->x0, c->sig, c->cap, lo, hi, d, npts, d + 3 * npts);
    CK(cudaGetLastError());
    c->launches++;
  }
  CK(cudaMemcpyAsync(vel, d + 3 * npts, 3 * npts * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  CK(cudaFreeAsync(d, c->st));
  CK(cudaStreamSynchronize(c->st));
  return PGPU_OK;
}

int pgpu_sync(pgpu_ctx *c) {
  if (!c) return PGPU_EINVAL;
  DeviceScope device_scope(c->cfg.device);
  CK(cudaStreamSynchronize(c->st));
  if (c->frozen) {
    int flag = 0;
    CK(cudaMemcpy(&flag, c->d_flag, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
      CK(cudaMemset(c->d_flag, 0, sizeof(int)));
      return fail(c, PGPU_ENUMERIC, "a time step produced a non-finite particle state");
    }
  }
  return PGPU_OK;
}

int pgpu_influence(pgpu_ctx *c) {
  if (!c) return PGPU_EINVAL;
  DeviceScope device_scope(c->cfg.device);
  NvtxRange nvtx("pgpu_influence");
  if (!c->frozen) return fail(c, PGPU_EINVAL, "no particles were uploaded");
  int r = check_contiguous(c);
  if (r) return r;
  if (!c->d_field) {
    const cudaError_t e = cudaMalloc((void **)&c->d_field, 6 * (size_t)c->cap * sizeof(double));
    if (e != cudaSuccess) {
      cudaGetLastError();
      c->d_field = nullptr;
      return fail(c, PGPU_ENOMEM, "cudaMalloc of the vorticity field failed: %s", cudaGetErrorString(e));
    }
  }
  // every particle of every system is a target, 256-target tiles
  const int shape = 2, block = 256;
  int64_t tiles = 0;
  std::vector<int> all(c->sys.size());
  for (size_t s = 0; s < all.size(); ++s) {
    all[s] = (int)s;
    tiles += ceil_div(sys_n(c, (int)s), block);
  }
  const int nch = (int)std::max<int64_t>(1, std::min<int64_t>(kMaxChunks, ceil_div(8LL * c->sms, std::max<int64_t>(1, tiles))));
  std::vector<PlanEntry> plan = build_plan(c, all, shape, nch, false);
  plan.resize(c->sys.size() + 1, plan.back());
  CK(cudaMemcpyAsync(c->d_plan_field, plan.data(), plan.size() * sizeof(PlanEntry), cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));  // the plan vector is pageable host memory
  if (plan.size() > 1 && plan.front().n > 0) {
    int grid = 0;
    FieldArgs a{c->x0, c->sig, c->partial, c->d_plan_field, (int)c->sys.size(), nch, c->cap, c->d_counters};
    auto fn = c->cfg.kernel == PGPU_KERNEL_HIGHORDER ? field_kernel<256, kHighOrder> : field_kernel<256, kGaussian>;
    CK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&grid, fn, block, 0));
    fn<<<std::max(1, grid) * c->sms, block, 0, c->st>>>(a);
    CK(cudaGetLastError());
    c->launches++;
  }
  const int rg = (int)std::min<int64_t>(ceil_div(c->cap, 256), 16LL * c->sms);
  field_reduce_kernel<<<rg, 256, 0, c->st>>>(c->partial, nch, c->cap, c->d_field);
  CK(cudaGetLastError());
  c->launches++;
  return PGPU_OK;
}

int pgpu_get_vorticity_field(pgpu_ctx *c, int32_t wake, double *field) {
  int r = wake_ok(c, wake);
  if (r) return r;
  DeviceScope device_scope(c->cfg.device);
  if (!field) return fail(c, PGPU_EINVAL, "null output array");
  if (!c->d_field) return fail(c, PGPU_EINVAL, "no vorticity field was computed (pgpu_influence)");
  const WakeRec &W = c->wakes[wake];
  std::vector<double> zeros(3 * (size_t)W.n);
  return download_rows(c, c->d_field, W, field, zeros.data());
}

int pgpu_set_timing(pgpu_ctx *c, int on) {
  if (!c) return PGPU_EINVAL;
  c->timing = on != 0;
  return PGPU_OK;
}

int pgpu_sync_timeout(pgpu_ctx *c, double seconds) {
  if (!c) return PGPU_EINVAL;
  DeviceScope device_scope(c->cfg.device);
  NvtxRange nvtx("pgpu_sync_timeout");
  const auto t0 = std::chrono::steady_clock::now();
  for (;;) {
    const cudaError_t e = cudaStreamQuery(c->st);
    if (e == cudaSuccess) break;
    if (e != cudaErrorNotReady) return fail(c, PGPU_ECUDA, "cudaStreamQuery failed: %s", cudaGetErrorString(e));
    const double waited = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (waited > seconds)
      return fail(c, PGPU_ETIMEOUT, "the queued work did not finish within %.3f s (it keeps running)", seconds);
    std::this_thread::sleep_for(std::chrono::microseconds(100));
  }
  return pgpu_sync(c);
}

int pgpu_snapshot_begin(pgpu_ctx *c, int32_t slot) {
  NvtxRange nvtx("pgpu_snapshot_begin");
  if (!c) return PGPU_EINVAL;
  DeviceScope device_scope(c->cfg.device);
  if (slot != 0 && slot != 1) return fail(c, PGPU_EINVAL, "snapshot slot %d is not 0 or 1", slot);
  if (!c->frozen) return fail(c, PGPU_EINVAL, "no particles were uploaded");
  if (c->capturing) return fail(c, PGPU_EINVAL, "a snapshot cannot be taken during graph capture");
  const size_t bytes = 6 * (size_t)c->cap * sizeof(double);
  if (!c->st_copy) CK(cudaStreamCreateWithFlags(&c->st_copy, cudaStreamNonBlocking));
  if (!c->d_snap[slot]) {
    if (cudaMalloc(&c->d_snap[slot], std::max<size_t>(bytes, 64)) != cudaSuccess) {
      cudaGetLastError();
      c->d_snap[slot] = nullptr;
      return fail(c, PGPU_ENOMEM, "snapshot buffer of %zu bytes", bytes);
    }
    if (cudaHostAlloc(reinterpret_cast<void **>(&c->h_snap[slot]), std::max<size_t>(bytes, 64), cudaHostAllocDefault) !=
        cudaSuccess) {
      cudaGetLastError();
      c->h_snap[slot] = nullptr;
      cudaFree(c->d_snap[slot]);
      c->d_snap[slot] = nullptr;
      return fail(c, PGPU_ENOMEM, "pinned snapshot buffer of %zu bytes", bytes);
    }
  }
  if (!c->snap_gathered[slot]) CK(cudaEventCreateWithFlags(&c->snap_gathered[slot], cudaEventDisableTiming));
  if (!c->snap_copied[slot]) CK(cudaEventCreateWithFlags(&c->snap_copied[slot], cudaEventDisableTiming));
  // the gather must not overwrite the slot while its previous copy reads it
  if (c->snap_begun[slot]) CK(cudaStreamWaitEvent(c->st, c->snap_copied[slot], 0));
  c->snap_begun[slot] = false;  // until this snapshot is fully queued
  auto &offs = c->snap_off[slot];
  auto &ns = c->snap_n[slot];
  offs.assign(c->wakes.size(), 0);
  ns.assign(c->wakes.size(), 0);
  int64_t total = 0;
  for (size_t w = 0; w < c->wakes.size(); ++w) {
    const WakeRec &W = c->wakes[w];
    offs[w] = total;
    ns[w] = W.n;
    if (W.n > 0) {
      const int grid = (int)std::min<int64_t>(ceil_div(W.n, 256), 16LL * c->sms);
      gather_kernel<<<grid, 256, 0, c->st>>>(c->x0, W.n, W.off, c->cap, c->d_snap[slot] + 6 * total);
      CK(cudaGetLastError());
      c->launches++;
    }
    total += W.n;
  }
  CK(cudaEventRecord(c->snap_gathered[slot], c->st));
  CK(cudaStreamWaitEvent(c->st_copy, c->snap_gathered[slot], 0));
  if (total > 0)
    CK(cudaMemcpyAsync(c->h_snap[slot], c->d_snap[slot], 6 * (size_t)total * sizeof(double), cudaMemcpyDeviceToHost,
                       c->st_copy));
  CK(cudaEventRecord(c->snap_copied[slot], c->st_copy));
  c->snap_begun[slot] = true;
  return PGPU_OK;
}

int pgpu_snapshot_wait(pgpu_ctx *c, int32_t slot, double seconds, const double **state, int64_t *off, int64_t *n,
                       int32_t nwakes) {
  NvtxRange nvtx("pgpu_snapshot_wait");
  if (!c) return PGPU_EINVAL;
  if (slot != 0 && slot != 1) return fail(c, PGPU_EINVAL, "snapshot slot %d is not 0 or 1", slot);
  if (!c->snap_begun[slot]) return fail(c, PGPU_EINVAL, "no snapshot was begun in slot %d", slot);
  if (seconds > 0) {
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
      const cudaError_t e = cudaEventQuery(c->snap_copied[slot]);
      if (e == cudaSuccess) break;
      if (e != cudaErrorNotReady) return fail(c, PGPU_ECUDA, "cudaEventQuery failed: %s", cudaGetErrorString(e));
      const double waited = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      if (waited > seconds)
        return fail(c, PGPU_ETIMEOUT, "snapshot %d did not land within %.3f s (the copy keeps running)", slot, seconds);
      std::this_thread::sleep_for(std::chrono::microseconds(50));
    }
  } else {
    CK(cudaEventSynchronize(c->snap_copied[slot]));
  }
  if (state) *state = c->h_snap[slot];
  const int32_t m = std::min<int32_t>(std::max(nwakes, 0), (int32_t)c->snap_off[slot].size());
  for (int32_t w = 0; w < m; ++w) {
    if (off) off[w] = c->snap_off[slot][w];
    if (n) n[w] = c->snap_n[slot][w];
  }
  return PGPU_OK;
}

int pgpu_pair_kernel_time(pgpu_ctx *c, double *ms, int64_t *launches) {
  if (!c) return PGPU_EINVAL;
  if (ms) *ms = c->pair_ms;
  if (launches) *launches = c->pair_launches;
  c->pair_ms = 0.0;
  c->pair_launches = 0;
  return PGPU_OK;
}

int64_t pgpu_launch_count(pgpu_ctx *c) { return c ? c->launches : -1; }

int pgpu_pair_counts(pgpu_ctx *c, int64_t *pairs, int64_t *full_pairs) {
  if (!c) return PGPU_EINVAL;
  DeviceScope device_scope(c->cfg.device);
  int64_t full = c->pairs_acc;
  // the Gaussian kernel has a far regime in both precisions (and counts its
  // full-formula pairs); the high-order kernel evaluates every pair in full
  if (c->frozen && c->cfg.kernel == PGPU_KERNEL_GAUSSIAN) {
    unsigned long long nf = 0;
    CK(cudaStreamSynchronize(c->st));
    CK(cudaMemcpy(&nf, c->d_nfull, sizeof(nf), cudaMemcpyDeviceToHost));
    CK(cudaMemset(c->d_nfull, 0, sizeof(nf)));
    full = (int64_t)nf - c->selfs_acc;
  }
  if (pairs) *pairs = c->pairs_acc;
  if (full_pairs) *full_pairs = full;
  c->pairs_acc = 0;
  c->selfs_acc = 0;
  return PGPU_OK;
}

int pgpu_kernel_shapes(int *block, int *tpt, int max) {
  for (int s = 0; s < kNumShapes && s < max; ++s) {
    if (block) block[s] = kShapes[s].block;
    if (tpt) tpt[s] = kShapes[s].tpt;
  }
  return kNumShapes;
}

int pgpu_autotune(pgpu_ctx *c, int reps, int *block, int *tpt, double *ms_per_launch) {
  if (!c) return PGPU_EINVAL;
  DeviceScope device_scope(c->cfg.device);
  if (!c->frozen) return fail(c, PGPU_EINVAL, "no particles were uploaded");
  if (reps < 1) reps = 1;
  c->sys_shape.clear();  // one shape for every system from here on
  const int saved = c->shape;
  double best = 1e300;
  int best_s = saved;
  double ms_acc;
  int64_t nl;
  int r = pgpu_pair_kernel_time(c, &ms_acc, &nl);  // reset counters
  for (int s = 0; s < kNumShapes; ++s) {
    c->shape = s;
    c->plan_dirty = true;
    if ((r = upload_plan(c))) return r;
    if ((r = launch_eval(c, 0))) return r;  // warm-up
    if ((r = collect_timing(c, 1))) return r;
    pgpu_pair_kernel_time(c, nullptr, nullptr);
    for (int k = 0; k < reps; ++k) {
      if ((r = launch_eval(c, 0))) return r;
      if ((r = collect_timing(c, 1))) return r;
    }
    double ms;
    pgpu_pair_kernel_time(c, &ms, &nl);
    ms /= reps;
    if (ms_per_launch) ms_per_launch[s] = ms;
    if (ms < best) { best = ms; best_s = s; }
  }
  c->shape = best_s;
  c->plan_dirty = true;
  if ((r = upload_plan(c))) return r;
  // The partial buffer now holds the last candidate's chunks: recompute the
  // rates of the current state with the chosen shape.
  if ((r = pgpu_solve(c))) return r;
  pgpu_pair_kernel_time(c, nullptr, nullptr);
  if (block) *block = kShapes[best_s].block;
  if (tpt) *tpt = kShapes[best_s].tpt;
  return PGPU_OK;
}

}  // extern "C"

namespace {

// Size class of a system of n particles: class 0 holds n < 4096, class k >= 1
// holds [1024 4^k, 1024 4^(k+1)).
int size_class(int64_t n) {
  int k = 0;
  for (int64_t hi = 4096; n >= hi && k < 30; hi *= 4) ++k;
  return k;
}
int64_t class_lo(int k) { return k == 0 ? 0 : (int64_t)1024 << (2 * k); }
int64_t class_hi(int k) { return (int64_t)1024 << (2 * (k + 1)); }

// Device time of one pair launch of `shape` over `systems` (their own plan and
// chunk count), mean of `reps` launches after one untimed.
template <typename T> int time_subset(pgpu_ctx *c, const std::vector<int> &systems, int shape, int reps, double *ms) {
  int r = upload_plan(c);  // system sizes on the device, for the source boxes
  if (r) return r;
  const int nch = choose_nch_for(c, shape, systems);
  std::vector<PlanEntry> plan = build_plan(c, systems, shape, nch);
  plan.resize(c->sys.size() + 1, plan.back());
  // d_plan now holds this subset's plan: the next evaluation rebuilds the
  // context's own, also when the tuning stops early on an error
  c->plan_dirty = true;
  CK(cudaMemcpyAsync(c->d_plan, plan.data(), plan.size() * sizeof(PlanEntry), cudaMemcpyHostToDevice, c->st));
  CK(cudaStreamSynchronize(c->st));
  PairArgs<T> a;
  a.P = static_cast<const v4_t<T> *>(c->P);
  a.Q = static_cast<const v4_t<T> *>(c->Q);
  a.partial = c->partial;
  a.plan = c->d_plan;
  a.nsys = (int)c->sys.size();
  a.nch = nch;
  a.cap = c->cap;
  a.nu2 = (T)(2.0 * c->cfg.nu);
  a.counters = c->d_counters;
  a.nfull = c->d_nfull;
  if (uses_boxes(c)) {
    if ((r = launch_boxes(c))) return r;
    a.box = c->d_box;
  }
  a.L = c->d_L;
  float total = 0.f;
  for (int k = 0; k <= reps; ++k) {
    CK(cudaEventRecord(c->ev[0][0], c->st));
    pair_fn<T>(shape, c->cfg.kernel, uses_split(c))<<<c->grid[shape], kShapes[shape].block, 0, c->st>>>(a);
    CK(cudaGetLastError());
    c->launches++;
    CK(cudaEventRecord(c->ev[0][1], c->st));
    CK(cudaEventSynchronize(c->ev[0][1]));
    float t = 0.f;
    CK(cudaEventElapsedTime(&t, c->ev[0][0], c->ev[0][1]));
    if (k > 0) total += t;
  }
  *ms = total / reps;
  return PGPU_OK;
}

std::string json_str(const std::string &line, const char *key) {
  const std::string k = std::string("\"") + key + "\": \"";
  const size_t p = line.find(k);
  if (p == std::string::npos) return "";
  const size_t e = line.find('"', p + k.size());
  return e == std::string::npos ? "" : line.substr(p + k.size(), e - p - k.size());
}

bool json_num(const std::string &line, const char *key, double *v) {
  const std::string k = std::string("\"") + key + "\": ";
  const size_t p = line.find(k);
  if (p == std::string::npos) return false;
  char *end = nullptr;
  *v = strtod(line.c_str() + p + k.size(), &end);
  return end != line.c_str() + p + k.size();
}

// Times of every shape for one cached class ("ms": [..] of the line).
bool json_ms(const std::string &line, double *ms, int n) {
  const size_t p = line.find("\"ms\": [");
  if (p == std::string::npos) return false;
  const char *q = line.c_str() + p + 7;
  for (int i = 0; i < n; ++i) {
    char *end = nullptr;
    ms[i] = strtod(q, &end);
    if (end == q) return false;
    q = end;
    while (*q == ',' || *q == ' ') ++q;
  }
  return true;
}

}  // namespace

extern "C" {

int pgpu_autotune_classes(pgpu_ctx *c, int reps, const char *cache_path, pgpu_tune_class *classes, int max_classes,
                          int *nclasses, int *per_class) {
  NvtxRange nvtx("pgpu_autotune_classes");
  if (!c) return PGPU_EINVAL;
  DeviceScope device_scope(c->cfg.device);
  if (!c->frozen) return fail(c, PGPU_EINVAL, "no particles were uploaded");
  if (c->sur) return fail(c, PGPU_EINVAL, "the surrogate evaluates one system; use pgpu_autotune");
  if (reps < 1) reps = 1;
  int r = check_contiguous(c);
  if (r) return r;
  // systems by size class
  std::map<int, std::vector<int>> cls;
  for (size_t s = 0; s < c->sys.size(); ++s)
    if (owned(c, (int)s).second > 0) cls[size_class(sys_n(c, (int)s))].push_back((int)s);
  if (cls.empty()) return fail(c, PGPU_EINVAL, "no system has particles");
  cudaDeviceProp prop;
  CK(cudaGetDeviceProperties(&prop, c->cfg.device));
  const std::string gpu = prop.name;
  const std::string prec = fp64(c) ? "fp64" : "fp32c";
  const std::string ker = c->cfg.kernel == PGPU_KERNEL_HIGHORDER ? "highorder" : "gaussian";
  // cached times: the last matching line of the file wins
  std::map<int, std::vector<double>> cached;
  if (cache_path && *cache_path) {
    if (FILE *f = fopen(cache_path, "r")) {
      char buf[2048];
      while (fgets(buf, sizeof(buf), f)) {
        const std::string line(buf);
        double k = -1;
        std::vector<double> ms(kNumShapes);
        if (json_str(line, "gpu") == gpu && json_str(line, "precision") == prec && json_str(line, "kernel") == ker &&
            json_num(line, "class", &k) && json_ms(line, ms.data(), kNumShapes))
          cached[(int)k] = ms;
      }
      fclose(f);
    }
  }
  double ms_acc;
  int64_t nl;
  pgpu_pair_kernel_time(c, &ms_acc, &nl);
  std::vector<int> keys;
  std::vector<std::vector<double>> tms;
  std::vector<int> from_cache;
  for (auto &kv : cls) {
    keys.push_back(kv.first);
    auto it = cached.find(kv.first);
    if (it != cached.end()) {
      tms.push_back(it->second);
      from_cache.push_back(1);
      continue;
    }
    std::vector<double> ms(kNumShapes);
    for (int sh = 0; sh < kNumShapes; ++sh) {
      r = fp64(c) ? time_subset<double>(c, kv.second, sh, reps, &ms[sh]) : time_subset<float>(c, kv.second, sh, reps, &ms[sh]);
      if (r) return r;
    }
    tms.push_back(ms);
    from_cache.push_back(0);
  }
  // fastest shape per class, and the one shape with the least total time
  const size_t K = keys.size();
  std::vector<int> best(K);
  for (size_t i = 0; i < K; ++i)
    best[i] = (int)(std::min_element(tms[i].begin(), tms[i].end()) - tms[i].begin());
  int single = 0;
  double single_t = 1e300;
  for (int sh = 0; sh < kNumShapes; ++sh) {
    double t = 0.0;
    for (size_t i = 0; i < K; ++i) t += tms[i][sh];
    if (t < single_t) { single_t = t; single = sh; }
  }
  // one launch per class shape only if the single shape loses more than 2%
  // on some class
  bool split = false;
  for (size_t i = 0; i < K; ++i)
    if (tms[i][single] > 1.02 * tms[i][best[i]]) split = true;
  if (split) {
    c->sys_shape.assign(c->sys.size(), single);
    for (size_t i = 0; i < K; ++i)
      for (int s : cls[keys[i]]) c->sys_shape[s] = best[i];
  } else {
    c->sys_shape.clear();
    c->shape = single;
  }
  bool cache_failed = false;
  if (cache_path && *cache_path) {
    if (FILE *f = fopen(cache_path, "a")) {
      for (size_t i = 0; i < K; ++i) {
        if (from_cache[i]) continue;
        fprintf(f, "{\"gpu\": \"%s\", \"precision\": \"%s\", \"kernel\": \"%s\", \"class\": %d, \"nmin\": %lld, "
                   "\"nmax\": %lld, \"block\": %d, \"tpt\": %d, \"ms\": [",
                gpu.c_str(), prec.c_str(), ker.c_str(), keys[i], (long long)class_lo(keys[i]),
                (long long)class_hi(keys[i]), kShapes[best[i]].block, kShapes[best[i]].tpt);
        for (int sh = 0; sh < kNumShapes; ++sh) fprintf(f, "%s%.6g", sh ? ", " : "", tms[i][sh]);
        fprintf(f, "]}\n");
      }
      fclose(f);
    } else {
      cache_failed = true;  // reported after the chosen launches are in place
    }
  }
  if (nclasses) *nclasses = (int)K;
  if (per_class) *per_class = split ? 1 : 0;
  for (size_t i = 0; i < K && classes && (int)i < max_classes; ++i) {
    pgpu_tune_class &o = classes[i];
    memset(&o, 0, sizeof(o));
    o.size_class = keys[i];
    o.nmin = class_lo(keys[i]);
    o.nmax = class_hi(keys[i]);
    o.systems = (int32_t)cls[keys[i]].size();
    o.block = kShapes[best[i]].block;
    o.tpt = kShapes[best[i]].tpt;
    o.from_cache = from_cache[i];
    for (int sh = 0; sh < kNumShapes && sh < 8; ++sh) o.ms[sh] = tms[i][sh];
    o.single_block = kShapes[single].block;
    o.single_tpt = kShapes[single].tpt;
  }
  // recompute the rates of the current state with the chosen launches (the
  // partial buffer holds the last candidate's chunks)
  c->plan_dirty = true;
  if ((r = upload_plan(c))) return r;
  if ((r = pgpu_solve(c))) return r;
  pgpu_pair_kernel_time(c, nullptr, nullptr);
  if (cache_failed) return fail(c, PGPU_EINVAL, "cannot append to the autotune cache %s", cache_path);
  return PGPU_OK;
}

int pgpu_get_stream(pgpu_ctx *c, void **stream) {
  if (!c || !stream) return PGPU_EINVAL;
  *stream = (void *)c->st;
  return PGPU_OK;
}

int pgpu_fp32_peaks(int device, double *ffma_tflops, double *ffma2_tflops) {
  pgpu_ctx *c = nullptr;  // for CK's error path
  CK(cudaSetDevice(device));
  int sms = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  float *out = nullptr;
  cudaStream_t st;
  CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  CK(cudaMallocAsync((void **)&out, sizeof(float), st));
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  const int block = 256, grid = sms * 8, iters = 1 << 14;
  // both loops do kFfmaChains FMAs per thread per iteration
  const double flops = 2.0 * kFfmaChains * (double)iters * grid * block;
  for (int packed = 0; packed < 2; ++packed) {
    auto run = [&]() {
      if (packed) ffma2_peak_kernel<<<grid, block, 0, st>>>(out, iters, 0.999f, 1e-3f);
      else ffma_peak_kernel<<<grid, block, 0, st>>>(out, iters, 0.999f, 1e-3f);
    };
    run();  // warm-up
    CK(cudaEventRecord(e0, st));
    run();
    CK(cudaEventRecord(e1, st));
    CK(cudaEventSynchronize(e1));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, e0, e1));
    double *dst = packed ? ffma2_tflops : ffma_tflops;
    if (dst) *dst = flops / (ms * 1e-3) / 1e12;
  }
  cudaFreeAsync(out, st);
  cudaStreamSynchronize(st);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  return PGPU_OK;
}

int pgpu_fp64_peak(int device, double *tflops) {
  pgpu_ctx *c = nullptr;  // for CK's error path
  CK(cudaSetDevice(device));
  int sms = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
  float *out = nullptr;
  cudaStream_t st;
  CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  CK(cudaMallocAsync((void **)&out, sizeof(float), st));
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  const int block = 256, grid = sms * 8, iters = 1 << 12;
  const double flops = 2.0 * kFfmaChains * (double)iters * grid * block;
  dfma_peak_kernel<<<grid, block, 0, st>>>(out, iters, 0.999, 1e-3);  // warm-up
  CK(cudaEventRecord(e0, st));
  dfma_peak_kernel<<<grid, block, 0, st>>>(out, iters, 0.999, 1e-3);
  CK(cudaEventRecord(e1, st));
  CK(cudaEventSynchronize(e1));
  float ms = 0.f;
  CK(cudaEventElapsedTime(&ms, e0, e1));
  if (tflops) *tflops = flops / (ms * 1e-3) / 1e12;
  cudaFreeAsync(out, st);
  cudaStreamSynchronize(st);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(st);
  return PGPU_OK;
}

int pgpu_fp32_peak(int device, double *tflops, double *ms_out) {
  double f1 = 0.0, f2 = 0.0;
  const int r = pgpu_fp32_peaks(device, &f1, &f2);
  if (r) return r;
  if (tflops) *tflops = f1 > f2 ? f1 : f2;
  if (ms_out) *ms_out = 0.0;
  return PGPU_OK;
}

const char *pgpu_last_error(pgpu_ctx *c) { return c ? c->err : g_create_err; }

}  // extern "C"

#include "mlp_host.inc"
#include "surrogate_host.inc"
#include "merge_host.inc"
