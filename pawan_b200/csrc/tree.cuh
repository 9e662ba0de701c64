// Octree of one system for the far-field surrogate (no PAWAN counterpart:
// PAWAN only has the O(N^2) direct sum).
//
// Build, all on the device:
//   1. bounding cube of the system (bbox_kernel)
//   2. 63-bit Morton codes, 21 bits per axis (morton_kernel), sorted with CUB
//   3. sorted copies of the source records (gather_sorted_kernel)
//   4. top-down adaptive split, one level per launch: a cell with more than
//      `leaf` particles is split into its non-empty octants, found by binary
//      search of the sorted codes (split_count_kernel / split_write_kernel;
//      child offsets from an exclusive scan, so the layout is deterministic)
//   5. per-cell moments about the particle centroid (moments_kernel)
//   6. per target leaf, the interaction lists (lists_kernel): a source cell
//      whose centroid is at least `near_widths` cube widths beyond the target
//      leaf's bounding sphere, and whose particles are all at least 4 sigma_ij
//      from the leaf's, is far (evaluated from its moments); a leaf that is not
//      far is near (exact pair sum).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace pgpu {

constexpr int kTreeLevels = 21;
constexpr int kCellFloats = 72;
constexpr int kListStack = 256;
// Smallest u = rho^2 / sigma_ij^2 between any particle of a far cell and any
// of the target leaf (rho >= 4 sigma_ij).  At 4M particles on the coaxial
// rings, u >= 16 / 25 / 36 give the same sampled error (1.4-1.8e-5) and cost
// 846 / 1022 / 1168 ms per evaluation with 256-particle leaves; without the
// test, 128-particle leaves put cells within ~2 sigma in the far field and the
// error grows to 7.5e-3.
constexpr float kFarAccept = 16.f;  // default of pgpu_surrogate_config.far_u

struct TreeCell {
  int start, end;       // sorted particle range
  int first_child;      // index of the first child cell (children are contiguous), -1 for leaves
  int nchild;
  int level;
  int pad;
  unsigned long long prefix;  // Morton prefix of the cell (3 * level bits)
};

// Per-cell data (floats), about the cell's particle centroid c, y = x - c:
//   0-2 c, 3-5 A = sum alpha, 6-14 M[a][b] = sum alpha_a y_b,
//   15-32 Q[a][bc] = sum alpha_a y_b y_c for bc in (00,01,02,11,12,22),
//   33 R = max |y|, 34 w = cube width, 35-37 cube centre, 38 mean sigma^2/2,
//   39 largest sigma^2/2,
//   40-69 T[a][bcd] = sum alpha_a y_b y_c y_d for bcd in (000,001,002,011,012,
//   022,111,112,122,222) (the third moments of the order-3 expansion), 70-71 0.
struct CellData { float v[kCellFloats]; };

__device__ __forceinline__ unsigned f2ord(float f) {
  const unsigned b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ord2f(unsigned u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

// box[0..2] = ordered min, box[3..5] = ordered max (initialised by the host to
// 0xffffffff / 0).
__global__ void bbox_kernel(const float4 *P, int64_t off, int64_t n, unsigned *box) {
  float mn[3] = {3e38f, 3e38f, 3e38f}, mx[3] = {-3e38f, -3e38f, -3e38f};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float4 p = P[off + i];
    mn[0] = fminf(mn[0], p.x); mn[1] = fminf(mn[1], p.y); mn[2] = fminf(mn[2], p.z);
    mx[0] = fmaxf(mx[0], p.x); mx[1] = fmaxf(mx[1], p.y); mx[2] = fmaxf(mx[2], p.z);
  }
  for (int o = 16; o > 0; o >>= 1)
    for (int k = 0; k < 3; ++k) {
      mn[k] = fminf(mn[k], __shfl_down_sync(0xffffffffu, mn[k], o));
      mx[k] = fmaxf(mx[k], __shfl_down_sync(0xffffffffu, mx[k], o));
    }
  if ((threadIdx.x & 31) == 0)
    for (int k = 0; k < 3; ++k) {
      atomicMin(&box[k], f2ord(mn[k]));
      atomicMax(&box[3 + k], f2ord(mx[k]));
    }
}

__device__ __forceinline__ unsigned long long spread21(unsigned long long v) {
  v &= 0x1fffffULL;
  v = (v | (v << 32)) & 0x1f00000000ffffULL;
  v = (v | (v << 16)) & 0x1f0000ff0000ffULL;
  v = (v | (v << 8)) & 0x100f00f00f00f00fULL;
  v = (v | (v << 4)) & 0x10c30c30c30c30c3ULL;
  v = (v | (v << 2)) & 0x1249249249249249ULL;
  return v;
}
__device__ __forceinline__ unsigned compact21(unsigned long long v) {
  v &= 0x1249249249249249ULL;
  v = (v ^ (v >> 2)) & 0x10c30c30c30c30c3ULL;
  v = (v ^ (v >> 4)) & 0x100f00f00f00f00fULL;
  v = (v ^ (v >> 8)) & 0x1f0000ff0000ffULL;
  v = (v ^ (v >> 16)) & 0x1f00000000ffffULL;
  v = (v ^ (v >> 32)) & 0x1fffffULL;
  return (unsigned)v;
}

// geo[0..2] = cube origin, geo[3] = cube edge.
__global__ void morton_kernel(const float4 *P, int64_t off, int64_t n, const float *geo, unsigned long long *code,
                              int *idx) {
  const float s = (float)(1 << 21) / geo[3];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const float4 p = P[off + i];
    const unsigned long long ix = (unsigned long long)min(max((p.x - geo[0]) * s, 0.f), 2097151.f);
    const unsigned long long iy = (unsigned long long)min(max((p.y - geo[1]) * s, 0.f), 2097151.f);
    const unsigned long long iz = (unsigned long long)min(max((p.z - geo[2]) * s, 0.f), 2097151.f);
    code[i] = spread21(ix) | (spread21(iy) << 1) | (spread21(iz) << 2);
    idx[i] = (int)i;
  }
}

__global__ void gather_sorted_kernel(const float4 *P, const float4 *Q, int64_t off, int64_t n, const int *idx,
                                     float4 *Ps, float4 *Qs) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const int j = idx[i];
    Ps[i] = P[off + j];
    Qs[i] = Q[off + j];
  }
}

// First index in [lo, hi) whose code >> shift is >= key.
__device__ __forceinline__ int lower_bound_prefix(const unsigned long long *code, int lo, int hi, int shift,
                                                  unsigned long long key) {
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if ((code[mid] >> shift) < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__device__ __forceinline__ bool splittable(const TreeCell &c, int leaf) {
  return c.end - c.start > leaf && c.level < kTreeLevels;
}

// Number of non-empty octants of every cell of the frontier [f0, f1).
__global__ void split_count_kernel(TreeCell *cells, int f0, int f1, const unsigned long long *code, int leaf,
                                   int *nchild) {
  const int i = f0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= f1) return;
  const TreeCell c = cells[i];
  int k = 0;
  if (splittable(c, leaf)) {
    const int shift = 3 * (kTreeLevels - c.level - 1);
    int lo = c.start;
    for (int o = 0; o < 8; ++o) {
      const int hi = lower_bound_prefix(code, lo, c.end, shift, (c.prefix << 3) + (unsigned long long)(o + 1));
      k += hi > lo;
      lo = hi;
    }
  }
  nchild[i - f0] = k;
}

// Writes the children of every frontier cell at base + offs[i] (exclusive scan of nchild).
__global__ void split_write_kernel(TreeCell *cells, int f0, int f1, const unsigned long long *code, int leaf,
                                   const int *offs, int base) {
  const int i = f0 + blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= f1) return;
  TreeCell c = cells[i];
  if (!splittable(c, leaf)) {
    cells[i].first_child = -1;
    cells[i].nchild = 0;
    return;
  }
  const int shift = 3 * (kTreeLevels - c.level - 1);
  int lo = c.start, w = base + offs[i - f0], k = 0;
  for (int o = 0; o < 8; ++o) {
    const int hi = lower_bound_prefix(code, lo, c.end, shift, (c.prefix << 3) + (unsigned long long)(o + 1));
    if (hi > lo) {
      TreeCell ch;
      ch.start = lo; ch.end = hi; ch.first_child = -1; ch.nchild = 0; ch.level = c.level + 1; ch.pad = 0;
      ch.prefix = (c.prefix << 3) | (unsigned long long)o;
      cells[w + k] = ch;
      ++k;
    }
    lo = hi;
  }
  cells[i].first_child = k ? w : -1;
  cells[i].nchild = k;
}

__device__ __forceinline__ double block_sum_d(double v, double *red) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = 0.0;
  for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r += red[k];
  return r;
}
__device__ __forceinline__ float block_max_f(float v, float *red) {
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_down_sync(0xffffffffu, v, o));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  float r = 0.f;
  for (int k = 0; k < (int)(blockDim.x >> 5); ++k) r = fmaxf(r, red[k]);
  return r;
}

// One CTA per cell: centroid, total strength, first and second moments of
// the strength about the centroid (FP64 sums, stored FP32).
__global__ void moments_kernel(const TreeCell *cells, int ncells, const float4 *Ps, const float4 *Qs, const float *geo,
                               CellData *out) {
  __shared__ double red[32];
  __shared__ float redf[32];
  for (int ci = blockIdx.x; ci < ncells; ci += gridDim.x) {
    const TreeCell c = cells[ci];
    double s[7] = {0, 0, 0, 0, 0, 0, 0};
    for (int i = c.start + threadIdx.x; i < c.end; i += blockDim.x) {
      const float4 p = Ps[i], q = Qs[i];
      s[0] += p.x; s[1] += p.y; s[2] += p.z; s[3] += q.x; s[4] += q.y; s[5] += q.z; s[6] += p.w;
    }
    double t[7];
    for (int k = 0; k < 7; ++k) t[k] = block_sum_d(s[k], red);
    const double cnt = (double)(c.end - c.start);
    const double cx = t[0] / cnt, cy = t[1] / cnt, cz = t[2] / cnt;
    double m[57];
    for (int k = 0; k < 57; ++k) m[k] = 0.0;
    float R = 0.f, H = 0.f;
    for (int i = c.start + threadIdx.x; i < c.end; i += blockDim.x) {
      const float4 p = Ps[i], q = Qs[i];
      H = fmaxf(H, p.w);
      const double y[3] = {p.x - cx, p.y - cy, p.z - cz};
      const double a[3] = {q.x, q.y, q.z};
      R = fmaxf(R, (float)sqrt(y[0] * y[0] + y[1] * y[1] + y[2] * y[2]));
      for (int aa = 0; aa < 3; ++aa) {
        for (int b = 0; b < 3; ++b) m[3 * aa + b] += a[aa] * y[b];
        m[9 + 6 * aa + 0] += a[aa] * y[0] * y[0];
        m[9 + 6 * aa + 1] += a[aa] * y[0] * y[1];
        m[9 + 6 * aa + 2] += a[aa] * y[0] * y[2];
        m[9 + 6 * aa + 3] += a[aa] * y[1] * y[1];
        m[9 + 6 * aa + 4] += a[aa] * y[1] * y[2];
        m[9 + 6 * aa + 5] += a[aa] * y[2] * y[2];
        double *o = m + 27 + 10 * aa;
        o[0] += a[aa] * y[0] * y[0] * y[0];
        o[1] += a[aa] * y[0] * y[0] * y[1];
        o[2] += a[aa] * y[0] * y[0] * y[2];
        o[3] += a[aa] * y[0] * y[1] * y[1];
        o[4] += a[aa] * y[0] * y[1] * y[2];
        o[5] += a[aa] * y[0] * y[2] * y[2];
        o[6] += a[aa] * y[1] * y[1] * y[1];
        o[7] += a[aa] * y[1] * y[1] * y[2];
        o[8] += a[aa] * y[1] * y[2] * y[2];
        o[9] += a[aa] * y[2] * y[2] * y[2];
      }
    }
    double mt[57];
    for (int k = 0; k < 57; ++k) mt[k] = block_sum_d(m[k], red);
    const float Rm = block_max_f(R, redf);
    const float Hm = block_max_f(H, redf);
    if (threadIdx.x == 0) {
      CellData d;
      d.v[0] = (float)cx; d.v[1] = (float)cy; d.v[2] = (float)cz;
      d.v[3] = (float)t[3]; d.v[4] = (float)t[4]; d.v[5] = (float)t[5];
      for (int k = 0; k < 27; ++k) d.v[6 + k] = (float)mt[k];
      d.v[33] = Rm;
      const float w = geo[3] / (float)(1u << c.level);
      d.v[34] = w;
      const unsigned long long pre = c.prefix;
      const unsigned ix = compact21(pre), iy = compact21(pre >> 1), iz = compact21(pre >> 2);
      d.v[35] = geo[0] + (ix + 0.5f) * w;
      d.v[36] = geo[1] + (iy + 0.5f) * w;
      d.v[37] = geo[2] + (iz + 0.5f) * w;
      d.v[38] = (float)(t[6] / cnt);
      d.v[39] = Hm;
      for (int k = 0; k < 30; ++k) d.v[40 + k] = (float)mt[27 + k];
      d.v[70] = 0.f;
      d.v[71] = 0.f;
      out[ci] = d;
    }
    __syncthreads();
  }
}

// Interaction lists of every leaf (one thread per leaf).  pass 0 counts,
// pass 1 writes at the offsets of an exclusive scan of the counts.  Near
// leaves are emitted as runs of the sorted particle order: consecutive near
// leaves whose ranges touch are merged (siblings are visited in octant order,
// which is sorted order, so runs are long).  The stack is bounded
// (kListStack); overflow sets *err, and the caller treats a non-zero *err as a
// failed build.
__global__ void lists_kernel(const TreeCell *cells, const CellData *cd, const int *leaves, int nleaves,
                             float near_widths, float far_u, int pass, int *far_cnt, int *near_cnt, const int *far_off,
                             const int *near_off, int *far_list, int2 *near_runs, int *err) {
  const int li = blockIdx.x * blockDim.x + threadIdx.x;
  if (li >= nleaves) return;
  const int T = leaves[li];
  const TreeCell tc = cells[T];
  const float tx = cd[T].v[0], ty = cd[T].v[1], tz = cd[T].v[2], tR = cd[T].v[33], tH = cd[T].v[39];
  int stack[kListStack];
  int sp = 0;
  stack[sp++] = 0;
  int nf = 0, nn = 0, run_s = -1, run_e = -1;
  const int fo = pass ? far_off[li] : 0, no = pass ? near_off[li] : 0;
  while (sp > 0) {
    const int ci = stack[--sp];
    const TreeCell c = cells[ci];
    const bool contains = c.start <= tc.start && tc.end <= c.end;
    const float dx = cd[ci].v[0] - tx, dy = cd[ci].v[1] - ty, dz = cd[ci].v[2] - tz;
    const float d = sqrtf(dx * dx + dy * dy + dz * dz) - tR;
    // far: beyond near_widths cube widths, and every pair of the two cells at
    // u = rho^2 / sigma_ij^2 >= far_u, so that the Gaussian regularisation
    // the singular-kernel expansion leaves out stays small
    const float gap = d - cd[ci].v[33];
    if (!contains && d >= near_widths * cd[ci].v[34] && gap > 0.f &&
        gap * gap >= far_u * (tH + cd[ci].v[39])) {
      if (pass) far_list[fo + nf] = ci;
      ++nf;
    } else if (c.nchild == 0) {
      if (c.start == run_e) {
        run_e = c.end;
      } else {
        if (run_s >= 0) {
          if (pass) near_runs[no + nn] = make_int2(run_s, run_e);
          ++nn;
        }
        run_s = c.start;
        run_e = c.end;
      }
    } else {
      if (sp + c.nchild > kListStack) {
        atomicExch(err, 1);
        break;
      }
      // push in reverse so the children are visited in octant (sorted) order
      for (int k = c.nchild - 1; k >= 0; --k) stack[sp++] = c.first_child + k;
    }
  }
  if (run_s >= 0) {
    if (pass) near_runs[no + nn] = make_int2(run_s, run_e);
    ++nn;
  }
  if (!pass) {
    far_cnt[li] = nf;
    near_cnt[li] = nn;
  }
}

__global__ void leaf_flags_kernel(const TreeCell *cells, int ncells, int *flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ncells) flag[i] = cells[i].nchild == 0;
}
__global__ void positive_flags_kernel(const int *cnt, int n, int *flag) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) flag[i] = cnt[i] > 0;
}
__global__ void leaf_scatter_kernel(const int *flag, const int *pos, int ncells, int *leaves) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < ncells && flag[i]) leaves[pos[i]] = i;
}

}  // namespace pgpu
