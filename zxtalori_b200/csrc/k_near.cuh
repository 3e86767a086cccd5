// Near-field force pass (src/near.zig, shaders/near.wgsl, shaders/shell.wgsl:18-130,
// shaders/pairs.wgsl:328-427).
//
// A source in the zone only feels orbit points within S3 angle r of it, and those lie within
// r of the zone. Per pass:
//   1. shell: every source's identity image, and for sources near a zone plane ("rim") each
//      image (operator, sign) inside every bisector half-space widened by sin(r + 1e-4);
//      counted, scanned and written in (source, image) order - deterministic sites;
//   2. the sites' stereographic chart box, a grid of sdim^3 cells, a counting sort of the
//      sites into row-major cells with each cell ordered by site index;
//   3. sources counting-sorted along a Hilbert curve of a 64^3 grid (then by index), so
//      consecutive sources are close together;
//   4. one warp per G sources (FP32, G = 2, 4 or 8; 32 in FP64) and slice: the warp's chart box,
//      the cell rows within the chart reach of the cutoff chord, each row's x-run trimmed;
//      runs stream through shared memory 32 sites at a time and the lanes test their
//      sources against each site;
//   5. the slices' partial rows summed in slice order into each source's row.
// Nothing is read back between passes: grid parameters live in device memory.
#pragma once
#include <algorithm>

#include "k_common.cuh"
#include "kernels.h"

namespace zo {

// ------------------------------------------------------------------ 1. shell
// Whether image q (of the normalised source `orig`) lies inside every widened bisector
// half-space (shell.wgsl:19-22; the rim test is done by the caller).
__device__ __forceinline__ bool inside_planes(double4 q, int poff, int planes, bool fp64, double margin) {
  for (int k = 0; k < planes; ++k) {
    const double4 h = fp64 ? c_planes64[poff + k] : to_d4(c_planes32[poff + k]);
    if (dot4(q, h) < -margin) return false;
  }
  return true;
}
// Whether a zone source lies within `margin` of some bisector plane. The planes are taken in
// order of reach and the test stops at the first that reaches no zone point within the
// margin: every later one reaches none either.
__device__ __forceinline__ bool on_rim(double4 orig, int poff, int planes, bool fp64, double margin) {
  for (int r = 0; r < planes; ++r) {
    if ((double)c_plane_reach[poff + r] > margin) break;
    const int k = c_plane_order[poff + r];
    const double4 h = fp64 ? c_planes64[poff + k] : to_d4(c_planes32[poff + k]);
    if (dot4(orig, h) <= margin) return true;
  }
  return false;
}

__device__ __forceinline__ double4 source_d(const float4* q32, const double4* q64, int j, bool fp64) {
  return fp64 ? q64[j] : to_d4(q32[j]);
}

// Classification image of (source, operator k, sign): normalize(orig * normalize(g_k)),
// negated; g is the normalised operator.
__device__ __forceinline__ double4 shell_image(double4 orig, double4 g, bool neg) {
  double4 c = normalize4(qmul(orig, g));
  return neg ? neg4(c) : c;
}

// The group's operators, normalised once per block into shared memory.
__device__ __forceinline__ void unit_operators(double4* g, int off, int order, bool fp64) {
  for (int k = threadIdx.x; k < order; k += blockDim.x) g[k] = normalize4(fp64 ? c_ops64[off + k] : c_ops32[off + k]);
  __syncthreads();
}

// Which images of each source are sites: bit img of a 128-bit mask (img = 2 operator +
// sign; the identity image always), so the write pass needs no second classification, and
// the source's site count.
//
// FP64 mode: one thread per source, FP64 classification (shell.wgsl:19-22 restated).
__global__ void __launch_bounds__(256) k_shell_count64(const double4* __restrict__ q64, int n, int gid, double s_margin,
                                                       uint32_t* __restrict__ counts, uint4* __restrict__ masks) {
  __shared__ double4 g64[60];
  const int off = c_group_offset[gid], order = c_group_order[gid];
  for (int k = threadIdx.x; k < order; k += blockDim.x) g64[k] = normalize4(c_ops64[off + k]);
  __syncthreads();
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int poff = c_plane_offset[gid], planes = 2 * order - 1;
  uint32_t w[4] = {1u, 0u, 0u, 0u};  // the identity image is always a (core) site
  const double margin = s_margin + 2e-6;
  const double4 orig = normalize4(q64[j]);
  if (on_rim(orig, poff, planes, true, margin)) {
    for (int img = 1; img < 2 * order; ++img) {
      const double4 y = shell_image(orig, g64[img / 2], img & 1);
      // Plane img - 1 (the bisector of the identity and the image's own operator) rejects
      // almost every image far from the zone: test it first.
      if (y.x > -0.9999999 && dot4(y, c_planes64[poff + img - 1]) >= -margin &&
          inside_planes(y, poff, planes, true, margin))
        w[img >> 5] |= 1u << (img & 31);
    }
  }
  counts[j] = (uint32_t)(__popc(w[0]) + __popc(w[1]) + __popc(w[2]) + __popc(w[3]));
  masks[j] = make_uint4(w[0], w[1], w[2], w[3]);
}

// FP32 mode, in FP32 with the float32 planes: rounding moves a decision only within ~1e-7
// of the widened plane, while the margin, sin(r + 1e-4) + 2e-6, leaves 1e-4 rad between it
// and any site a zone source can reach within r. Three steps, so that the few rim sources'
// images spread over whole warps: (1) the rim test per source, listing the rim sources and
// their positions; (2) a warp per rim source, its lanes over the images, setting the mask
// bit of each site; (3) the counts.
__global__ void __launch_bounds__(256) k_shell_rim32(const float4* __restrict__ q32, int n, int gid, float margin,
                                                     uint4* __restrict__ masks, uint32_t* __restrict__ rim_list,
                                                     float4* __restrict__ rim_q, uint32_t* __restrict__ rim_count) {
  const unsigned full = 0xffffffffu;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  bool rim = false;
  float4 orig = make_float4(1.f, 0.f, 0.f, 0.f);
  if (j < n) {
    const int poff = c_plane_offset[gid], planes = 2 * c_group_order[gid] - 1;
    orig = q32[j];  // unit to 1e-7 (folded in FP64), far inside the margin's slack
    // Planes in order of reach, up to the first that no zone point comes within the margin
    // of (for I at small cutoffs, the 12 faces of the zone instead of 119 planes).
    for (int r = 0; r < planes && !rim; ++r) {
      if (c_plane_reach[poff + r] > margin) break;
      const float4 h = c_planes32[poff + c_plane_order[poff + r]];
      rim = fmaf(orig.x, h.x, fmaf(orig.y, h.y, fmaf(orig.z, h.z, orig.w * h.w))) <= margin;
    }
    masks[j] = make_uint4(1u, 0u, 0u, 0u);  // the identity image is always a (core) site
  }
  const unsigned m = __ballot_sync(full, rim);  // one atomic per warp for its rim sources
  if (m) {
    const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(rim_count, (uint32_t)__popc(m));
    base = __shfl_sync(full, base, leader);
    if (rim) {
      const uint32_t at = base + (uint32_t)__popc(m & ((1u << lane) - 1u));
      rim_list[at] = (uint32_t)j;
      rim_q[at] = orig;
    }
  }
}

__global__ void __launch_bounds__(256) k_shell_classify32(int gid, float margin, const uint32_t* __restrict__ rim_list,
                                                          const float4* __restrict__ rim_q,
                                                          const uint32_t* __restrict__ rim_count, uint4* masks) {
  // The group's operators and planes in shared memory: lanes read different ones at once,
  // which constant memory would serialise.
  __shared__ float4 g32[60];
  __shared__ float4 h32[119];
  const int off = c_group_offset[gid], order = c_group_order[gid];
  const int poff = c_plane_offset[gid], planes = 2 * order - 1;
  for (int k = threadIdx.x; k < order; k += blockDim.x) g32[k] = to_f4(normalize4(c_ops32[off + k]));
  for (int k = threadIdx.x; k < planes; k += blockDim.x) h32[k] = c_planes32[poff + k];
  __syncthreads();
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const uint32_t rims = *rim_count;
  auto plane_dot = [&](const float4& y, int k) {
    const float4 h = h32[k];
    return fmaf(y.x, h.x, fmaf(y.y, h.y, fmaf(y.z, h.z, y.w * h.w)));
  };
  // One warp per rim source (grid-stride), its lanes over the images 1 .. 2|K|-1, 32 at a
  // time. Image img = 2j + sign of x is y = +-x g_j, and plane img - 1 is the bisector of the
  // identity and +-g_j: its dot with y is proportional to y_w - x_w, negative unless y lies
  // near the zone. Each lane tests that plane alone; the few images that pass are checked
  // against every plane by the whole warp together.
  for (uint32_t r = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; r < rims; r += (gridDim.x * blockDim.x) >> 5) {
    const float4 a = rim_q[r];
    uint32_t* word = reinterpret_cast<uint32_t*>(&masks[rim_list[r]]);
    for (int base = 1; base < 2 * order; base += 32) {
      const int img = base + lane;
      float4 y = make_float4(0.f, 0.f, 0.f, 0.f);
      bool alive = false;
      if (img < 2 * order) {
        const float4 b = g32[img / 2];
        y = make_float4(a.x * b.x - a.y * b.y - a.z * b.z - a.w * b.w, a.x * b.y + a.y * b.x + a.z * b.w - a.w * b.z,
                        a.x * b.z - a.y * b.w + a.z * b.x + a.w * b.y, a.x * b.w + a.y * b.z - a.z * b.y + a.w * b.x);
        if (img & 1) y = make_float4(-y.x, -y.y, -y.z, -y.w);
        alive = y.x > -0.9999999f && plane_dot(y, img - 1) >= -margin;
      }
      unsigned survivors = __ballot_sync(full, alive);
      while (survivors) {
        const int src = __ffs(survivors) - 1;
        survivors &= survivors - 1;
        const float4 z = make_float4(__shfl_sync(full, y.x, src), __shfl_sync(full, y.y, src),
                                     __shfl_sync(full, y.z, src), __shfl_sync(full, y.w, src));
        bool out = false;
        for (int k = lane; k < planes; k += 32) out |= plane_dot(z, k) < -margin;
        if (!__any_sync(full, out) && lane == src) atomicOr(word + (img >> 5), 1u << (img & 31));
      }
    }
  }
}

__global__ void k_shell_popc(const uint4* __restrict__ masks, int n, uint32_t* __restrict__ counts) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const uint4 w = masks[j];
  counts[j] = (uint32_t)(__popc(w.x) + __popc(w.y) + __popc(w.z) + __popc(w.w));
}

// The shell's masks and counts (all three FP32 steps, or the FP64 kernel); returns the
// number of kernels launched through `launches`.
inline cudaError_t launch_shell_masks(int prec, const float4* q32, const double4* q64, int n, int gid,
                                      double s_margin, uint32_t* counts, uint4* masks, uint32_t* rim_list,
                                      float4* rim_q, uint32_t* rim_count, cudaStream_t s, int* launches) {
  if (prec == kFP64) {
    k_shell_count64<<<(n + 255) / 256, 256, 0, s>>>(q64, n, gid, s_margin, counts, masks);
    *launches = 1;
    return cudaGetLastError();
  }
  const float margin = (float)(s_margin + 2e-6);
  cudaError_t e = cudaMemsetAsync(rim_count, 0, sizeof(uint32_t), s);
  if (e) return e;
  k_shell_rim32<<<(n + 255) / 256, 256, 0, s>>>(q32, n, gid, margin, masks, rim_list, rim_q, rim_count);
  const int blocks = std::min((n + 7) / 8, 4096);  // a warp per rim source, at most n of them
  k_shell_classify32<<<blocks, 256, 0, s>>>(gid, margin, rim_list, rim_q, rim_count, masks);
  k_shell_popc<<<(n + 255) / 256, 256, 0, s>>>(masks, n, counts);
  *launches = 3;
  return cudaGetLastError();
}

// Writes the sites of each source at its scanned offset: the rebuilt image quaternion
// (pairs.wgsl:181 / near.wgsl:263-269), its code (source, high bit for the identity
// image), its image number 2*operator+sign, and its chart position; plus the chart box.
// The images are those k_shell_count recorded in the source's mask.
template <bool FP64>
__global__ void __launch_bounds__(256) k_shell_write(const float4* __restrict__ q32, const double4* __restrict__ q64,
                                                     int n, int gid, const uint4* __restrict__ masks,
                                                     const uint32_t* __restrict__ offsets, int capacity,
                                                     float4* __restrict__ site_q32, double4* __restrict__ site_q64,
                                                     uint4* __restrict__ site_meta, float4* __restrict__ site_pos,
                                                     NearGrid* grid) {
  __shared__ double4 g[60];
  const int off = c_group_offset[gid], order = c_group_order[gid];
  unit_operators(g, off, order, FP64);
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  float lo[3] = {3e38f, 3e38f, 3e38f}, hi[3] = {-3e38f, -3e38f, -3e38f};
  bool overflow = false;
  if (j < n) {
    const double4 src = source_d(q32, q64, j, FP64);
    const double4 orig = normalize4(src);
    uint32_t at = offsets[j];
    auto emit = [&](double4 cls, int img, bool identity) {
      if ((int)at >= capacity) {
        overflow = true;
        return;
      }
      const float3 p = chart(cls);
      if (FP64) {
        double4 y = identity ? src : (img / 2 == 0 ? src : normalize4(qmul(src, c_ops64[off + img / 2])));
        site_q64[at] = (img & 1) ? neg4(y) : y;
      } else {
        const float4 s = q32[j];
        float4 y = (img / 2 == 0) ? s : to_f4(normalize4(qmul(to_d4(s), c_ops32[off + img / 2])));
        if (img & 1) y = make_float4(-y.x, -y.y, -y.z, -y.w);
        site_q32[at] = y;
      }
      // What the sorted copy needs of the site in one 16-byte record (one random read there).
      site_meta[at] = make_uint4((uint32_t)j | (identity ? kIdentityBit : 0u), (uint32_t)img, __float_as_uint(p.x), 0u);
      site_pos[at] = make_float4(p.x, p.y, p.z, 0.f);
      lo[0] = fminf(lo[0], p.x);
      lo[1] = fminf(lo[1], p.y);
      lo[2] = fminf(lo[2], p.z);
      hi[0] = fmaxf(hi[0], p.x);
      hi[1] = fmaxf(hi[1], p.y);
      hi[2] = fmaxf(hi[2], p.z);
      ++at;
    };
    const uint4 m = masks[j];
    const uint32_t words[4] = {m.x, m.y, m.z, m.w};
    emit(orig, 0, true);
    for (int w = 0; w < 4; ++w) {
      uint32_t b = words[w] & (w == 0 ? ~1u : ~0u);
      while (b) {
        const int img = 32 * w + __ffs(b) - 1;
        b &= b - 1;
        emit(shell_image(orig, g[img / 2], img & 1), img, false);
      }
    }
  }
  // Block-reduce the box, then one atomic per block and axis.
  __shared__ float red[6][8];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (int a = 0; a < 3; ++a) {
    const float l = warp_min(lo[a]), h = warp_max(hi[a]);
    if (lane == 0) {
      red[a][w] = l;
      red[3 + a][w] = h;
    }
  }
  const int any_overflow = __syncthreads_or(overflow);
  if (threadIdx.x < 3) {
    float l = red[threadIdx.x][0], h = red[3 + threadIdx.x][0];
    for (int k = 1; k < (int)(blockDim.x >> 5); ++k) {
      l = fminf(l, red[threadIdx.x][k]);
      h = fmaxf(h, red[3 + threadIdx.x][k]);
    }
    if (l <= h) {
      atomicMin(&grid->box_bits[threadIdx.x], ordered_bits(l));
      atomicMax(&grid->box_bits[3 + threadIdx.x], ordered_bits(h));
    }
  }
  if (threadIdx.x == 0 && any_overflow) atomicOr(&grid->overflow, 1u);
}

// ------------------------------------------------------------------ 2. grid and site sort
// Chart grid from the box (near.zig:124-137): a 5% margin, width 1.1x the largest extent,
// sdim = clamp(round(cbrt(sites/kSitesPerCell)), 1, sdim_max). The reference aims at 8 sites
// per cell; fewer trims the candidate runs closer to the cutoff ball (the FP32 gather
// concatenates runs, so short rows cost nothing extra).
// The box is reset for the next pass.
__global__ void k_grid_setup(NearGrid* g, const uint32_t* __restrict__ total, int capacity, int sdim_max,
                             float sites_per_cell, int* __restrict__ cells) {
  const uint32_t s = *total;
  g->sites = (int)min((uint32_t)capacity, s);
  if (s > (uint32_t)capacity) g->overflow = 1u;
  float lo[3], hi[3];
  float width = 1e-6f;
  for (int a = 0; a < 3; ++a) {
    lo[a] = unordered_bits(g->box_bits[a]);
    hi[a] = unordered_bits(g->box_bits[3 + a]);
    if (!(hi[a] >= lo[a])) lo[a] = hi[a] = 0.f;
    width = fmaxf(width, hi[a] - lo[a]);
  }
  for (int a = 0; a < 3; ++a) g->lower[a] = lo[a] - 0.05f * width;
  width *= 1.1f;
  int sdim = (int)rint(cbrt((double)g->sites / sites_per_cell));
  sdim = max(1, min(sdim, sdim_max));
  g->width = width;
  g->sdim = sdim;
  g->cells_per_unit = (float)sdim / width;
  g->order_per_unit = (float)kOrderDim / width;
  *cells = sdim * sdim * sdim;
  for (int a = 0; a < 3; ++a) {
    g->box_bits[a] = 0xffffffffu;
    g->box_bits[3 + a] = 0u;
  }
}

__device__ __forceinline__ int cell_axis(float v, float lower, float per_unit, int dim) {
  const float c = floorf((v - lower) * per_unit);
  return (int)fminf(fmaxf(c, 0.f), (float)(dim - 1));
}

__global__ void k_cell_count(const float4* __restrict__ pos, const NearGrid* __restrict__ gp, uint32_t* __restrict__ cell,
                             uint32_t* __restrict__ rank, uint32_t* __restrict__ counts) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= gp->sites) return;
  const float4 p = pos[s];
  const int d = gp->sdim;
  const float u = gp->cells_per_unit;
  const int c = cell_axis(p.x, gp->lower[0], u, d) + d * (cell_axis(p.y, gp->lower[1], u, d) + d * cell_axis(p.z, gp->lower[2], u, d));
  cell[s] = (uint32_t)c;
  rank[s] = atomicAdd(&counts[c], 1u);
}

__global__ void k_scatter(const uint32_t* __restrict__ key, const uint32_t* __restrict__ rank,
                          const uint32_t* __restrict__ offsets, int max_items, const int* __restrict__ items,
                          uint32_t* __restrict__ perm) {
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  const int count = items ? min(*items, max_items) : max_items;
  if (s >= count) return;
  perm[offsets[key[s]] + rank[s]] = (uint32_t)s;
}

// Each bucket's items in a fixed order, so every pass sums in the same order: by index
// (near.wgsl:270-282), or with `pos` by chart x and then index (a cell row's sites are then
// sorted along x, and the walk trims its runs to the balls' x extent). Insertion sort;
// buckets hold a handful of items on average.
__device__ __forceinline__ bool sorts_before(uint32_t a, uint32_t b, const float4* __restrict__ pos) {
  if (pos) {
    const float xa = pos[a].x, xb = pos[b].x;
    if (xa != xb) return xa < xb;
  }
  return a < b;
}
__global__ void k_bucket_sort(const uint32_t* __restrict__ offsets, int max_buckets, const int* __restrict__ buckets,
                              uint32_t* __restrict__ perm, const float4* __restrict__ pos = nullptr) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  const int count = buckets ? min(*buckets, max_buckets) : max_buckets;
  if (b >= count) return;
  const uint32_t begin = offsets[b], end = offsets[b + 1];
  for (uint32_t at = begin + 1; at < end; ++at) {
    const uint32_t v = perm[at];
    uint32_t k = at;
    while (k > begin && sorts_before(v, perm[k - 1], pos)) {
      perm[k] = perm[k - 1];
      --k;
    }
    perm[k] = v;
  }
}

// The sites in sorted order: position, code, image number and chart x of sorted site p from
// unsorted site perm[p] (two random reads: the position and the 16-byte record).
template <bool FP64>
__global__ void k_site_gather(const uint32_t* __restrict__ perm, const NearGrid* __restrict__ gp,
                              const float4* __restrict__ q32, const double4* __restrict__ q64,
                              const uint4* __restrict__ meta, float4* __restrict__ sq32, double4* __restrict__ sq64,
                              uint32_t* __restrict__ scode, uint32_t* __restrict__ simg, float* __restrict__ sx) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= gp->sites) return;
  const uint32_t s = perm[p];
  if (FP64) sq64[p] = q64[s];
  else sq32[p] = q32[s];
  const uint4 m = meta[s];
  scode[p] = m.x;
  simg[p] = m.y;
  sx[p] = __uint_as_float(m.z);
}

// ------------------------------------------------------------------ 3. sources in Hilbert order
// Index of cell (x, y, z) along the Hilbert curve of a 2^bits grid: J. Skilling's transpose
// algorithm ("Programming the Hilbert curve", AIP Conf. Proc. 707, 381, 2004), the three
// transposed words then interleaved most significant bit first. Consecutive indices are
// face-adjacent cells, so 32 consecutive sources (one warp) form a compact blob; a Morton
// order (the reference's, near.wgsl:224-229) jumps at every power-of-two boundary.
__device__ __forceinline__ uint32_t hilbert3(uint32_t x, uint32_t y, uint32_t z, int bits) {
  uint32_t X[3] = {x, y, z};
  const uint32_t m = 1u << (bits - 1);
  for (uint32_t q = m; q > 1; q >>= 1) {
    const uint32_t p = q - 1;
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      if (X[i] & q) {
        X[0] ^= p;
      } else {
        const uint32_t t = (X[0] ^ X[i]) & p;
        X[0] ^= t;
        X[i] ^= t;
      }
    }
  }
  X[1] ^= X[0];
  X[2] ^= X[1];
  uint32_t t = 0;
  for (uint32_t q = m; q > 1; q >>= 1)
    if (X[2] & q) t ^= q - 1;
  uint32_t h = 0;
  for (int b = bits - 1; b >= 0; --b)
    h = (h << 3) | ((((X[0] ^ t) >> b) & 1u) << 2) | ((((X[1] ^ t) >> b) & 1u) << 1) | (((X[2] ^ t) >> b) & 1u);
  return h;
}

template <bool FP64>
__global__ void k_source_count(const float4* __restrict__ q32, const double4* __restrict__ q64, int n,
                               const NearGrid* __restrict__ gp, uint32_t* __restrict__ code,
                               uint32_t* __restrict__ rank, uint32_t* __restrict__ counts) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float3 p = FP64 ? chart(q64[i]) : chart(q32[i]);
  const float u = gp->order_per_unit;
  const uint32_t cx = cell_axis(p.x, gp->lower[0], u, kOrderDim), cy = cell_axis(p.y, gp->lower[1], u, kOrderDim),
                 cz = cell_axis(p.z, gp->lower[2], u, kOrderDim);
  const uint32_t m = hilbert3(cx, cy, cz, kOrderBits);
  code[i] = m;
  rank[i] = atomicAdd(&counts[m], 1u);
}

// ------------------------------------------------------------------ 4. the gather
inline NearCut near_cut(double cut2, double chord, double cut_z, double cut_w) {
  const double r = cut_z + 1.0 / cut_w;
  const double s = 2.0 * std::sin(0.5 * std::min(1.25 * r, 1.5));
  return NearCut{cut2, chord, cut_z, cut_w, s * s, cut2};
}

// Bound on |FP32 chord^2 - FP64 chord^2| of a source x and a site y of the FP32 gather, at
// chord^2 d, against the oracle's definition (unit x and y formed in FP64). The gather
// reads x as stored (float32, |x| = 1 within 2^-24) and y as the float32 rounding of the
// FP64 image (within 2^-24 per component), and forms |x - y|^2 with four FP32 roundings:
//   |x - y|^2 - |x^ - y^|^2 <= 2 |m| 2^-24 + 2^-24 d + (2^-23)^2, m = x^ - y^, |m|^2 = d,
//   FP32 differences and the sum of squares add at most 6 2^-24 d.
// That is 4.2e-7 d + 1.2e-7 sqrt(d) + 1.5e-14; the bound below is 2.4 times it.
__host__ __device__ __forceinline__ double chord_error32(double d) {
  return 1e-6 * d + 3e-7 * sqrt(fmax(d, 0.0)) + 1e-13;
}

constexpr int kNearWarps = 4;

struct WarpBox {
  float lo[3], hi[3];
  int clo[3], chi[3];
  float d;
};

// The warp's chart box and the cells within chart reach d of it (pairs.wgsl:368-379):
// chart distance = chord/2 sqrt((1+|p|^2)(1+|p'|^2)), bounded by fixed-point iteration from
// below. When the cutoff is wide (C2 at small N, r near 1.5) the iteration has no fixed point
// and four steps fall short; then the bound with |p'| at the chart box's farthest corner
// (every site lies in the box) is used instead.
__device__ __forceinline__ bool warp_box(float3 pos, bool live, const NearGrid& g, float chord, WarpBox& b) {
  float v[6] = {live ? pos.x : 3e38f, live ? pos.y : 3e38f, live ? pos.z : 3e38f,
                live ? pos.x : -3e38f, live ? pos.y : -3e38f, live ? pos.z : -3e38f};
  for (int a = 0; a < 3; ++a) {
    b.lo[a] = warp_min(v[a]);
    b.hi[a] = warp_max(v[3 + a]);
  }
  if (!(b.lo[0] <= b.hi[0])) return false;
  float r2 = 0.f;
  for (int a = 0; a < 3; ++a) {
    const float m = fmaxf(fabsf(b.lo[a]), fabsf(b.hi[a]));
    r2 += m * m;
  }
  const float reach = sqrtf(r2), lift = 1.0f + reach * reach;
  float d = 0.5f * chord * lift;
  for (int k = 0; k < 4; ++k) d = 0.5f * chord * sqrtf(lift * (1.0f + (reach + d) * (reach + d)));
  if (0.5f * chord * sqrtf(lift * (1.0f + (reach + d) * (reach + d))) > d * 1.001f) {
    float p2 = 0.f;
    for (int a = 0; a < 3; ++a) {
      const float m = fmaxf(fabsf(g.lower[a]), fabsf(g.lower[a] + g.width));
      p2 += m * m;
    }
    d = 0.5f * chord * sqrtf(lift * (1.0f + p2));
  }
  d = d * 1.01f + 1e-6f;
  b.d = d;
  for (int a = 0; a < 3; ++a) {
    b.clo[a] = cell_axis(b.lo[a] - d, g.lower[a], g.cells_per_unit, g.sdim);
    b.chi[a] = cell_axis(b.hi[a] + d, g.lower[a], g.cells_per_unit, g.sdim);
  }
  return true;
}

// Row r of the warp's (y, z) cell rows: the run of sorted sites of its x cells within reach.
__device__ __forceinline__ bool row_run(const WarpBox& b, const NearGrid& g, const uint32_t* cell_off, int r,
                                        uint32_t& start, uint32_t& end) {
  const int ny = b.chi[1] - b.clo[1] + 1;
  const int y = b.clo[1] + r % ny, z = b.clo[2] + r / ny;
  const float width = 1.0f / g.cells_per_unit;
  const float cy = g.lower[1] + (float)y * width, cz = g.lower[2] + (float)z * width;
  const float gy = fmaxf(0.f, fmaxf(cy - b.hi[1], b.lo[1] - (cy + width)));
  const float gz = fmaxf(0.f, fmaxf(cz - b.hi[2], b.lo[2] - (cz + width)));
  const float rest = b.d * b.d - gy * gy - gz * gz;
  if (rest < 0.f) return false;
  const float span = sqrtf(rest);
  const int x0 = cell_axis(b.lo[0] - span, g.lower[0], g.cells_per_unit, g.sdim);
  const int x1 = cell_axis(b.hi[0] + span, g.lower[0], g.cells_per_unit, g.sdim);
  const int row = g.sdim * (y + g.sdim * z);
  start = cell_off[row + x0];
  end = cell_off[row + x1 + 1];
  return start < end;
}

// The gather (pairs.wgsl:363-416). A warp holds G sources (consecutive along the
// Hilbert order), each on 32 / G lanes that split its sites between
// them. The warp walks the cell rows that its sources' chart balls reach 32 rows at a time,
// one lane per row finding the row's run of sorted sites; the runs are concatenated and
// streamed through shared memory in tiles of kNearTile sites, and every lane evaluates its
// source against kNearTile G / 32 sites of each tile, two per instruction with packed
// FP32 arithmetic. For cutoffs up to 0.4 rad the windowed pair is a function of the chord
// alone (near_chord_pair32x2); wider ones use dp2 = 2(|x|^2+|y|^2) - dm2 (parallelogram
// law; the site is the near twin). Sites beyond the cutoff contribute exactly zero through
// the window, and the nearest chord is taken over every site and reset to 4 when it exceeds
// the cutoff (no site within it), which is the same as testing each site. The force is kept
// as sum c (x - y), turned into a force once per source. Lane sums are FP32 over 32 sites,
// then FP64; the lanes of a source are added in lane order at the end. With one slice each
// warp writes its sources' rows in place; the spacing pass runs a nearest-only variant.
//
// The tile shape is a template parameter G, the sources per warp (2, 4 or 8; 4 unless the
// tile table picks another for the sample's group and size): G sources on 32 / G lanes each.
constexpr int kNearTile = 128;  // sites per tile
template <int G>
struct NearShape {
  static_assert(G == 2 || G == 4 || G == 8, "sources per warp");
  static constexpr int sub = 32 / G;                           // lanes per source
  static constexpr int slots = kNearTile / (2 * sub);         // site pairs per lane and tile
  static constexpr int merge = slots >= 16 ? 1 : 16 / slots;  // tiles between FP64 merges
};

// One tile. Slot u holds elements 2u and 2u + 1; lane (source s, sub-lane j) evaluates
// slots j + sub m, m < slots. NORM: the arctangent form reads the sites' norms; AT: a pass
// that tracks the nearest site reads their indices (the other variants keep one element of
// each).
template <bool NORM, bool AT>
struct NearTile {
  float4 wx[kNearTile / 2];              // (w, w', x, x')
  float4 yz[kNearTile / 2];              // (y, y', z, z')
  float2 norm[NORM ? kNearTile / 2 : 1];  // (2|y|^2, 2|y'|^2)
  uint2 code[kNearTile / 2];             // (code, code')
  uint32_t at[AT ? kNearTile : 1];       // sorted-site index of each element
};
// Per-warp data of the row walk, kept in shared memory (it is warp-uniform) so the hot
// loop's registers go to the pair arithmetic. Stereographic projection maps spheres to
// spheres: the sites within the cutoff of source x (x . y >= k, k = 1 - cut2/2) are the
// chart points within rho = sqrt(1 - k^2) / (x_w + k) of c = x_v / (x_w + k) (exactly, for
// a unit x and k > -x_w). The walk covers the union of its sources' balls.
template <int G>
struct NearWalk {
  float cen[G][3];
  float rad[G];      // < 0: no source in this place
  uint32_t src[G];   // the sources' indices (codes' low bits); 0xfffffffe when absent
  int clo[3], chi[3];     // cells of the balls' bounding box
  float lower[3], cells_per_unit;
  int sdim;
  uint2 runs[32];  // a batch's nonempty row runs (start, length), compacted
};

// Row r of the walk's (y, z) cell rows: the run of sorted sites of the x cells that some
// source's ball reaches in this row.
template <int G>
__device__ __forceinline__ bool walk_row(const NearWalk<G>& W, const uint32_t* cell_off, const float* site_x, int r,
                                         uint32_t& start, uint32_t& end) {
  const int ny = W.chi[1] - W.clo[1] + 1;
  const int y = W.clo[1] + r % ny, z = W.clo[2] + r / ny;
  const float width = 1.0f / W.cells_per_unit;
  const float cy = W.lower[1] + (float)y * width, cz = W.lower[2] + (float)z * width;
  float x0 = 3e38f, x1 = -3e38f;
#pragma unroll
  for (int s = 0; s < G; ++s) {
    const float rho = W.rad[s];
    if (rho < 0.f) continue;
    const float gy = fmaxf(0.f, fmaxf(cy - W.cen[s][1], W.cen[s][1] - (cy + width)));
    const float gz = fmaxf(0.f, fmaxf(cz - W.cen[s][2], W.cen[s][2] - (cz + width)));
    const float rest = rho * rho - gy * gy - gz * gz;
    if (rest < 0.f) continue;
    const float span = sqrtf(rest);
    x0 = fminf(x0, W.cen[s][0] - span);
    x1 = fmaxf(x1, W.cen[s][0] + span);
  }
  if (!(x0 <= x1)) return false;
  const int c0 = cell_axis(x0, W.lower[0], W.cells_per_unit, W.sdim);
  const int c1 = cell_axis(x1, W.lower[0], W.cells_per_unit, W.sdim);
  const int row = W.sdim * (y + W.sdim * z);
  start = cell_off[row + c0];
  end = cell_off[row + c1 + 1];
  // Each cell's sites are sorted by chart x: drop those of the end cells outside [x0, x1],
  // widened by 2e-6 (chart coordinates are below 2 here, so that is many FP32 roundings of
  // a site's x and of the span) on top of the balls' own 0.1% + 1e-6.
  const float lo_x = x0 - 2e-6f, hi_x = x1 + 2e-6f;
  const uint32_t first_end = cell_off[row + c0 + 1], last_begin = cell_off[row + c1];
  while (start < first_end && site_x[start] < lo_x) ++start;
  while (end > last_begin && end > start && site_x[end - 1] > hi_x) --end;
  return start < end;
}

// Adds a lane's FP32 sums into its FP64 sums in shared memory and clears them.
__device__ __forceinline__ void merge_sums(double (*sums)[kNearWarps * 32], float2& sw, float2& sx, float2& sy,
                                           float2& sz, float2& sc, float2& se) {
  sums[0][threadIdx.x] += (double)sw.x + (double)sw.y;
  sums[1][threadIdx.x] += (double)sx.x + (double)sx.y;
  sums[2][threadIdx.x] += (double)sy.x + (double)sy.y;
  sums[3][threadIdx.x] += (double)sz.x + (double)sz.y;
  sums[4][threadIdx.x] += (double)sc.x + (double)sc.y;
  sums[5][threadIdx.x] += (double)se.x + (double)se.y;
  sw = sx = sy = sz = sc = se = splat(0.f);
}

// The slots of one tile for one lane of k_near32: slot u = sub + (32 / G) m holds elements
// 2u and 2u + 1. No branches in the slot: sites past the batch's end are blank and sites
// beyond the cutoff contribute zero, so every slot runs the same arithmetic and the compiler
// can overlap consecutive slots. OWN: the tile may hold images of the warp's sources, so
// each site's source is tested (the thread's own source gets no force from its images, and
// its identity image is no neighbour); without it that test is left out. SHORT: cutoffs up
// to 0.4 rad take the chord form (near_chord_pair32x2), wider ones the arctangent of near
// over far. se sums energy / pi. NEAREST: only the nearest site is tracked.
// COUNT (a diagnostic pass only): the lane also counts the sites it evaluates (candidates)
// and those inside the cutoff that exert a force (in).
template <int G, bool TRACK, bool SHORT, bool OWN, bool NEAREST, bool COUNT, class Tile>
__device__ __forceinline__ void near_slots(const Tile& T, int count, int sub, uint32_t i, float2 xw, float2 xx,
                                           float2 xy, float2 xz, float2 xn, float cut_hi, float cw, float czw,
                                           float pk, float2& sw, float2& sx, float2& sy, float2& sz, float2& sc,
                                           float2& se, float& best, int& best_at, float& second, float cut2,
                                           uint32_t& candidates, uint32_t& in) {
  constexpr int kSub = NearShape<G>::sub;
#pragma unroll
  for (int m = 0; m < NearShape<G>::slots; ++m) {
    // Slots m.. hold elements from 2 kSub m on; in a batch's last tile (count < 128) the
    // warp stops at a 32-element boundary once they are all blank (count is warp-uniform,
    // so the branch is too).
    if (m > 0 && (2 * kSub * m) % 32 == 0 && 2 * kSub * m >= count) break;
    const int u = sub + kSub * m;
    const int first = 2 * u;
    const float4 A = T.wx[u], B = T.yz[u];
    const float2 mw = fma2(make_float2(A.x, A.y), splat(-1.0f), xw);
    const float2 mx = fma2(make_float2(A.z, A.w), splat(-1.0f), xx);
    const float2 my = fma2(make_float2(B.x, B.y), splat(-1.0f), xy);
    const float2 mz = fma2(make_float2(B.z, B.w), splat(-1.0f), xz);
    const float2 dm2 = fma2(mw, mw, fma2(mx, mx, fma2(my, my, mul2(mz, mz))));
    bool own0 = false, own1 = false;
    float n0 = dm2.x, n1 = dm2.y;
    if (OWN) {
      const uint2 c = T.code[u];
      own0 = ((c.x ^ i) & ~kIdentityBit) == 0;
      own1 = ((c.y ^ i) & ~kIdentityBit) == 0;
      if (own0 && c.x != i) n0 = 4.0f;
      if (own1 && c.y != i) n1 = 4.0f;
    }
    if (COUNT) {
      candidates += (first < count) + (first + 1 < count);
      in += (n0 <= cut2 && !own0) + (n1 <= cut2 && !own1);
    }
    if (NEAREST) {
      // The two smallest chords (of distinct sites) and where the smallest is.
      second = fminf(second, fmaxf(best, fminf(n0, n1)));
      second = fminf(second, fmaxf(n0, n1));
      if (n0 < best) {
        best = n0;
        best_at = (int)T.at[first];
      }
      if (n1 < best) {
        best = n1;
        best_at = (int)T.at[first + 1];
      }
      continue;
    }
    if (TRACK) {
      if (n0 < best) {
        best = n0;
        best_at = (int)T.at[first];
      }
      if (n1 < best) {
        best = n1;
        best_at = (int)T.at[first + 1];
      }
    } else {
      best = fminf(best, fminf(n0, n1));
    }
    // A site beyond the cutoff takes the chord at 1.25 r: its terms stay finite (a site
    // nearer the antipode, dm2 > 2, would drive the half-angle out of range) and the
    // window makes them exactly zero.
    const float2 dmc = make_float2(fminf(dm2.x, cut_hi), fminf(dm2.y, cut_hi));
    NearPair2 pr;
    if (SHORT)
      pr = near_chord_pair32x2(dmc, cw, czw, pk);
    else
      pr = near_pair32x2<false>(dmc, fma2(dmc, splat(-1.0f), add2(xn, T.norm[u])), cw, czw, pk);
    float2 coef = pr.coef;
    if (OWN) {
      const float2 keep = make_float2(own0 ? 0.f : 1.f, own1 ? 0.f : 1.f);
      coef = mul2(coef, keep);
      pr.w = mul2(pr.w, keep);
    }
    sc = fma2(pr.q, pr.w, sc);
    se = fma2(pr.rab, pr.w, se);
    sw = fma2(coef, mw, sw);
    sx = fma2(coef, mx, sx);
    sy = fma2(coef, my, sy);
    sz = fma2(coef, mz, sz);
  }
}

// One warp task of the gather: warp `warp` (G sources along the Hilbert order) and slice
// `slice` of the sample in A; T, W and sums are the warp's shared memory.
template <bool TRACK, bool SHORT, bool NEAREST>
using NearTileOf = NearTile<!SHORT && !NEAREST, TRACK>;

template <int G, bool TRACK, bool SHORT, bool NEAREST, bool COUNT = false>
__device__ __forceinline__ void near32_warp(const NearArgs& A, int warp, int slice, NearTileOf<TRACK, SHORT, NEAREST>& T,
                                            NearWalk<G>& W, double (*sums)[kNearWarps * 32]) {
  constexpr int kSub = NearShape<G>::sub;
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int n = A.n, slices = A.slices;
  const uint32_t* __restrict__ cell_off = A.cell_off;
  const float* __restrict__ site_x = A.site_x;
  const float4* __restrict__ sq = A.sq;
  const uint32_t* __restrict__ scode = A.scode;
  const NearCut& cut = A.cut;
  if (warp * G >= n) return;
  const int sub = lane % kSub;
  const int p = warp * G + lane / kSub;
  const bool live = p < n;
  const uint32_t i = live ? A.src_perm[p] : 0u;
  const float4 x = A.q[i];
  {
    // This source's chart ball, 0.1% wider (plus 1e-6) for the FP32 rounding of the chart.
    const NearGrid g = *A.gp;
    const double kappa = 1.0 - 0.5 * cut.walk2;
    const double den = 1.0 / ((double)x.x + kappa);
    const float c[3] = {(float)(x.y * den), (float)(x.z * den), (float)(x.w * den)};
    const float rho = (float)(sqrt(1.0 - kappa * kappa) * den) * 1.001f + 1e-6f;
    float lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
      lo[a] = warp_min(live ? c[a] - rho : 3e38f);
      hi[a] = warp_max(live ? c[a] + rho : -3e38f);
    }
    if (!(lo[0] <= hi[0])) return;  // no live source in this warp
    if (sub == 0) {
      const int s = lane / kSub;
      for (int a = 0; a < 3; ++a) W.cen[s][a] = c[a];
      W.rad[s] = live ? rho : -1.0f;
      W.src[s] = live ? i : 0xfffffffeu;
    }
    if (lane == 0) {
      for (int a = 0; a < 3; ++a) {
        W.clo[a] = cell_axis(lo[a], g.lower[a], g.cells_per_unit, g.sdim);
        W.chi[a] = cell_axis(hi[a], g.lower[a], g.cells_per_unit, g.sdim);
        W.lower[a] = g.lower[a];
      }
      W.cells_per_unit = g.cells_per_unit;
      W.sdim = g.sdim;
    }
  }
  for (int k = 0; k < 6; ++k) sums[k][threadIdx.x] = 0.0;
  __syncwarp();
  const float cut2 = (float)cut.cut2, cut_hi = (float)cut.cut_hi, cw = (float)cut.cut_w,
              czw = (float)(cut.cut_z * cut.cut_w), pk = (float)(-6.0 * kPi * cut.cut_w);
  const float nx2 = 2.0f * fmaf(x.x, x.x, fmaf(x.y, x.y, fmaf(x.z, x.z, x.w * x.w)));
  const float2 xw = splat(x.x), xx = splat(x.y), xy = splat(x.z), xz = splat(x.w), xn = splat(nx2);
  float best = 4.0f, second = 4.0f;
  int best_at = -1;
  uint32_t candidates = 0, in = 0;  // COUNT only
  float2 sw = splat(0.f), sx = splat(0.f), sy = splat(0.f), sz = splat(0.f), sc = splat(0.f), se = splat(0.f);
  int since = 0;  // tiles since the last FP64 merge
  const int rows = (W.chi[1] - W.clo[1] + 1) * (W.chi[2] - W.clo[2] + 1);
  const int mine = rows > slice ? (rows - slice + slices - 1) / slices : 0;  // rows slice, slice+slices, ...
  for (int rb = 0; rb < mine; rb += 32) {
    uint32_t start = 0, len = 0;
    if (rb + lane < mine) {
      uint32_t a, b;
      if (walk_row(W, cell_off, site_x, slice + (rb + lane) * slices, a, b)) {
        start = a;
        len = b - a;
      }
    }
    // Compact the nonempty runs to the first lanes (in row order), so every row boundary
    // the tiles cross is a real one.
    const unsigned nonempty = __ballot_sync(full, len > 0);
    __syncwarp();
    if (len > 0) W.runs[__popc(nonempty & ((1u << lane) - 1u))] = make_uint2(start, len);
    __syncwarp();
    const int nr = __popc(nonempty);
    start = 0;
    len = 0;
    if (lane < nr) {
      const uint2 run = W.runs[lane];
      start = run.x;
      len = run.y;
    }
    uint32_t incl = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t v = __shfl_up_sync(full, incl, o);
      if (lane >= o) incl += v;
    }
    const uint32_t total = __shfl_sync(full, incl, 31);
    const uint32_t shift = start - (incl - len);  // element e of run k is site shift_k + e
    int k = 0;  // the run of this lane's next element: the first lane with incl > e
    for (uint32_t tb = 0; tb < total; tb += kNearTile) {
      const int count = (int)min((uint32_t)kNearTile, total - tb);
      bool mine = false;  // this lane loaded an image of one of the warp's sources
      __syncwarp();
#pragma unroll
      for (int h = 0; h < kNearTile / 64; ++h) {
        // Lane l loads elements 64h + 2l and 64h + 2l + 1 (slot 32h + l) and writes the slot
        // whole. An element past the batch's end is a blank site: at the origin,
        // dm2 = |x|^2 ~ 1 lies beyond every cutoff of the chart-grid path (r < 0.9 rad,
        // cut2 < 0.76), and its code matches no source.
        const int el = 64 * h + 2 * lane;
        const uint32_t e = tb + el;
        uint32_t kin;
        // Warp-uniform advance; it ends: each pass moves some lane's k, and k stops at 31.
        for (;;) {
          kin = __shfl_sync(full, incl, k);
          const bool advance = k < 31 && kin <= e;
          if (!__any_sync(full, advance)) break;
          if (advance) ++k;
        }
        // Element e + 1 is in run k, or starts run k + 1 (runs are nonempty).
        const int k1 = (e + 1 >= kin && k < 31) ? k + 1 : k;
        uint32_t site[2];
        site[0] = __shfl_sync(full, shift, k) + e;
        site[1] = __shfl_sync(full, shift, k1) + e + 1;
        float4 y[2];
        uint32_t code[2];
#pragma unroll
        for (int b = 0; b < 2; ++b) {
          y[b] = make_float4(0.f, 0.f, 0.f, 0.f);
          code[b] = 0xffffffffu;
          if (el + b < count) {
            y[b] = sq[site[b]];
            code[b] = scode[site[b]];
          }
        }
        const int slot = 32 * h + lane;
        T.wx[slot] = make_float4(y[0].x, y[1].x, y[0].y, y[1].y);
        T.yz[slot] = make_float4(y[0].z, y[1].z, y[0].w, y[1].w);
        T.code[slot] = make_uint2(code[0], code[1]);
        if (!SHORT && !NEAREST)
          T.norm[slot] = make_float2(2.0f * fmaf(y[0].x, y[0].x, fmaf(y[0].y, y[0].y, fmaf(y[0].z, y[0].z, y[0].w * y[0].w))),
                                     2.0f * fmaf(y[1].x, y[1].x, fmaf(y[1].y, y[1].y, fmaf(y[1].z, y[1].z, y[1].w * y[1].w))));
        if (TRACK) reinterpret_cast<uint2*>(T.at)[slot] = make_uint2(site[0], site[1]);
#pragma unroll
        for (int s2 = 0; s2 < G; ++s2)
          mine |= ((code[0] & ~kIdentityBit) == W.src[s2]) | ((code[1] & ~kIdentityBit) == W.src[s2]);
      }
      // Whether the tile holds an image of one of the warp's sources (rare): only then does
      // the slot loop test each site's source.
      const bool tile_own = __any_sync(full, mine);
      __syncwarp();
      if (live) {
        if (tile_own)
          near_slots<G, TRACK, SHORT, true, NEAREST, COUNT>(T, count, sub, i, xw, xx, xy, xz, xn, cut_hi, cw, czw, pk, sw,
                                                         sx, sy, sz, sc, se, best, best_at, second, cut2, candidates,
                                                         in);
        else
          near_slots<G, TRACK, SHORT, false, NEAREST, COUNT>(T, count, sub, i, xw, xx, xy, xz, xn, cut_hi, cw, czw, pk, sw,
                                                          sx, sy, sz, sc, se, best, best_at, second, cut2, candidates,
                                                          in);
      }
      if (!NEAREST && ++since == NearShape<G>::merge) {
        merge_sums(sums, sw, sx, sy, sz, sc, se);
        since = 0;
      }
    }
  }
  merge_sums(sums, sw, sx, sy, sz, sc, se);
  if (COUNT) {
    unsigned long long c = live ? candidates : 0u, v = live ? in : 0u;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      c += __shfl_xor_sync(full, c, o);
      v += __shfl_xor_sync(full, v, o);
    }
    if (lane == 0) {
      atomicAdd(&A.pair_counts[0], c);
      atomicAdd(&A.pair_counts[1], v);
    }
  }
  // The nearest over the source's lanes: smallest chord, then smallest sorted-site index
  // (the first such site in the walk's order).
#pragma unroll
  for (int o = kSub / 2; o > 0; o >>= 1) {
    const float ob = __shfl_xor_sync(full, best, o);
    if (NEAREST) {
      const float os = __shfl_xor_sync(full, second, o);
      second = fminf(fminf(second, os), fmaxf(best, ob));
    }
    if (TRACK) {
      const int oa = __shfl_xor_sync(full, best_at, o);
      if (ob < best || (ob == best && (unsigned)oa < (unsigned)best_at)) {
        best = ob;
        best_at = oa;
      }
    } else {
      best = fminf(best, ob);
    }
  }
  __syncwarp();
  if (!live || sub != 0) return;
  if (NEAREST) {
    // The FP32 winner is the FP64 nearest when no other site's FP32 chord is within twice
    // the chord error of it, and when the FP64 nearest cannot lie outside the walked ball;
    // any other source is listed for the exact FP64 search (k_nearest_exact), which
    // overwrites its row.
    const double b = best, margin = 2.0 * chord_error32(b);
    if ((double)second <= b + margin || b + margin > cut.walk2) {
      const uint32_t slot = atomicAdd(A.exact_count, 1u);
      A.exact_list[slot] = i;
    }
  }
  if (best > cut2) {  // no site within the cutoff
    best = 4.0f;
    best_at = -1;
  }
  double t[6];
  for (int c = 0; c < 6; ++c) {
    t[c] = 0.0;
    for (int l = 0; l < kSub; ++l) t[c] += sums[c][threadIdx.x + l];
  }
  const double3 f = force_from_differences(to_d4(x), make_double4(t[0], t[1], t[2], t[3]));
  // direct (one slice): the source's own row; else row p of this slice's partial rows.
  const size_t at = A.direct ? (size_t)i : (size_t)slice * A.stride + p;
  A.out.force[at] = make_double4(f.x, f.y, f.z, t[4]);
  A.out.energy[at] = kPi * t[5];
  A.out.nearest[at] = best;
  if (TRACK) A.out.nearest_at[at] = best_at;
}

template <int G, bool TRACK, bool SHORT, bool NEAREST, bool COUNT = false>
__global__ void __launch_bounds__(kNearWarps * 32, 7) k_near32(const NearArgs A) {
  __shared__ NearTileOf<TRACK, SHORT, NEAREST> tiles[kNearWarps];
  __shared__ NearWalk<G> walks[kNearWarps];
  __shared__ double sums[6][kNearWarps * 32];  // FP64 lane sums: force differences, curvature, energy
  const int w = threadIdx.x >> 5;
  near32_warp<G, TRACK, SHORT, NEAREST, COUNT>(A, blockIdx.x * kNearWarps + w, blockIdx.y, tiles[w], walks[w], sums);
}

// The spacing pass's FP32 nearest-site search with one source per thread (tile shape 1):
// each thread walks its own source's first ball, cell row by cell row, reading the sorted
// sites straight from global memory - consecutive threads hold Hilbert-consecutive sources,
// whose rows overlap, so the reads mostly hit in L1 - and keeps its two best chords. No
// union of several sources' balls and no shared-memory staging: the work per site (one
// squared chord) is too small to pay for either. The proof test, the exact-search list and
// the rows written are those of k_near32's nearest-only variant (direct rows, one slice).
__global__ void __launch_bounds__(256) k_nearest_lane(const NearArgs A) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= A.n) return;
  const uint32_t i = A.src_perm[p];
  const float4 x = A.q[i];
  const NearGrid* __restrict__ gp = A.gp;
  const float lower[3] = {gp->lower[0], gp->lower[1], gp->lower[2]};
  const float per = gp->cells_per_unit;
  const int sdim = gp->sdim;
  const double kappa = 1.0 - 0.5 * A.cut.walk2;
  const double den = 1.0 / ((double)x.x + kappa);
  const float c[3] = {(float)(x.y * den), (float)(x.z * den), (float)(x.w * den)};
  const float rho = (float)(sqrt(1.0 - kappa * kappa) * den) * 1.001f + 1e-6f;
  int lo[3], hi[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    lo[a] = cell_axis(c[a] - rho, lower[a], per, sdim);
    hi[a] = cell_axis(c[a] + rho, lower[a], per, sdim);
  }
  const float width = 1.0f / per;
  const uint32_t* __restrict__ cell_off = A.cell_off;
  const float4* __restrict__ sq = A.sq;
  // The source's own (identity) site holds x itself, bit for bit, and is no neighbour: the
  // first site equal to x is taken for it. Any further site equal to x (a duplicate of the
  // source, or an image of it that rounds onto it) is a neighbour at distance 0.
  bool self_seen = false;
  float best = 4.0f, second = 4.0f;
  int best_at = -1;
  for (int z = lo[2]; z <= hi[2]; ++z) {
    const float cz = lower[2] + (float)z * width;
    const float gz = fmaxf(0.f, fmaxf(cz - c[2], c[2] - (cz + width)));
    for (int y = lo[1]; y <= hi[1]; ++y) {
      const float cy = lower[1] + (float)y * width;
      const float gy = fmaxf(0.f, fmaxf(cy - c[1], c[1] - (cy + width)));
      const float rest = rho * rho - gy * gy - gz * gz;
      if (rest < 0.f) continue;
      const float span = sqrtf(rest);
      const int row = sdim * (y + sdim * z);
      const uint32_t end = __ldg(&cell_off[row + cell_axis(c[0] + span, lower[0], per, sdim) + 1]);
      for (uint32_t t = __ldg(&cell_off[row + cell_axis(c[0] - span, lower[0], per, sdim)]); t < end; ++t) {
        const float4 s = __ldg(&sq[t]);
        const float mw = x.x - s.x, mx = x.y - s.y, my = x.z - s.z, mz = x.w - s.w;
        float d = fmaf(mw, mw, fmaf(mx, mx, fmaf(my, my, mz * mz)));
        if (d == 0.0f && !self_seen && s.x == x.x && s.y == x.y && s.z == x.z && s.w == x.w) {
          self_seen = true;  // (an equal site has d = 0: the rare branch)
          d = 4.0f;
        }
        second = fminf(second, fmaxf(best, d));
        if (d < best) {
          best = d;
          best_at = (int)t;
        }
      }
    }
  }
  const double b = best, margin = 2.0 * chord_error32(b);
  if ((double)second <= b + margin || b + margin > A.cut.walk2) {
    const uint32_t slot = atomicAdd(A.exact_count, 1u);
    A.exact_list[slot] = i;
  }
  // Only the chosen site: the refinement that follows computes its FP64 chord (4 when there
  // is none within the cutoff), and a nearest-only pass has no forces or energies.
  A.out.nearest_at[i] = best > (float)A.cut.cut2 ? -1 : best_at;
}

// The exact nearest orbit neighbour of each source the FP32 spacing gather listed: every
// site in the chart ball of the cutoff (the whole shell's reach, not the first walk's
// smaller ball), its chord in FP64 from the float32 positions with the image formed in FP64
// and both normalised (the oracle's definition), and the smallest chord kept, then the
// smallest source index, then the first sorted site. A warp per listed source, its lanes
// over the ball's cell rows. Writes the source's nearest chord and site (the refinement
// that follows recomputes the chord of that site and its source index), and counts the
// sources whose nearest chord is shared exactly by two different sources (exact ties).
__global__ void __launch_bounds__(128) k_nearest_exact(const float4* __restrict__ q, int gid,
                                                       const uint32_t* __restrict__ scode,
                                                       const uint32_t* __restrict__ simg,
                                                       const uint32_t* __restrict__ cell_off,
                                                       const NearGrid* __restrict__ gp, double cut2,
                                                       const uint32_t* __restrict__ list,
                                                       const uint32_t* __restrict__ listed, Rows out,
                                                       unsigned int* __restrict__ ties) {
  __shared__ double4 ops[kMaxGroupOrder];  // the group's rows: each lane reads its own site's
  {
    const int off = c_group_offset[gid], order = c_group_order[gid];
    for (int k = threadIdx.x; k < order; k += blockDim.x) ops[k] = c_ops32[off + k];
  }
  __syncthreads();
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const uint32_t count = *listed;
  const NearGrid g = *gp;
  const uint32_t stride = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < count; w += stride) {
    const uint32_t i = list[w];
    const double4 x = normalize4(to_d4(q[i]));
    // The cutoff's chart ball (as in k_near32), 0.1% wider plus 1e-6.
    const double kappa = 1.0 - 0.5 * cut2;
    const double den = 1.0 / (x.x + kappa);
    const double cen[3] = {x.y * den, x.z * den, x.w * den};
    const double rho = sqrt(1.0 - kappa * kappa) * den * 1.001 + 1e-6;
    int lo[3], hi[3];
    for (int a = 0; a < 3; ++a) {
      lo[a] = cell_axis((float)(cen[a] - rho), g.lower[a], g.cells_per_unit, g.sdim);
      hi[a] = cell_axis((float)(cen[a] + rho), g.lower[a], g.cells_per_unit, g.sdim);
    }
    const int ny = hi[1] - lo[1] + 1, rows = ny * (hi[2] - lo[2] + 1);
    double best = 4.0;
    uint32_t best_src = 0xffffffffu, best_site = 0xffffffffu;
    bool tie = false;
    for (int r = lane; r < rows; r += 32) {
      const int row = g.sdim * (lo[1] + r % ny + g.sdim * (lo[2] + r / ny));
      const uint32_t end = cell_off[row + hi[0] + 1];
      for (uint32_t t = cell_off[row + lo[0]]; t < end; ++t) {
        const uint32_t code = scode[t];
        if (code == (i | kIdentityBit)) continue;  // the source itself
        const uint32_t j = code & ~kIdentityBit, im = simg[t];
        const int op = (int)(im >> 1);
        double4 y = normalize4(op == 0 ? to_d4(q[j]) : qmul(to_d4(q[j]), ops[op]));
        if (im & 1u) y = neg4(y);
        const double mw = x.x - y.x, mx = x.y - y.y, my = x.z - y.z, mz = x.w - y.w;
        const double d = mw * mw + mx * mx + my * my + mz * mz;
        if (d < best) {
          best = d;
          best_src = j;
          best_site = t;
          tie = false;
        } else if (d == best) {
          tie |= j != best_src;
          if (j < best_src || (j == best_src && t < best_site)) {
            best_src = j;
            best_site = t;
          }
        }
      }
    }
    for (int o = 16; o; o >>= 1) {
      const double ob = __shfl_xor_sync(full, best, o);
      const uint32_t os = __shfl_xor_sync(full, best_src, o), ot = __shfl_xor_sync(full, best_site, o);
      const bool otie = __shfl_xor_sync(full, tie ? 1 : 0, o) != 0;
      if (ob < best) {
        best = ob;
        best_src = os;
        best_site = ot;
        tie = otie;
      } else if (ob == best) {
        tie = tie || otie || (os != best_src && ob < 4.0);
        if (os < best_src || (os == best_src && ot < best_site)) {
          best_src = os;
          best_site = ot;
        }
      }
    }
    if (lane == 0) {
      const bool found = best <= cut2;
      out.nearest[i] = found ? best : 4.0;
      out.nearest_at[i] = found ? (int)best_site : -1;
      if (found && tie) atomicAdd(ties, 1u);
    }
  }
}

template <bool TRACK>
__global__ void __launch_bounds__(kNearWarps * 32) k_near64(const double4* __restrict__ q, int n,
                                                              const uint32_t* __restrict__ src_perm,
                                                              const double4* __restrict__ sq,
                                                              const uint32_t* __restrict__ scode,
                                                              const uint32_t* __restrict__ cell_off,
                                                              const NearGrid* __restrict__ gp, NearCut cut, int slices,
                                                              Rows out, int stride) {
  __shared__ double4 tq[kNearWarps][32];
  __shared__ double tn[kNearWarps][32];
  __shared__ uint32_t tc[kNearWarps][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int warp = blockIdx.x * kNearWarps + w;
  const int slice = blockIdx.y;
  if (warp * 32 >= n) return;
  const int p = warp * 32 + lane;
  const bool live = p < n;
  const uint32_t i = live ? src_perm[p] : 0u;
  const double4 x = q[i];
  const NearGrid g = *gp;
  WarpBox box;
  if (!warp_box(chart(x), live, g, (float)cut.chord, box)) return;
  const double nx2 = 2.0 * dot4(x, x);
  double yw = 0, yx = 0, yy = 0, yz = 0, fc = 0, fe = 0, best = 4.0;
  int best_at = -1;
  const int ny = box.chi[1] - box.clo[1] + 1, nz = box.chi[2] - box.clo[2] + 1;
  const int rows = ny * nz;
  for (int r = slice; r < rows; r += slices) {
    uint32_t start, end;
    if (!row_run(box, g, cell_off, r, start, end)) continue;
    for (uint32_t base = start; base < end; base += 32) {
      const int count = (int)min(32u, end - base);
      __syncwarp();
      if (lane < count) {
        const double4 s = sq[base + lane];
        tq[w][lane] = s;
        tn[w][lane] = 2.0 * dot4(s, s);
        tc[w][lane] = scode[base + lane];
      }
      __syncwarp();
      if (!live) continue;
      for (int t = 0; t < count; ++t) {
        const double4 y = tq[w][t];
        const double mw = x.x - y.x, mx = x.y - y.y, my = x.z - y.z, mz = x.w - y.w;
        const double dm2 = mw * mw + mx * mx + my * my + mz * mz;
        if (dm2 > cut.cut2) continue;
        const uint32_t code = tc[w][t];
        if ((code & ~kIdentityBit) == i) {
          if (code == i && dm2 < best) {
            best = dm2;
            if (TRACK) best_at = (int)(base + t);
          }
          continue;
        }
        if (dm2 < best) {
          best = dm2;
          if (TRACK) best_at = (int)(base + t);
        }
        const double dp2 = nx2 + tn[w][t] - dm2;
        PairD pr = quey_pair64(dm2, dp2);
        window64(pr, dm2, dp2, cut.cut_z, cut.cut_w);
        yw += pr.coef * mw;
        yx += pr.coef * mx;
        yy += pr.coef * my;
        yz += pr.coef * mz;
        fc += pr.curv;
        fe += pr.energy;
      }
    }
  }
  if (!live) return;
  const double3 f = force_from_differences(x, make_double4(yw, yx, yy, yz));
  const size_t at = (size_t)slice * stride + p;
  out.force[at] = make_double4(f.x, f.y, f.z, fc);
  out.energy[at] = fe;
  out.nearest[at] = best;
  if (TRACK) out.nearest_at[at] = best_at;
}

// ------------------------------------------------------------------ dense near field
// Wide cutoffs on small samples (and FP64 mode from r = 0.5 rad on) are summed over every
// image like all pairs, with the same near-field semantics: the near twin of each image
// (y or -y) counts when its chord is within the cutoff, the windowed pair applies, the own
// orbit is excluded from forces and its non-identity images bound the nearest. FP32 mode
// uses the all-pairs tile (pairs of images, packed f32x2 arithmetic, near twin by the sign
// of x . y): a site beyond the cutoff is evaluated at the 1.25 r chord, where the window is
// exactly zero, and the nearest chord is reset to 4 when no site is within the cutoff.
template <bool TRACK, bool MASKED, bool SHORT>
__device__ __forceinline__ void dense32_tile(const float4 x, float nx2, const PairSlots& S, int count, int i, int j0,
                                             int k, int n, float cut_hi, float cw, float czw, float pk, float2& sw,
                                             float2& sx, float2& sy, float2& sz, float2& sc, float2& se, float& best,
                                             int& best_at) {
  const float2 xw = splat(x.x), xx = splat(x.y), xy = splat(x.z), xz = splat(x.w), xn = splat(nx2);
  const int slots = (count + 1) >> 1;
#pragma unroll 2
  for (int u = 0; u < slots; ++u) {
    const float4 A = S.wx[u], B = S.yz[u];
    const float2 yw = make_float2(A.x, A.y), yx = make_float2(A.z, A.w);
    const float2 yy = make_float2(B.x, B.y), yz = make_float2(B.z, B.w);
    const float2 dot = fma2(xw, yw, fma2(xx, yx, fma2(xy, yy, mul2(xz, yz))));
    const float2 ms = make_float2(dot.x >= 0.f ? -1.f : 1.f, dot.y >= 0.f ? -1.f : 1.f);
    const float2 dw = fma2(ms, yw, xw), dx = fma2(ms, yx, xx), dy = fma2(ms, yy, xy), dz = fma2(ms, yz, xz);
    const float2 nearv = fma2(dw, dw, fma2(dx, dx, fma2(dy, dy, mul2(dz, dz))));
    float n0 = nearv.x, n1 = nearv.y;
    float2 keep = splat(1.0f);
    if (MASKED) {
      const int j = j0 + 2 * u;
      const bool own0 = j == i, own1 = j + 1 == i, pad1 = 2 * u + 1 >= count;
      if (own0 && k == 0) n0 = 4.0f;
      if ((own1 && k == 0) || pad1) n1 = 4.0f;
      keep = make_float2(own0 ? 0.f : 1.f, (own1 || pad1) ? 0.f : 1.f);
    }
    if (TRACK) {
      if (n0 < best) {
        best = n0;
        best_at = k * n + j0 + 2 * u;
      }
      if (n1 < best) {
        best = n1;
        best_at = k * n + j0 + 2 * u + 1;
      }
    } else {
      best = fminf(best, fminf(n0, n1));
    }
    const float2 dmc = make_float2(fminf(nearv.x, cut_hi), fminf(nearv.y, cut_hi));
    const float2 farv = fma2(dmc, splat(-1.0f), add2(xn, S.n2[u]));
    NearPair2 p = near_pair32x2<SHORT>(dmc, farv, cw, czw, pk);
    if (MASKED) {
      p.coef = mul2(p.coef, keep);
      p.w = mul2(p.w, keep);
    }
    sw = fma2(p.coef, dw, sw);
    sx = fma2(p.coef, dx, sx);
    sy = fma2(p.coef, dy, sy);
    sz = fma2(p.coef, dz, sz);
    sc = fma2(p.q, p.w, sc);
    se = fma2(p.rab, p.w, se);  // energy / pi
  }
}

template <bool TRACK, bool SHORT>
__global__ void __launch_bounds__(kPairBlock, 8) k_dense32(const float4* __restrict__ q, int n, int op_off, int jtiles,
                                                           int total_tiles, int tiles_per_chunk, NearCut cut, Rows out,
                                                           int stride) {
  __shared__ PairSlots S;
  __shared__ double sums[6][kPairBlock];  // FP64 row sums (shared: registers go to the pairs)
  const int i0 = blockIdx.x * kPairBlock;
  const int i = i0 + threadIdx.x;
  const bool live = i < n;
  const float4 x = live ? q[i] : make_float4(1.f, 0.f, 0.f, 0.f);
  const float nx2 = 2.0f * fmaf(x.x, x.x, fmaf(x.y, x.y, fmaf(x.z, x.z, x.w * x.w)));
  const float cut2 = (float)cut.cut2, cut_hi = (float)cut.cut_hi, cw = (float)cut.cut_w,
              czw = (float)(cut.cut_z * cut.cut_w), pk = (float)(-6.0 * kPi * cut.cut_w);
  for (int c = 0; c < 6; ++c) sums[c][threadIdx.x] = 0.0;
  float best = 4.0f;
  int best_at = -1;
  const int t0 = blockIdx.y * tiles_per_chunk, t1 = min(total_tiles, t0 + tiles_per_chunk);
  const int slot = threadIdx.x >> 1, half = threadIdx.x & 1;
  for (int tid = t0; tid < t1; ++tid) {
    const PairTile pt = pair_tile(tid, jtiles, n);
    __syncthreads();
    {
      const float4 y = (int)threadIdx.x < pt.count ? image32(q[pt.j0 + threadIdx.x], op_off + pt.k, pt.k == 0)
                                                   : make_float4(1.f, 0.f, 0.f, 0.f);
      float* wx = reinterpret_cast<float*>(&S.wx[slot]);
      float* yz = reinterpret_cast<float*>(&S.yz[slot]);
      wx[half] = y.x;
      wx[2 + half] = y.y;
      yz[half] = y.z;
      yz[2 + half] = y.w;
      reinterpret_cast<float*>(&S.n2[slot])[half] = 2.0f * fmaf(y.x, y.x, fmaf(y.y, y.y, fmaf(y.z, y.z, y.w * y.w)));
    }
    __syncthreads();
    if (!live) continue;
    float2 sw = splat(0.f), sx = splat(0.f), sy = splat(0.f), sz = splat(0.f), sc = splat(0.f), se = splat(0.f);
    const bool masked = (pt.j0 < i0 + kPairBlock && i0 < pt.j0 + pt.count) || (pt.count & 1);
    if (masked)
      dense32_tile<TRACK, true, SHORT>(x, nx2, S, pt.count, i, pt.j0, pt.k, n, cut_hi, cw, czw, pk, sw, sx, sy, sz, sc,
                                       se, best, best_at);
    else
      dense32_tile<TRACK, false, SHORT>(x, nx2, S, pt.count, i, pt.j0, pt.k, n, cut_hi, cw, czw, pk, sw, sx, sy, sz,
                                        sc, se, best, best_at);
    sums[0][threadIdx.x] += (double)sw.x + (double)sw.y;
    sums[1][threadIdx.x] += (double)sx.x + (double)sx.y;
    sums[2][threadIdx.x] += (double)sy.x + (double)sy.y;
    sums[3][threadIdx.x] += (double)sz.x + (double)sz.y;
    sums[4][threadIdx.x] += (double)sc.x + (double)sc.y;
    sums[5][threadIdx.x] += (double)se.x + (double)se.y;
  }
  if (!live) return;
  if (best > cut2) {  // no image within the cutoff
    best = 4.0f;
    best_at = -1;
  }
  const size_t at = (size_t)blockIdx.y * stride + i;
  const double3 f = force_from_differences(
      to_d4(x), make_double4(sums[0][threadIdx.x], sums[1][threadIdx.x], sums[2][threadIdx.x], sums[3][threadIdx.x]));
  out.force[at] = make_double4(f.x, f.y, f.z, sums[4][threadIdx.x]);
  out.energy[at] = kPi * sums[5][threadIdx.x];
  out.nearest[at] = best;
  if (TRACK) out.nearest_at[at] = best_at;
}

template <bool TRACK>
__global__ void __launch_bounds__(kPairBlock) k_dense64(const double4* __restrict__ q, int n, int op_off, int jtiles,
                                                        int total_tiles, int tiles_per_chunk, NearCut cut, Rows out,
                                                        int stride) {
  __shared__ double4 tile[kPairBlock];
  const int i0 = blockIdx.x * kPairBlock;
  const int i = i0 + threadIdx.x;
  const bool live = i < n;
  const double4 x = live ? q[i] : make_double4(1, 0, 0, 0);
  double yw = 0, yx = 0, yy = 0, yz = 0, fc = 0, fe = 0, best = 4.0;
  int best_at = -1;
  const int t0 = blockIdx.y * tiles_per_chunk, t1 = min(total_tiles, t0 + tiles_per_chunk);
  for (int tid = t0; tid < t1; ++tid) {
    const PairTile pt = pair_tile(tid, jtiles, n);
    __syncthreads();
    if ((int)threadIdx.x < pt.count) tile[threadIdx.x] = image64(q[pt.j0 + threadIdx.x], op_off + pt.k, pt.k == 0);
    __syncthreads();
    if (!live) continue;
    for (int t = 0; t < pt.count; ++t) {
      const double4 y = tile[t];
      const double mw = x.x - y.x, mx = x.y - y.y, my = x.z - y.z, mz = x.w - y.w;
      const double pw = x.x + y.x, px = x.y + y.y, py = x.z + y.z, pz = x.w + y.w;
      const double dm2 = mw * mw + mx * mx + my * my + mz * mz;
      const double dp2 = pw * pw + px * px + py * py + pz * pz;
      const bool minus = dm2 <= dp2;
      const double nearv = minus ? dm2 : dp2;
      if (nearv > cut.cut2) continue;
      if (pt.j0 + t == i) {
        if (pt.k != 0 && nearv < best) {
          best = nearv;
          if (TRACK) best_at = pt.k * n + pt.j0 + t;
        }
        continue;
      }
      if (nearv < best) {
        best = nearv;
        if (TRACK) best_at = pt.k * n + pt.j0 + t;
      }
      PairD pr = quey_pair64(nearv, minus ? dp2 : dm2);
      window64(pr, nearv, minus ? dp2 : dm2, cut.cut_z, cut.cut_w);
      const double c = pr.coef;
      yw += c * (minus ? mw : pw);
      yx += c * (minus ? mx : px);
      yy += c * (minus ? my : py);
      yz += c * (minus ? mz : pz);
      fc += pr.curv;
      fe += pr.energy;
    }
  }
  if (!live) return;
  const size_t at = (size_t)blockIdx.y * stride + i;
  const double3 f = force_from_differences(x, make_double4(yw, yx, yy, yz));
  out.force[at] = make_double4(f.x, f.y, f.z, fc);
  out.energy[at] = fe;
  out.nearest[at] = best;
  if (TRACK) out.nearest_at[at] = best_at;
}

cudaError_t launch_dense_near(int prec, bool track, bool short_atan, const float4* q32, const double4* q64, int n,
                              int gid, const PairsPlan& pl, double cut2, double chord, double cut_z, double cut_w,
                              Rows partial, Rows out, cudaStream_t s) {
  const int op_off = host_group_offset(gid);
  const dim3 grid(pl.jtiles, pl.chunks);
  const bool direct = pl.chunks == 1;
  const Rows dst = direct ? out : partial;
  const NearCut cut = near_cut(cut2, chord, cut_z, cut_w);
  probe_mark(s);
  if (prec == kFP64) {
    if (track) k_dense64<true><<<grid, kPairBlock, 0, s>>>(q64, n, op_off, pl.jtiles, pl.total_tiles, pl.tiles_per_chunk, cut, dst, n);
    else k_dense64<false><<<grid, kPairBlock, 0, s>>>(q64, n, op_off, pl.jtiles, pl.total_tiles, pl.tiles_per_chunk, cut, dst, n);
  } else {
    auto kernel = track ? (short_atan ? k_dense32<true, true> : k_dense32<true, false>)
                        : (short_atan ? k_dense32<false, true> : k_dense32<false, false>);
    kernel<<<grid, kPairBlock, 0, s>>>(q32, n, op_off, pl.jtiles, pl.total_tiles, pl.tiles_per_chunk, cut, dst, n);
  }
  probe_mark(s);
  probe_count(direct ? 1 : 2);
  if (!direct)
    k_rows_reduce<<<(n + 31) / 32, 32 * kReduceWarps, 0, s>>>(partial, n, pl.chunks, n, nullptr, out, track ? 1 : 0);
  return cudaGetLastError();
}

// ------------------------------------------------------------------ the pass
// The FP32 gather kernel of a tile shape (G sources per warp) and variant.
template <int G>
cudaError_t launch_near32_shape(bool track, bool short_atan, bool nearest, dim3 grid, const NearArgs& A,
                                cudaStream_t s) {
  auto kernel = nearest ? k_near32<G, true, false, true>
                        : track ? (short_atan ? k_near32<G, true, true, false> : k_near32<G, true, false, false>)
                                : (short_atan ? k_near32<G, false, true, false> : k_near32<G, false, false, false>);
  // A diagnostic pass that counts its pairs (a relaxation's force pass only).
  if (A.pair_counts && !nearest && !track)
    kernel = short_atan ? k_near32<G, false, true, false, true> : k_near32<G, false, false, false, true>;
  kernel<<<grid, kNearWarps * 32, 0, s>>>(A);
  return cudaGetLastError();
}
inline cudaError_t launch_near32(int G, bool track, bool short_atan, bool nearest, dim3 grid, const NearArgs& A,
                                 cudaStream_t s) {
  switch (G) {
    case 2: return launch_near32_shape<2>(track, short_atan, nearest, grid, A, s);
    case 4: return launch_near32_shape<4>(track, short_atan, nearest, grid, A, s);
    case 8: return launch_near32_shape<8>(track, short_atan, nearest, grid, A, s);
    default: return cudaErrorInvalidValue;
  }
}

// Site count of a shell pass (offsets[n] after the scan), for sizing the workspace.
cudaError_t launch_shell_count(int prec, const float4* q32, const double4* q64, int n, int gid, double s_margin,
                               uint32_t* counts, uint32_t* offsets, uint32_t* scan_tmp, uint4* masks,
                               uint32_t* rim_list, float4* rim_q, uint32_t* rim_count, cudaStream_t s) {
  int launches = 0;
  cudaError_t e = launch_shell_masks(prec, q32, q64, n, gid, s_margin, counts, masks, rim_list, rim_q, rim_count, s,
                                     &launches);
  if (e) return e;
  return launch_scan(counts, offsets, n, nullptr, scan_tmp, s);
}

// Parts 1-3 of a pass: shell, chart grid and site sort, sources in Hilbert order.
cudaError_t launch_near_structure(const NearLaunch& L, cudaStream_t s, int* launches) {
  const int n = L.n;
  const bool fp64 = L.prec == kFP64;
  const int tb = 256;
  // 1. shell
  int shell_launches = 0;
  cudaError_t e = launch_shell_masks(L.prec, L.q32, L.q64, n, L.gid, L.s_margin, L.counts, L.shell_mask, L.rim_list,
                                     L.rim_q, L.rim_count, s, &shell_launches);
  if (e) return e;
  e = launch_scan(L.counts, L.offsets, n, nullptr, L.scan_tmp, s);
  if (e) return e;
  if (fp64)
    k_shell_write<true><<<(n + tb - 1) / tb, tb, 0, s>>>(L.q32, L.q64, n, L.gid, L.shell_mask, L.offsets, L.capacity,
                                                         L.site_q32, L.site_q64, L.site_meta, L.site_pos,
                                                         L.grid);
  else
    k_shell_write<false><<<(n + tb - 1) / tb, tb, 0, s>>>(L.q32, L.q64, n, L.gid, L.shell_mask, L.offsets, L.capacity,
                                                          L.site_q32, L.site_q64, L.site_meta, L.site_pos,
                                                          L.grid);
  // 2. grid and the site sort
  k_grid_setup<<<1, 1, 0, s>>>(L.grid, L.offsets + n, L.capacity, L.sdim_max, (float)L.sites_per_cell, L.cells);
  const int max_cells = L.sdim_max * L.sdim_max * L.sdim_max;
  if ((e = cudaMemsetAsync(L.cell_count, 0, sizeof(uint32_t) * (max_cells + 1), s))) return e;
  k_cell_count<<<(L.capacity + tb - 1) / tb, tb, 0, s>>>(L.site_pos, L.grid, L.site_cell, L.site_rank, L.cell_count);
  if ((e = launch_scan(L.cell_count, L.cell_off, max_cells, L.cells, L.scan_tmp, s))) return e;
  k_scatter<<<(L.capacity + tb - 1) / tb, tb, 0, s>>>(L.site_cell, L.site_rank, L.cell_off, L.capacity,
                                                      &L.grid->sites, L.perm);
  k_bucket_sort<<<(max_cells + tb - 1) / tb, tb, 0, s>>>(L.cell_off, max_cells, L.cells, L.perm, L.site_pos);
  if (fp64)
    k_site_gather<true><<<(L.capacity + tb - 1) / tb, tb, 0, s>>>(L.perm, L.grid, L.site_q32, L.site_q64, L.site_meta,
                                                                  L.sq32, L.sq64, L.scode, L.simg, L.sx);
  else
    k_site_gather<false><<<(L.capacity + tb - 1) / tb, tb, 0, s>>>(L.perm, L.grid, L.site_q32, L.site_q64,
                                                                   L.site_meta, L.sq32, L.sq64, L.scode, L.simg, L.sx);
  // 3. sources in Hilbert order
  const int mcells = kOrderDim * kOrderDim * kOrderDim;
  if ((e = cudaMemsetAsync(L.mcount, 0, sizeof(uint32_t) * (mcells + 1), s))) return e;
  if (fp64)
    k_source_count<true><<<(n + tb - 1) / tb, tb, 0, s>>>(L.q32, L.q64, n, L.grid, L.src_key, L.src_rank, L.mcount);
  else
    k_source_count<false><<<(n + tb - 1) / tb, tb, 0, s>>>(L.q32, L.q64, n, L.grid, L.src_key, L.src_rank, L.mcount);
  if ((e = launch_scan(L.mcount, L.moff, mcells, nullptr, L.scan_tmp, s))) return e;
  k_scatter<<<(n + tb - 1) / tb, tb, 0, s>>>(L.src_key, L.src_rank, L.moff, n, nullptr, L.src_perm);
  // Sources within a Hilbert cell in index order, so that a warp's sources (and with them the
  // order of its sums) are the same every pass. The one-source-per-thread spacing search
  // computes each source's row alone, in any order, and keeps the arrival order.
  const bool any_order = !fp64 && L.nearest_only && L.group_size == 1;
  if (!any_order) k_bucket_sort<<<(mcells + tb - 1) / tb, tb, 0, s>>>(L.moff, mcells, nullptr, L.src_perm);
  // shell masks (1 or 3), shell write, grid, cell count, scatter, bucket sort, site gather,
  // source count, scatter, bucket sort (scans counted by launch_scan; memsets aside)
  *launches = (any_order ? 8 : 9) + shell_launches;
  return cudaGetLastError();
}

// Slices of the gather of a pass: the FP32 spacing pass writes rows in place (one slice), so
// that its exact search can overwrite the rows of the sources it takes over.
inline int near_slices(const NearLaunch& L) {
  return L.prec == kFP64 ? L.slices : (L.nearest_only ? 1 : L.slices32);
}

NearTask near_task(const NearLaunch& L) {
  const int slices = near_slices(L);
  const int direct = slices == 1 ? 1 : 0;
  NearTask t{};
  t.a = NearArgs{L.q32, L.n, L.src_perm, L.sq32, L.scode, L.cell_off, L.sx, L.grid,
                 near_cut(L.cut2, L.chord, L.cut_z, L.cut_w), slices, direct ? L.out : L.partial, L.n, direct,
                 L.exact_list, L.exact_count, L.pair_counts};
  t.group_size = L.group_size;
  t.short_atan = L.short_atan ? 1 : 0;
  t.warps = (L.n + L.group_size - 1) / L.group_size;
  t.slices = slices;
  return t;
}

// Part 5: the slices' partial rows summed in slice order into the rows (more than one slice).
cudaError_t launch_near_reduce(const NearLaunch& L, cudaStream_t s) {
  const int slices = near_slices(L);
  if (L.prec != kFP64 && slices == 1) return cudaSuccess;
  k_rows_reduce<<<(L.n + 31) / 32, 32 * kReduceWarps, 0, s>>>(L.partial, L.n, slices, L.n, (const int*)L.src_perm,
                                                             L.out, L.track ? 1 : 0);
  probe_count();
  return cudaGetLastError();
}

cudaError_t launch_near(const NearLaunch& L, cudaStream_t s) {
  const int n = L.n;
  const bool fp64 = L.prec == kFP64;
  int structure_launches = 0;
  cudaError_t e = launch_near_structure(L, s, &structure_launches);
  if (e) return e;
  probe_count(structure_launches);
  // 4. gather, 5. slices summed into rows
  const int G = L.group_size;
  const int warps = fp64 ? (n + 31) / 32 : (n + G - 1) / G;
  const bool nearest_only = !fp64 && L.nearest_only;
  const int slices = near_slices(L);
  const dim3 grid((warps + kNearWarps - 1) / kNearWarps, slices);
  NearCut cut = near_cut(L.cut2, L.chord, L.cut_z, L.cut_w);
  if (nearest_only) {
    cut.walk2 = std::min(L.walk_cut2, L.cut2);
    if ((e = cudaMemsetAsync(L.exact_count, 0, 2 * sizeof(uint32_t), s))) return e;
  }
  probe_mark(s);
  if (fp64) {
    if (L.track) k_near64<true><<<grid, kNearWarps * 32, 0, s>>>(L.q64, n, L.src_perm, L.sq64, L.scode, L.cell_off, L.grid, cut, L.slices, L.partial, n);
    else k_near64<false><<<grid, kNearWarps * 32, 0, s>>>(L.q64, n, L.src_perm, L.sq64, L.scode, L.cell_off, L.grid, cut, L.slices, L.partial, n);
  } else {
    NearTask t = near_task(L);
    t.a.cut = cut;
    if (nearest_only && G == 1) {
      k_nearest_lane<<<(n + 255) / 256, 256, 0, s>>>(t.a);
      e = cudaGetLastError();
    } else {
      e = launch_near32(G, L.track, L.short_atan, nearest_only, grid, t.a, s);
    }
    if (e) return e;
  }
  probe_mark(s);
  probe_count();
  if (nearest_only) {
    // A warp per listed source, grid-stride; the list's length is read on the device.
    const int blocks = std::max(1, std::min((n + 3) / 4, 148 * 8));
    k_nearest_exact<<<blocks, 128, 0, s>>>(L.q32, L.gid, L.scode, L.simg, L.cell_off, L.grid, L.cut2, L.exact_list,
                                           L.exact_count, L.out, L.exact_count + 1);
    probe_count();
  }
  if ((e = launch_near_reduce(L, s))) return e;
  return cudaGetLastError();
}

// ------------------------------------------------------------------ many samples, one gather
// The gathers of many samples' passes in one persistent launch per tile variant (sources per
// warp and pair form; a batch has one or a few): every resident warp takes the next warp
// task (a sample's warp of sources and slice) from a device counter until all are done, so
// samples of any size share the GPU without a tail per sample. Tasks are in the order of
// `tasks` (largest first); prefix[k] is the first warp task of sample k. Each task runs the
// same warp function as the sample's own gather launch, so its rows are the same bit for
// bit. Relaxation steps only (no neighbour tracking, no spacing pass).
template <int G, bool SHORT>
__global__ void __launch_bounds__(kNearWarps * 32, 7) k_near32_batch(const NearTask* __restrict__ tasks,
                                                                    const uint32_t* __restrict__ prefix, int count,
                                                                    uint32_t total, uint32_t* __restrict__ counter) {
  __shared__ NearTileOf<false, SHORT, false> tiles[kNearWarps];
  __shared__ NearWalk<G> walks[kNearWarps];
  __shared__ double sums[6][kNearWarps * 32];
  __shared__ NearTask mine[kNearWarps];  // the warp's current task, copied in by its lanes
  static_assert(sizeof(NearTask) % 4 == 0, "task words");
  constexpr int kWords = (int)(sizeof(NearTask) / 4);
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  for (;;) {
    uint32_t t = 0;
    if (lane == 0) t = atomicAdd(counter, 1u);
    t = __shfl_sync(full, t, 0);
    if (t >= total) break;
    int lo = 0, hi = count - 1;  // the last sample whose first task is at most t
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (prefix[mid] <= t) lo = mid;
      else hi = mid - 1;
    }
    const uint32_t* from = reinterpret_cast<const uint32_t*>(&tasks[lo]);
    uint32_t* to = reinterpret_cast<uint32_t*>(&mine[w]);
    for (int k = lane; k < kWords; k += 32) to[k] = from[k];
    __syncwarp();
    const uint32_t local = t - prefix[lo];
    const uint32_t warps = (uint32_t)mine[w].warps;
    near32_warp<G, false, SHORT, false>(mine[w].a, (int)(local % warps), (int)(local / warps), tiles[w], walks[w],
                                        sums);
    __syncwarp();
  }
}

// Tile variant of a task: index into the six (sources per warp 2, 4, 8) x (pair form) kernels.
int near_variant(const NearTask& t) {
  return (t.group_size == 2 ? 0 : t.group_size == 4 ? 1 : 2) * 2 + (t.short_atan ? 1 : 0);
}

cudaError_t launch_near32_batch(const NearTask* tasks, const uint32_t* prefix, int count, uint32_t total,
                                uint32_t* counter, int variant, int sms, cudaStream_t s) {
  if (count <= 0 || total == 0) return cudaSuccess;
  cudaError_t e = cudaMemsetAsync(counter, 0, sizeof(uint32_t), s);
  if (e) return e;
  const uint32_t resident = (uint32_t)sms * 7;  // blocks of four warps, seven per SM
  const uint32_t blocks = std::max(1u, std::min(resident, (total + kNearWarps - 1) / kNearWarps));
  decltype(&k_near32_batch<4, true>) kernel;
  switch (variant) {
    case 0: kernel = k_near32_batch<2, false>; break;
    case 1: kernel = k_near32_batch<2, true>; break;
    case 2: kernel = k_near32_batch<4, false>; break;
    case 3: kernel = k_near32_batch<4, true>; break;
    case 4: kernel = k_near32_batch<8, false>; break;
    case 5: kernel = k_near32_batch<8, true>; break;
    default: return cudaErrorInvalidValue;
  }
  probe_mark(s);
  kernel<<<blocks, kNearWarps * 32, 0, s>>>(tasks, prefix, count, total, counter);
  probe_mark(s);
  probe_count();
  return cudaGetLastError();
}

}  // namespace zo
