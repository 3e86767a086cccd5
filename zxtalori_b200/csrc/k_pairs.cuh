// Tables, sampler, fold, scan and the all-pairs row kernels.
//
// All-pairs rows (shaders/pairs.wgsl:151-326, src/pairs.zig:52-128): one thread per source,
// 128 sources per block; the images j*g_k of a block's chunk stream through shared memory
// in tiles of 128 (each built once per block, in registers from the constant operator
// table, never stored in HBM). Tiles are plain FP32 sums merged into FP64 row sums
// once per tile. A chunk's partial rows are reduced in chunk order afterwards, so the sums
// do not depend on scheduling.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "k_common.cuh"
#include "kernels.h"

namespace zo {

cudaError_t upload_tables(const HostTables& t) {
  cudaError_t e;
  double4 ops64[kMaxOperatorRows], ops32[kMaxOperatorRows], planes64[kMaxPlaneRows];
  float4 planes32[kMaxPlaneRows];
  for (int r = 0; r < kMaxOperatorRows; ++r) {
    ops64[r] = make_double4(t.ops64[r][0], t.ops64[r][1], t.ops64[r][2], t.ops64[r][3]);
    ops32[r] = make_double4(t.ops32[r][0], t.ops32[r][1], t.ops32[r][2], t.ops32[r][3]);
  }
  for (int r = 0; r < kMaxPlaneRows; ++r) {
    planes64[r] = make_double4(t.planes64[r][0], t.planes64[r][1], t.planes64[r][2], t.planes64[r][3]);
    planes32[r] = make_float4(t.planes32[r][0], t.planes32[r][1], t.planes32[r][2], t.planes32[r][3]);
  }
  if ((e = cudaMemcpyToSymbol(c_ops64, ops64, sizeof(ops64)))) return e;
  if ((e = cudaMemcpyToSymbol(c_ops32, ops32, sizeof(ops32)))) return e;
  if ((e = cudaMemcpyToSymbol(c_planes64, planes64, sizeof(planes64)))) return e;
  if ((e = cudaMemcpyToSymbol(c_planes32, planes32, sizeof(planes32)))) return e;
  if ((e = cudaMemcpyToSymbol(c_plane_order, t.plane_order, sizeof(t.plane_order)))) return e;
  if ((e = cudaMemcpyToSymbol(c_plane_reach, t.plane_reach, sizeof(t.plane_reach)))) return e;
  if ((e = cudaMemcpyToSymbol(c_group_offset, t.group_offset, sizeof(int) * 11))) return e;
  if ((e = cudaMemcpyToSymbol(c_group_order, t.group_order, sizeof(int) * 11))) return e;
  return cudaMemcpyToSymbol(c_plane_offset, t.plane_offset, sizeof(int) * 11);
}

// ------------------------------------------------------------------ Haar sampler
__device__ __forceinline__ uint32_t hash32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  return x ^ (x >> 16);
}
__device__ __forceinline__ float unit_random(uint32_t v) {
  return ((float)(hash32(v) >> 8) + 0.5f) / 16777216.0f;
}

// Shoemake uniform quaternions (shaders/haar.wgsl:5-10): u, a, b exactly as the shader
// forms them in float32, the quaternion evaluated in FP64 and rounded once.
__global__ void k_haar(float4* __restrict__ q, int n, uint32_t seed_hash) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t base = hash32((uint32_t)i ^ seed_hash);
  const float two_pi = 6.28318530718f;
  const float u = unit_random(base);
  const float a = __fmul_rn(two_pi, unit_random(base + 1u));
  const float b = __fmul_rn(two_pi, unit_random(base + 2u));
  const double su = sqrt((double)u), sv = sqrt(1.0 - (double)u);
  double sa, ca, sb, cb;
  sincos((double)a, &sa, &ca);
  sincos((double)b, &sb, &cb);
  q[i] = make_float4((float)(su * cb), (float)(sv * sa), (float)(sv * ca), (float)(su * sb));
}

// ------------------------------------------------------------------ fold
// Normalisation of an imported float32 quaternion with the reference's exponent rescale
// (shaders/state.wgsl:31-40): components whose rescaled exponent would be subnormal become
// signed zeros; the power-of-two scale itself cancels in the FP64 normalisation.
__device__ __forceinline__ double4 flush_normalize(float4 a) {
  const unsigned int bx = __float_as_uint(a.x), by = __float_as_uint(a.y);
  const unsigned int bz = __float_as_uint(a.z), bw = __float_as_uint(a.w);
  const int ex = (bx >> 23) & 255, ey = (by >> 23) & 255, ez = (bz >> 23) & 255, ew = (bw >> 23) & 255;
  const int em = max(max(ex, ey), max(ez, ew));
  auto keep = [em](float v, int e) -> double {
    return (e > 0 && e + 127 - em > 0) ? (double)v : copysign(0.0, (double)v);
  };
  return normalize4(make_double4(keep(a.x, ex), keep(a.y, ey), keep(a.z, ez), keep(a.w, ew)));
}

// Every quaternion to its zone representative (shaders/state.wgsl:30-46, src/engine.zig:233).
__global__ void k_fold(float4* __restrict__ q32, double4* __restrict__ q64, int n, int gid, int prec, int from_q32) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const bool fp64 = prec == kFP64;
  double4 p = (from_q32 || !q64) ? flush_normalize(q32[i]) : normalize4(q64[i]);
  p = fold64(p, gid, !fp64);
  q32[i] = to_f4(p);
  if (q64) q64[i] = p;  // the FP64 master positions (both modes)
}

// ------------------------------------------------------------------ device-wide scan
// Exclusive scan of uint32 counts in tiles of 4096 (1024 threads x 4), block totals
// scanned by one block, then added back. out[count] receives the total.
constexpr int kScanTile = 4096;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* warp_sums, uint32_t& total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[wid] = x;
  __syncthreads();
  if (wid == 0) {
    uint32_t s = lane < (int)(blockDim.x >> 5) ? warp_sums[lane] : 0u;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    warp_sums[lane] = s;
  }
  __syncthreads();
  total = warp_sums[(blockDim.x >> 5) - 1];
  const uint32_t before = wid ? warp_sums[wid - 1] : 0u;
  __syncthreads();
  return before + x - v;
}

__global__ void __launch_bounds__(1024) k_scan_tiles(const uint32_t* __restrict__ in, uint32_t* __restrict__ out,
                                                      int max_count, const int* count_dev, uint32_t* block_sums) {
  __shared__ uint32_t warp_sums[32];
  const int count = count_dev ? min(*count_dev, max_count) : max_count;
  const int base = blockIdx.x * kScanTile;
  if (base >= count && !(blockIdx.x == 0)) return;
  uint32_t v[4];
  uint32_t local = 0;
  for (int r = 0; r < 4; ++r) {
    const int idx = base + threadIdx.x * 4 + r;
    v[r] = idx < count ? in[idx] : 0u;
    local += v[r];
  }
  uint32_t total;
  uint32_t at = block_exclusive_scan(local, warp_sums, total);
  for (int r = 0; r < 4; ++r) {
    const int idx = base + threadIdx.x * 4 + r;
    if (idx < count) out[idx] = at;
    at += v[r];
  }
  if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(1024) k_scan_sums(uint32_t* block_sums, uint32_t* __restrict__ out, int max_count,
                                                     const int* count_dev) {
  __shared__ uint32_t warp_sums[32];
  const int count = count_dev ? min(*count_dev, max_count) : max_count;
  const int blocks = (count + kScanTile - 1) / kScanTile;
  uint32_t v[4];
  uint32_t local = 0;
  for (int r = 0; r < 4; ++r) {
    const int idx = threadIdx.x * 4 + r;
    v[r] = idx < blocks ? block_sums[idx] : 0u;
    local += v[r];
  }
  uint32_t total;
  uint32_t at = block_exclusive_scan(local, warp_sums, total);
  for (int r = 0; r < 4; ++r) {
    const int idx = threadIdx.x * 4 + r;
    if (idx < blocks) block_sums[idx] = at;
    at += v[r];
  }
  if (threadIdx.x == 0) out[count] = total;
}

__global__ void k_scan_add(uint32_t* __restrict__ out, int max_count, const int* count_dev,
                           const uint32_t* __restrict__ block_sums) {
  const int count = count_dev ? min(*count_dev, max_count) : max_count;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx < count) out[idx] += block_sums[idx / kScanTile];
}

cudaError_t launch_scan(const uint32_t* in, uint32_t* out, int max_count, const int* count_dev, uint32_t* block_sums,
                        cudaStream_t s) {
  if (max_count > kScanTile * kScanTile) return cudaErrorInvalidValue;
  const int tiles = max(1, (max_count + kScanTile - 1) / kScanTile);
  k_scan_tiles<<<tiles, 1024, 0, s>>>(in, out, max_count, count_dev, block_sums);
  k_scan_sums<<<1, 1024, 0, s>>>(block_sums, out, max_count, count_dev);
  if (max_count > kScanTile) k_scan_add<<<(max_count + 255) / 256, 256, 0, s>>>(out, max_count, count_dev, block_sums);
  probe_count(max_count > kScanTile ? 3 : 2);
  return cudaGetLastError();
}

// ------------------------------------------------------------------ all-pairs rows
constexpr int kPairBlock = 128;

struct PairTile {
  int k, j0, count;
};
__device__ __forceinline__ PairTile pair_tile(int tile, int jtiles, int n) {
  PairTile t;
  t.k = tile / jtiles;
  t.j0 = (tile - t.k * jtiles) * kPairBlock;
  t.count = min(kPairBlock, n - t.j0);
  return t;
}

// FP32 rows (the relaxation's force pass, quey_partial semantics, shaders/pairs.wgsl:266-308):
// force and energy over every image of every other source; nearest over every image
// but the identity self pair. TRACK keeps the first image index of the nearest chord.
//
// A block holds 128 sources, one per thread, and walks tiles of 128 images of one operator
// built in shared memory; each thread evaluates two images per iteration with packed FP32
// arithmetic. The next tile's 128 points (2 KB, contiguous) are copied into shared memory by
// cp.async while the current tile's pairs run, one point per thread into a double buffer,
// so a tile starts without waiting on global memory. The tile stores the images as pairs, component by component (w, w', x, x')
// and (y, y', z, z'), plus 2|y|^2 of each, so one broadcast load gives a component of both.
// The near twin of an image is chosen by the sign of x . y; its difference d = x - y~
// gives the near chord |d|^2 directly and the far chord by the parallelogram law
// (2|x|^2 + 2|y|^2 - |d|^2 >= 2, no cancellation), and the force sum is
// sum coef (x - y~), turned into the tangent force once per source.
struct PairSlots {
  float4 wx[kPairBlock / 2];
  float4 yz[kPairBlock / 2];
  float2 n2[kPairBlock / 2];
};

// MASKED: the tile holds the thread's own source or ends in half a slot.
template <bool TRACK, bool MASKED>
__device__ __forceinline__ void pairs32_tile(const float4 x, float nx2, const PairSlots& S, int count, int i, int j0,
                                             int k, int n, float2& sw, float2& sx, float2& sy, float2& sz, float2& sc,
                                             float2& se, float& best, int& best_at) {
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
    const float2 farv = fma2(nearv, splat(-1.0f), add2(xn, S.n2[u]));
    float2 keep = splat(1.0f);  // force and energy weight of each pair
    float n0 = nearv.x, n1 = nearv.y;
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
    QueyPair2 p = quey_pair32x2(max2(nearv, 1e-30f), farv);
    if (MASKED) {
      p.coef = mul2(p.coef, keep);
      p.cr = mul2(p.cr, keep);
      p.rab = mul2(p.rab, keep);
    }
    sw = fma2(p.coef, dw, sw);
    sx = fma2(p.coef, dx, sx);
    sy = fma2(p.coef, dy, sy);
    sz = fma2(p.coef, dz, sz);
    sc = fma2(p.cs, p.cr, sc);
    se = add2(se, p.rab);  // energy / pi
  }
}

template <bool TRACK>
__global__ void __launch_bounds__(kPairBlock, 8) k_pairs32(const float4* __restrict__ q, int n, int op_off, int jtiles,
                                                           int total_tiles, int tiles_per_chunk, Rows out, int stride) {
  __shared__ PairSlots S;
  __shared__ float4 raw[2][kPairBlock];   // tile points as they arrive; thread t copies and reads point t
  __shared__ double sums[6][kPairBlock];  // FP64 row sums (shared: registers go to the pairs)
  const int i0 = blockIdx.x * kPairBlock;
  const int i = i0 + threadIdx.x;
  const bool live = i < n;
  const float4 x = live ? q[i] : make_float4(1.f, 0.f, 0.f, 0.f);
  const float nx2 = 2.0f * fmaf(x.x, x.x, fmaf(x.y, x.y, fmaf(x.z, x.z, x.w * x.w)));
  for (int k = 0; k < 6; ++k) sums[k][threadIdx.x] = 0.0;
  float best = 4.0f;
  int best_at = -1;
  const int t0 = blockIdx.y * tiles_per_chunk, t1 = min(total_tiles, t0 + tiles_per_chunk);
  const int slot = threadIdx.x >> 1, half = threadIdx.x & 1;
  // Copies this thread's point of tile `tile` into raw[buffer] (none past the tile's end);
  // one commit group per tile, empty or not, so the waits count tiles.
  auto stage = [&](int tile, int buffer) {
    const PairTile nt = pair_tile(tile, jtiles, n);
    if ((int)threadIdx.x < nt.count) copy_async16(&raw[buffer][threadIdx.x], &q[nt.j0 + threadIdx.x]);
    copy_async_commit();
  };
  if (t0 < t1) stage(t0, 0);
  for (int tid = t0; tid < t1; ++tid) {
    const PairTile pt = pair_tile(tid, jtiles, n);
    const int buffer = (tid - t0) & 1;
    // The other buffer was last read for the previous tile, before this thread went on.
    if (tid + 1 < t1) {
      stage(tid + 1, buffer ^ 1);
      copy_async_wait<1>();  // this tile's copy has landed; the next one may be in flight
    } else {
      copy_async_wait<0>();
    }
    __syncthreads();
    {
      const float4 y = (int)threadIdx.x < pt.count ? image32(raw[buffer][threadIdx.x], op_off + pt.k, pt.k == 0)
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
      pairs32_tile<TRACK, true>(x, nx2, S, pt.count, i, pt.j0, pt.k, n, sw, sx, sy, sz, sc, se, best, best_at);
    else
      pairs32_tile<TRACK, false>(x, nx2, S, pt.count, i, pt.j0, pt.k, n, sw, sx, sy, sz, sc, se, best, best_at);
    sums[0][threadIdx.x] += (double)sw.x + (double)sw.y;
    sums[1][threadIdx.x] += (double)sx.x + (double)sx.y;
    sums[2][threadIdx.x] += (double)sy.x + (double)sy.y;
    sums[3][threadIdx.x] += (double)sz.x + (double)sz.y;
    sums[4][threadIdx.x] += (double)sc.x + (double)sc.y;
    sums[5][threadIdx.x] += (double)se.x + (double)se.y;
  }
  if (!live) return;
  const size_t at = (size_t)blockIdx.y * stride + i;
  const double3 f = force_from_differences(
      to_d4(x), make_double4(sums[0][threadIdx.x], sums[1][threadIdx.x], sums[2][threadIdx.x], sums[3][threadIdx.x]));
  out.force[at] = make_double4(f.x, f.y, f.z, sums[4][threadIdx.x]);
  out.energy[at] = kPi * sums[5][threadIdx.x];
  out.nearest[at] = best;
  if (TRACK) out.nearest_at[at] = best_at;
}

// The same rows in FP64 (the plain method).
template <bool TRACK, bool CHECK>
__device__ __forceinline__ void pairs64_tile(const double4 x, const double4* tile, int count, int i, int j0, int k, int n,
                                             double& f1, double& f2, double& f3, double& fc, double& fe, double& best,
                                             int& best_at) {
  for (int t = 0; t < count; ++t) {
    const double4 y = tile[t];
    const double mw = x.x - y.x, mx = x.y - y.y, my = x.z - y.z, mz = x.w - y.w;
    const double pw = x.x + y.x, px = x.y + y.y, py = x.z + y.z, pz = x.w + y.w;
    const double dm2 = mw * mw + mx * mx + my * my + mz * mz;
    const double dp2 = pw * pw + px * px + py * py + pz * pz;
    const double c = fmin(dm2, dp2);
    const bool own = CHECK && (j0 + t == i);
    if (!(own && k == 0)) {
      if (c < best) {
        best = c;
        if (TRACK) best_at = k * n + j0 + t;
      }
    }
    if (own) continue;
    const PairD p = quey_pair64(dm2, dp2);
    double d1, d2, d3;
    pair_direction(x, y, d1, d2, d3);
    f1 += p.coef * d1;
    f2 += p.coef * d2;
    f3 += p.coef * d3;
    fc += p.curv;
    fe += p.energy;
  }
}

template <bool TRACK>
__global__ void __launch_bounds__(kPairBlock) k_pairs64(const double4* __restrict__ q, int n, int op_off, int jtiles,
                                                        int total_tiles, int tiles_per_chunk, Rows out, int stride) {
  __shared__ double4 tile[kPairBlock];
  const int i0 = blockIdx.x * kPairBlock;
  const int i = i0 + threadIdx.x;
  const bool live = i < n;
  const double4 x = live ? q[i] : make_double4(1, 0, 0, 0);
  double f1 = 0, f2 = 0, f3 = 0, fc = 0, fe = 0, best = 4.0;
  int best_at = -1;
  const int t0 = blockIdx.y * tiles_per_chunk, t1 = min(total_tiles, t0 + tiles_per_chunk);
  for (int tid = t0; tid < t1; ++tid) {
    const PairTile pt = pair_tile(tid, jtiles, n);
    __syncthreads();
    if ((int)threadIdx.x < pt.count) tile[threadIdx.x] = image64(q[pt.j0 + threadIdx.x], op_off + pt.k, pt.k == 0);
    __syncthreads();
    if (!live) continue;
    if (pt.j0 < i0 + kPairBlock && i0 < pt.j0 + pt.count)
      pairs64_tile<TRACK, true>(x, tile, pt.count, i, pt.j0, pt.k, n, f1, f2, f3, fc, fe, best, best_at);
    else
      pairs64_tile<TRACK, false>(x, tile, pt.count, i, pt.j0, pt.k, n, f1, f2, f3, fc, fe, best, best_at);
  }
  if (!live) return;
  const size_t at = (size_t)blockIdx.y * stride + i;
  out.force[at] = make_double4(f1, f2, f3, fc);
  out.energy[at] = fe;
  out.nearest[at] = best;
  if (TRACK) out.nearest_at[at] = best_at;
}

// Partial rows of `parts` chunks (or slices) summed into rows indexed by `dest` (identity
// when null). A block takes 32 rows (a lane per row, coalesced) and kReduceWarps warps: warp
// w sums chunks w, w + kReduceWarps, ... in order, then warp 0 adds the warps' sums in warp
// order, so the sums do not depend on how blocks were scheduled. The nearest keeps the
// earliest chunk among equal chords, as a walk through the chunks in order would.
constexpr int kReduceWarps = 8;
__global__ void __launch_bounds__(32 * kReduceWarps) k_rows_reduce(Rows part, int stride, int parts, int n,
                                                                   const int* __restrict__ dest, Rows out, int track) {
  __shared__ double4 sf[kReduceWarps][32];
  __shared__ double se[kReduceWarps][32], sb[kReduceWarps][32];
  __shared__ int sa[kReduceWarps][32], sc[kReduceWarps][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int p = blockIdx.x * 32 + lane;
  double4 f = make_double4(0, 0, 0, 0);
  double e = 0, best = 4.0;
  int best_at = -1, best_c = parts;
  if (p < n) {
    for (int c = w; c < parts; c += kReduceWarps) {
      const size_t at = (size_t)c * stride + p;
      const double4 g = part.force[at];
      f.x += g.x;
      f.y += g.y;
      f.z += g.z;
      f.w += g.w;
      e += part.energy[at];
      const double b = part.nearest[at];
      if (b < best) {
        best = b;
        best_c = c;
        if (track) best_at = part.nearest_at[at];
      }
    }
  }
  sf[w][lane] = f;
  se[w][lane] = e;
  sb[w][lane] = best;
  sa[w][lane] = best_at;
  sc[w][lane] = best_c;
  __syncthreads();
  if (w != 0 || p >= n) return;
  for (int k = 1; k < kReduceWarps; ++k) {
    const double4 g = sf[k][lane];
    f.x += g.x;
    f.y += g.y;
    f.z += g.z;
    f.w += g.w;
    e += se[k][lane];
    const double b = sb[k][lane];
    if (b < best || (b == best && sc[k][lane] < best_c)) {
      best = b;
      best_c = sc[k][lane];
      best_at = sa[k][lane];
    }
  }
  const int i = dest ? dest[p] : p;
  out.force[i] = f;
  out.energy[i] = e;
  out.nearest[i] = best;
  if (track) out.nearest_at[i] = best_at;
}

PairsPlan plan_pairs(int n, int order, double budget_scale, int sms) {
  PairsPlan pl;
  pl.jtiles = (n + kPairBlock - 1) / kPairBlock;
  pl.total_tiles = order * pl.jtiles;
  const int blocks = pl.jtiles;
  const int target = sms * 16;  // several resident blocks per SM, a few waves
  int chunks = (target + blocks - 1) / blocks;
  if (budget_scale > 0 && budget_scale < 1) chunks = (int)(chunks / budget_scale + 0.5);
  chunks = max(1, min(chunks, pl.total_tiles));
  pl.tiles_per_chunk = (pl.total_tiles + chunks - 1) / chunks;
  pl.chunks = (pl.total_tiles + pl.tiles_per_chunk - 1) / pl.tiles_per_chunk;
  return pl;
}

cudaError_t launch_pairs(int prec, bool track, const float4* q32, const double4* q64, int n, int gid, const PairsPlan& pl,
                         Rows partial, Rows out, cudaStream_t s) {
  const int op_off = host_group_offset(gid);
  const dim3 grid(pl.jtiles, pl.chunks);
  const bool direct = pl.chunks == 1;
  Rows dst = direct ? out : partial;
  probe_mark(s);
  if (prec == kFP64) {
    if (track) k_pairs64<true><<<grid, kPairBlock, 0, s>>>(q64, n, op_off, pl.jtiles, pl.total_tiles, pl.tiles_per_chunk, dst, n);
    else k_pairs64<false><<<grid, kPairBlock, 0, s>>>(q64, n, op_off, pl.jtiles, pl.total_tiles, pl.tiles_per_chunk, dst, n);
  } else {
    if (track) k_pairs32<true><<<grid, kPairBlock, 0, s>>>(q32, n, op_off, pl.jtiles, pl.total_tiles, pl.tiles_per_chunk, dst, n);
    else k_pairs32<false><<<grid, kPairBlock, 0, s>>>(q32, n, op_off, pl.jtiles, pl.total_tiles, pl.tiles_per_chunk, dst, n);
  }
  probe_mark(s);
  probe_count(direct ? 1 : 2);
  if (!direct)
    k_rows_reduce<<<(n + 31) / 32, 32 * kReduceWarps, 0, s>>>(partial, n, pl.chunks, n, nullptr, out, track ? 1 : 0);
  return cudaGetLastError();
}

cudaError_t launch_haar(float4* q, int n, uint32_t seed, cudaStream_t s) {
  // hash(seed) on the host side of the formula: base = hash(i ^ hash(seed)).
  uint32_t x = seed;
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  k_haar<<<(n + 255) / 256, 256, 0, s>>>(q, n, x);
  probe_count();
  return cudaGetLastError();
}

cudaError_t launch_fold(float4* q32, double4* q64, int n, int gid, int prec, bool from_q32, cudaStream_t s) {
  k_fold<<<(n + 255) / 256, 256, 0, s>>>(q32, q64, n, gid, prec, from_q32 ? 1 : 0);
  probe_count();
  return cudaGetLastError();
}

}  // namespace zo
