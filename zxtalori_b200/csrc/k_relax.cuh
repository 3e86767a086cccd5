// Barzilai-Borwein relaxation step, resident on the GPU (shaders/relax.wgsl,
// src/pairs.zig:339-363): FP64 inner products s.y, y.y, s.s, f.f and the energy total,
// the exact median curvature by radix select, the BB step length, then one fused pass that
// moves every source along its preconditioned force (clipped to half the mean radius),
// renormalises in FP64 and folds it into the zone. Nothing is read back.
#pragma once
#include "k_common.cuh"
#include "kernels.h"

namespace zo {

constexpr int kRelaxBlock = 256;

// Deterministic block sums: each block publishes its partials, the last block to finish
// adds them in block order (strided per thread, then a fixed tree).
template <int K>
__device__ __forceinline__ void block_partials(double (&v)[K], double* __restrict__ partials) {
  __shared__ double red[K][kRelaxBlock / 32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < K; ++c) {
    const double s = warp_sum(v[c]);
    if (lane == 0) red[c][w] = s;
  }
  __syncthreads();
  if (threadIdx.x < K) {
    double s = 0;
    for (int k = 0; k < kRelaxBlock / 32; ++k) s += red[threadIdx.x][k];
    partials[(size_t)blockIdx.x * K + threadIdx.x] = s;
  }
}
template <int K>
__device__ __forceinline__ void sum_partials(const double* __restrict__ partials, int blocks, double (&out)[K]) {
  __shared__ double red[K][kRelaxBlock / 32];
  double v[K];
#pragma unroll
  for (int c = 0; c < K; ++c) v[c] = 0;
  for (int b = threadIdx.x; b < blocks; b += blockDim.x)
#pragma unroll
    for (int c = 0; c < K; ++c) v[c] += partials[(size_t)b * K + c];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
  for (int c = 0; c < K; ++c) {
    const double s = warp_sum(v[c]);
    if (lane == 0) red[c][w] = s;
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < K; ++c) {
    double s = 0;
    for (int k = 0; k < kRelaxBlock / 32; ++k) s += red[c][k];
    out[c] = s;
  }
}

__device__ __forceinline__ bool finite3(double4 f) { return isfinite(f.x) && isfinite(f.y) && isfinite(f.z); }

// relax_stats + relax_sums (relax.wgsl:29-74): flags, the BB sums, and the radix select's
// starting ranks (lower and upper middle, equal for odd n).
__global__ void __launch_bounds__(kRelaxBlock) k_relax_stats(Rows rows, const double4* __restrict__ prev_f,
                                                             const double4* __restrict__ prev_d, int n, int fixed,
                                                             double* __restrict__ partials, RelaxDev* st) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool first = st->iteration == 0;
  double v[5] = {0, 0, 0, 0, 0};
  unsigned int flags = 0;
  if (i < n) {
    const double4 f = rows.force[i];
    if (!finite3(f)) flags |= 1u;
    if (!(rows.nearest[i] > 0.0)) flags |= 2u;
    v[3] = f.x * f.x + f.y * f.y + f.z * f.z;
    v[4] = rows.energy[i];
    if (!first && i != fixed) {
      const double4 s = prev_d[i], p = prev_f[i];
      const double yx = f.x - p.x, yy = f.y - p.y, yz = f.z - p.z;
      v[0] = s.x * yx + s.y * yy + s.z * yz;
      v[1] = yx * yx + yy * yy + yz * yz;
      v[2] = s.x * s.x + s.y * s.y + s.z * s.z;
    }
  }
  flags = __reduce_or_sync(0xffffffffu, flags);
  if ((threadIdx.x & 31) == 0 && flags) atomicOr(&st->flags, flags);
  block_partials<5>(v, partials);
  if (!last_block(&st->ticket)) return;
  double s[5];
  sum_partials<5>(partials, gridDim.x, s);
  if (threadIdx.x == 0) {
    for (int c = 0; c < 5; ++c) st->sums[c] = s[c];
    st->rank[0] = (unsigned long long)((n - 1) / 2);
    st->rank[1] = (unsigned long long)(n / 2);
    st->prefix[0] = st->prefix[1] = 0ull;
    st->step_bits = 0ull;
  }
}

// One radix round of the exact median of max(curvature, 0) (relax.wgsl:76-134), 8-bit
// digits, most significant first: float32 keys (FP32 mode, 4 rounds, as the reference's
// float rows) or FP64 keys (FP64 mode, 8 rounds). The last block picks the digit holding
// each middle rank; the last round sets the median, the BB step length and the iteration.
template <bool KEY64>
__global__ void __launch_bounds__(256) k_median_round(Rows rows, int n, int round, RelaxDev* st,
                                                      unsigned int* __restrict__ hist, double alpha0, double radius) {
  constexpr int kBits = KEY64 ? 64 : 32;
  constexpr int kRounds = kBits / 8;
  __shared__ unsigned int local[512];
  local[threadIdx.x] = 0;
  local[threadIdx.x + 256] = 0;
  __syncthreads();
  const int shift = kBits - 8 - 8 * round;
  const unsigned long long high = round == 0 ? 0ull : (~0ull << (kBits - 8 * round)) & (KEY64 ? ~0ull : 0xffffffffull);
  const unsigned long long p0 = st->prefix[0], p1 = st->prefix[1];
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double c = rows.force[i].w;
    unsigned long long key;
    if (KEY64) key = (unsigned long long)__double_as_longlong(c > 0.0 ? c : 0.0);
    else key = __float_as_uint(c > 0.0 ? (float)c : 0.0f);
    const unsigned int digit = (unsigned int)(key >> shift) & 255u;
    if ((key & high) == p0) atomicAdd(&local[digit], 1u);
    if ((key & high) == p1) atomicAdd(&local[256 + digit], 1u);
  }
  __syncthreads();
  for (int b = threadIdx.x; b < 512; b += 256)
    if (local[b]) atomicAdd(&hist[b], local[b]);
  if (!last_block(&st->ticket)) return;
  // Digit holding each rank: exclusive <= rank < inclusive, one thread per bin.
  __shared__ unsigned int scan[256];
  for (int r = 0; r < 2; ++r) {
    const unsigned int count = atomicAdd(&hist[256 * r + threadIdx.x], 0u);
    scan[threadIdx.x] = count;
    __syncthreads();
    for (int o = 1; o < 256; o <<= 1) {
      const unsigned int add = threadIdx.x >= (unsigned)o ? scan[threadIdx.x - o] : 0u;
      __syncthreads();
      scan[threadIdx.x] += add;
      __syncthreads();
    }
    const unsigned long long rank = st->rank[r];
    const unsigned int incl = scan[threadIdx.x], excl = incl - count;
    __syncthreads();
    if ((unsigned long long)excl <= rank && rank < (unsigned long long)incl) {
      st->rank[r] = rank - excl;
      st->prefix[r] |= (unsigned long long)threadIdx.x << shift;
    }
    hist[256 * r + threadIdx.x] = 0u;
    __syncthreads();
  }
  if (round == kRounds - 1 && threadIdx.x == 0) {
    double v0, v1;
    if (KEY64) {
      v0 = __longlong_as_double((long long)st->prefix[0]);
      v1 = __longlong_as_double((long long)st->prefix[1]);
    } else {
      v0 = (double)__uint_as_float((unsigned int)st->prefix[0]);
      v1 = (double)__uint_as_float((unsigned int)st->prefix[1]);
    }
    const double median = fmax(1e-12, 0.5 * (v0 + v1));
    st->median = median;
    const int it = st->iteration;
    double alpha = alpha0;
    if (it > 0) {
      const double sty = st->sums[0], yty = st->sums[1], sts = st->sums[2];
      const double a1 = fabs(yty) > 1e-20 ? fabs(sty / yty) : alpha0;
      const double a2 = fabs(sty) > 1e-20 ? fabs(sts / sty) : alpha0;
      alpha = fmin(fmax((it % 2 == 1) ? a1 : a2, 1e-12), fmax(1.0, 10.0 * radius));
    }
    st->alpha = alpha;
    st->iteration = it + 1;
  }
}

// relax_move (relax.wgsl:140-165) fused with the fold: d = f alpha/max(1e-6, c/median+0.01),
// clipped to 0.5 d_r, q <- normalize(exp(d) q), w >= 0, folded; FP64. The move starts from
// the FP64 master positions q64 and writes them back with their float32 rounding q32, which
// the pair kernels of FP32 mode read (without a master, q64 null, it starts from q32).
// A held identity stays (1,0,0,0); after a flag nothing moves.
__global__ void k_move_fold(float4* __restrict__ q32, double4* __restrict__ q64, int n, int gid, int prec, Rows rows,
                            double4* __restrict__ prev_f, double4* __restrict__ prev_d, RelaxDev* st, int fixed,
                            double radius, double step_scale) {
  if (st->flags != 0u) return;  // the step stopped (uniform across the grid)
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const bool fp64 = prec == kFP64;
  double moved_by = 0.0;  // this source's step length (>= 0)
  if (i < n && i == fixed) {
    prev_f[i] = make_double4(0, 0, 0, 0);
    prev_d[i] = make_double4(0, 0, 0, 0);
    q32[i] = make_float4(1.f, 0.f, 0.f, 0.f);
    if (q64) q64[i] = make_double4(1, 0, 0, 0);
  } else if (i < n) {
    const double alpha = st->alpha, median = st->median;
    const double4 f = rows.force[i];
    const double scale = alpha * step_scale / fmax(1e-6, f.w / median + 1e-2);
    const double size = sqrt(f.x * f.x + f.y * f.y + f.z * f.z) * scale;
    const double clip = fmin(1.0, 0.5 * radius / fmax(size, 1e-12));
    const double k = scale * clip;
    const double dx = f.x * k, dy = f.y * k, dz = f.z * k;
    prev_f[i] = make_double4(f.x, f.y, f.z, 0.0);
    prev_d[i] = make_double4(dx, dy, dz, 0.0);
    moved_by = size * clip;
    const double angle = sqrt(dx * dx + dy * dy + dz * dz);
    const double sinc = angle > 1e-4 ? sin(angle) / angle : 1.0 - angle * angle / 6.0;
    const double4 rot = make_double4(cos(angle), dx * sinc, dy * sinc, dz * sinc);
    const double4 qi = q64 ? q64[i] : to_d4(q32[i]);
    double4 moved = normalize4(qmul(rot, qi));
    moved = fold64(moved, gid, !fp64);
    q32[i] = to_f4(moved);
    if (q64) q64[i] = moved;
  }
  // The largest step: non-negative doubles order as their bit patterns; one atomic per warp.
  unsigned long long bits = (unsigned long long)__double_as_longlong(moved_by);
  for (int o = 16; o; o >>= 1) {
    const unsigned long long other = __shfl_xor_sync(0xffffffffu, bits, o);
    bits = other > bits ? other : bits;
  }
  if ((threadIdx.x & 31) == 0 && bits) atomicMax(&st->step_bits, bits);
}

// A nearest chord^2 as the SO(3) angle in degrees, rounded to float (pairs.wgsl:428-434).
__device__ __forceinline__ float nearest_degrees_of(double chord2) {
  const double c = fmin(1.0, sqrt(fmax(chord2, 0.0)) * 0.5);
  return (float)(4.0 * asin(c) * (180.0 / kPi));
}

// Quick measures of a force pass (src/pairs.zig:130-140, 182-199): energy sum, force^2 sum
// and the smallest nearest chord with its source, deterministic. A nearest-only pass (the
// spacing pass) writes no forces or energies, and its sums are left 0.
__global__ void __launch_bounds__(kRelaxBlock) k_row_summary(Rows rows, int n, double* __restrict__ partials,
                                                             double* __restrict__ near_partials,
                                                             int* __restrict__ near_rows, RowSummary* out,
                                                             int nearest_only) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double v[2] = {0, 0};
  double best = 4.0;
  int at = -1;
  if (i < n) {
    if (!nearest_only) {
      const double4 f = rows.force[i];
      v[0] = rows.energy[i];
      v[1] = f.x * f.x + f.y * f.y + f.z * f.z;
    }
    best = rows.nearest[i];
    at = i;
  }
  block_partials<2>(v, partials);
  // Block minimum with the lowest row on ties.
  for (int o = 16; o; o >>= 1) {
    const double b2 = __shfl_xor_sync(0xffffffffu, best, o);
    const int a2 = __shfl_xor_sync(0xffffffffu, at, o);
    if (b2 < best || (b2 == best && a2 >= 0 && (at < 0 || a2 < at))) {
      best = b2;
      at = a2;
    }
  }
  __shared__ double wb[kRelaxBlock / 32];
  __shared__ int wa[kRelaxBlock / 32];
  if ((threadIdx.x & 31) == 0) {
    wb[threadIdx.x >> 5] = best;
    wa[threadIdx.x >> 5] = at;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = wb[0];
    int a = wa[0];
    for (int k = 1; k < kRelaxBlock / 32; ++k)
      if (wb[k] < b) {
        b = wb[k];
        a = wa[k];
      }
    near_partials[blockIdx.x] = b;
    near_rows[blockIdx.x] = a;
  }
  if (!last_block(&out->ticket)) return;
  double s[2];
  sum_partials<2>(partials, gridDim.x, s);
  // The blocks' minima, reduced by the whole block: smallest chord, then lowest row (rows
  // grow with the block index, so this is the first block holding the minimum).
  double b = 4.0;
  int a = -1;
  for (int k = threadIdx.x; k < (int)gridDim.x; k += blockDim.x) {
    const double v = near_partials[k];
    const int r = near_rows[k];
    if (v < b || (v == b && r >= 0 && (a < 0 || r < a))) {
      b = v;
      a = r;
    }
  }
  for (int o = 16; o; o >>= 1) {
    const double b2 = __shfl_xor_sync(0xffffffffu, b, o);
    const int a2 = __shfl_xor_sync(0xffffffffu, a, o);
    if (b2 < b || (b2 == b && a2 >= 0 && (a < 0 || a2 < a))) {
      b = b2;
      a = a2;
    }
  }
  __syncthreads();  // wb / wa reused
  if ((threadIdx.x & 31) == 0) {
    wb[threadIdx.x >> 5] = b;
    wa[threadIdx.x >> 5] = a;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int k = 1; k < kRelaxBlock / 32; ++k)
      if (wb[k] < b || (wb[k] == b && wa[k] >= 0 && (a < 0 || wa[k] < a))) {
        b = wb[k];
        a = wa[k];
      }
    out->energy = s[0];
    out->force2 = s[1];
    out->nearest = b;
    out->nearest_row = a;
    out->least_degrees = nearest_degrees_of(b);  // the point value of the nearest source
  }
}

// Per-source nearest orbit neighbour as an SO(3) angle in degrees (pairs.wgsl:428-434).
__global__ void k_nearest_degrees(const double* __restrict__ nearest, int n, float* __restrict__ out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = nearest_degrees_of(nearest[i]);
}

// FP32 mode: the nearest chord of each source's chosen neighbour recomputed in FP64 from
// the float32 positions (images formed in FP64), so separations carry FP64 accuracy.
// `near_sites` selects the near-field encoding of `nearest_at` (a sorted site) over the
// all-pairs one (image index k*n+j). Also writes each source's neighbour source index.
// The group's operator rows are copied into shared memory first: each thread reads the row
// of its own neighbour's image, and constant memory would serve a warp's distinct rows one
// after another.
__global__ void __launch_bounds__(256) k_refine_nearest(const float4* __restrict__ q32, int n, int gid, Rows rows,
                                                        int near_sites, const uint32_t* __restrict__ scode,
                                                        const uint32_t* __restrict__ simg,
                                                        int* __restrict__ neighbour) {
  __shared__ double4 ops[kMaxGroupOrder];
  {
    const int off = c_group_offset[gid], order = c_group_order[gid];
    for (int k = threadIdx.x; k < order; k += blockDim.x) ops[k] = c_ops32[off + k];
  }
  __syncthreads();
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int at = rows.nearest_at[i];
  if (at < 0) {  // no orbit neighbour within the cutoff
    rows.nearest[i] = 4.0;
    neighbour[i] = -1;
    return;
  }
  int j, op;
  bool neg = false, any_sign = false;
  if (near_sites) {
    j = (int)(scode[at] & ~kIdentityBit);
    const uint32_t im = simg[at];
    op = (int)(im >> 1);
    neg = (im & 1u) != 0;
  } else {
    op = at / n;
    j = at - op * n;
    any_sign = true;
  }
  const double4 x = normalize4(to_d4(q32[i]));
  double4 y = normalize4(op == 0 ? to_d4(q32[j]) : qmul(to_d4(q32[j]), ops[op]));
  if (neg) y = neg4(y);
  const double mw = x.x - y.x, mx = x.y - y.y, my = x.z - y.z, mz = x.w - y.w;
  double c = mw * mw + mx * mx + my * my + mz * mz;
  if (any_sign) {
    const double pw = x.x + y.x, px = x.y + y.y, py = x.z + y.z, pz = x.w + y.w;
    c = fmin(c, pw * pw + px * px + py * py + pz * pz);
  }
  rows.nearest[i] = c;
  neighbour[i] = j;
}

// FP64 mode: neighbour source indices from the tracked positions.
__global__ void k_neighbour_index(const Rows rows, int n, int near_sites, const uint32_t* __restrict__ scode,
                                  int* __restrict__ neighbour) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int at = rows.nearest_at[i];
  if (at < 0) neighbour[i] = -1;
  else neighbour[i] = near_sites ? (int)(scode[at] & ~kIdentityBit) : at % n;
}

}  // namespace zo
