// Full pair measures (shaders/pairs.wgsl:151-244, src/pairs.zig:52-84): per source, over
// every image but the identity self pair, the Riesz s=1,2,3 chord sums, the Green kernel,
// the logarithmic energy, plus the force-pass row (force, curvature, Quey energy, nearest).
//
// The log remainder is summed in FP64 as a product of unit-chord terms per tile, rescaled by
// powers of two and logged once per tile (the reference emulates the same with
// double-single floats; B200 runs FP64 natively). In FP32 mode the other sums use FP32
// pair arithmetic on the float32 images and the log uses the FP64 images; in FP64 mode
// everything is FP64. The self pair's antipode (1/2, 1/4, 1/8, -3/(8 pi^2), 1/4 - ln 2) is
// added by the host.
#pragma once
#include "k_common.cuh"
#include "kernels.h"

namespace zo {

struct FullTile32 {
  float4 y32[kPairBlock];
  double4 y64[kPairBlock];
};

// Multiply `prod` by `term`, keeping the product's exponent in `expo` every 8 terms.
__device__ __forceinline__ void log_product(double& prod, int& expo, int& pending, double term) {
  prod *= term;
  if (++pending == 8) {
    int e;
    prod = frexp(prod, &e);
    expo += e;
    pending = 0;
  }
}
__device__ __forceinline__ double log_total(double prod, int expo) {
  return log(prod) + (double)expo * 0.69314718055994530942;
}

template <bool CHECK>
__device__ __forceinline__ void full32_tile(const float4 x, const double4 x64, const FullTile32& tile, int count, int i,
                                            int j0, int k, int n, float* s, double& lsum, int& degenerate,
                                            float& best, int& best_at) {
  // s: force xyz, curvature, energy, riesz1, riesz2, riesz3, green
  double prod = 1.0;
  int expo = 0, pending = 0, terms = 0;
  for (int t = 0; t < count; ++t) {
    const float4 y = tile.y32[t];
    const float mw = x.x - y.x, mx = x.y - y.y, my = x.z - y.z, mz = x.w - y.w;
    const float pw = x.x + y.x, px = x.y + y.y, py = x.z + y.z, pz = x.w + y.w;
    const float dm2 = fmaf(mw, mw, fmaf(mx, mx, fmaf(my, my, mz * mz)));
    const float dp2 = fmaf(pw, pw, fmaf(px, px, fmaf(py, py, pz * pz)));
    const bool own = CHECK && (j0 + t == i);
    const bool self = own && k == 0;
    if (self) continue;
    const float c = fminf(dm2, dp2);
    if (c < best) {
      best = c;
      best_at = k * n + j0 + t;
    }
    const PairF p = quey_pair32(dm2, dp2);
    const float im = rsqrtf(fmaxf(dm2, 1e-30f)), ip = rsqrtf(fmaxf(dp2, 1e-30f));
    const float im2 = im * im, ip2 = ip * ip;
    s[5] += im + ip;
    s[6] += im2 + ip2;
    s[7] += fmaf(im2, im, ip2 * ip);
    const float cot = fabsf(dp2 - dm2) * 0.5f * im * ip;
    s[8] += fmaf(kPiF - 2.0f * p.a, cot, -1.0f);
    const double4 y64 = tile.y64[t];
    const double aw = x64.x - y64.x, ax = x64.y - y64.y, ay = x64.z - y64.z, az = x64.w - y64.w;
    const double bw = x64.x + y64.x, bx = x64.y + y64.y, by = x64.z + y64.z, bz = x64.w + y64.w;
    const double term = (aw * aw + ax * ax + ay * ay + az * az) * (bw * bw + bx * bx + by * by + bz * bz);
    degenerate |= !(term > 0.0);
    log_product(prod, expo, pending, term);
    ++terms;
    if (own) continue;
    float d1, d2, d3;
    pair_direction(x, y, d1, d2, d3);
    s[0] = fmaf(p.coef, d1, s[0]);
    s[1] = fmaf(p.coef, d2, s[1]);
    s[2] = fmaf(p.coef, d3, s[2]);
    s[3] += p.curv;
    s[4] += p.energy;
  }
  if (terms > 0) lsum += -0.5 * log_total(prod, expo) + 0.5 * terms;
}

template <bool CHECK>
__device__ __forceinline__ void full64_tile(const double4 x, const double4* tile, int count, int i, int j0, int k, int n,
                                            double* s, double& lsum, int& degenerate, double& best, int& best_at) {
  double prod = 1.0;
  int expo = 0, pending = 0, terms = 0;
  for (int t = 0; t < count; ++t) {
    const double4 y = tile[t];
    const double mw = x.x - y.x, mx = x.y - y.y, my = x.z - y.z, mz = x.w - y.w;
    const double pw = x.x + y.x, px = x.y + y.y, py = x.z + y.z, pz = x.w + y.w;
    const double dm2 = mw * mw + mx * mx + my * my + mz * mz;
    const double dp2 = pw * pw + px * px + py * py + pz * pz;
    const bool own = CHECK && (j0 + t == i);
    const bool self = own && k == 0;
    if (self) continue;
    const double c = fmin(dm2, dp2);
    if (c < best) {
      best = c;
      best_at = k * n + j0 + t;
    }
    const PairD p = quey_pair64(dm2, dp2);
    const double im = 1.0 / sqrt(fmax(dm2, 1e-30)), ip = 1.0 / sqrt(fmax(dp2, 1e-30));
    s[5] += im + ip;
    s[6] += im * im + ip * ip;
    s[7] += im * im * im + ip * ip * ip;
    const double cot = fabs(dp2 - dm2) * 0.5 * im * ip;
    s[8] += (kPi - 2.0 * p.a) * cot - 1.0;
    const double term = dm2 * dp2;
    degenerate |= !(term > 0.0);
    log_product(prod, expo, pending, term);
    ++terms;
    if (own) continue;
    double d1, d2, d3;
    pair_direction(x, y, d1, d2, d3);
    s[0] += p.coef * d1;
    s[1] += p.coef * d2;
    s[2] += p.coef * d3;
    s[3] += p.curv;
    s[4] += p.energy;
  }
  if (terms > 0) lsum += -0.5 * log_total(prod, expo) + 0.5 * terms;
}

// Partial full rows [chunk][n]: `rows` as the force pass, `extra` 5 doubles per source
// (riesz1, riesz2, riesz3, green, log) and a degenerate flag.
__global__ void __launch_bounds__(kPairBlock) k_full32(const float4* __restrict__ q, int n, int op_off, int jtiles,
                                                       int total_tiles, int tiles_per_chunk, Rows out,
                                                       double* __restrict__ extra, int* __restrict__ degen, int stride) {
  __shared__ FullTile32 tile;
  const int i0 = blockIdx.x * kPairBlock;
  const int i = i0 + threadIdx.x;
  const bool live = i < n;
  const float4 x = live ? q[i] : make_float4(1.f, 0.f, 0.f, 0.f);
  const double4 x64 = normalize4(to_d4(x));
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  double lsum = 0.0;
  int degenerate = 0;
  float best = 4.0f;
  int best_at = -1;
  const int t0 = blockIdx.y * tiles_per_chunk, t1 = min(total_tiles, t0 + tiles_per_chunk);
  for (int tid = t0; tid < t1; ++tid) {
    const PairTile pt = pair_tile(tid, jtiles, n);
    __syncthreads();
    if ((int)threadIdx.x < pt.count) {
      const float4 qj = q[pt.j0 + threadIdx.x];
      const double4 y64 = pt.k == 0 ? normalize4(to_d4(qj)) : normalize4(qmul(to_d4(qj), c_ops32[op_off + pt.k]));
      tile.y64[threadIdx.x] = y64;
      tile.y32[threadIdx.x] = pt.k == 0 ? qj : to_f4(y64);
    }
    __syncthreads();
    if (!live) continue;
    float s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (pt.j0 < i0 + kPairBlock && i0 < pt.j0 + pt.count)
      full32_tile<true>(x, x64, tile, pt.count, i, pt.j0, pt.k, n, s, lsum, degenerate, best, best_at);
    else
      full32_tile<false>(x, x64, tile, pt.count, i, pt.j0, pt.k, n, s, lsum, degenerate, best, best_at);
#pragma unroll
    for (int c = 0; c < 9; ++c) acc[c] += s[c];
  }
  if (!live) return;
  const size_t at = (size_t)blockIdx.y * stride + i;
  out.force[at] = make_double4(acc[0], acc[1], acc[2], acc[3]);
  out.energy[at] = acc[4];
  out.nearest[at] = best;
  out.nearest_at[at] = best_at;
  extra[at * 5 + 0] = acc[5];
  extra[at * 5 + 1] = acc[6];
  extra[at * 5 + 2] = acc[7];
  extra[at * 5 + 3] = acc[8] / (4.0 * kPi * kPi);
  extra[at * 5 + 4] = lsum;
  degen[at] = degenerate;
}

__global__ void __launch_bounds__(kPairBlock) k_full64(const double4* __restrict__ q, int n, int op_off, int jtiles,
                                                       int total_tiles, int tiles_per_chunk, Rows out,
                                                       double* __restrict__ extra, int* __restrict__ degen, int stride) {
  __shared__ double4 tile[kPairBlock];
  const int i0 = blockIdx.x * kPairBlock;
  const int i = i0 + threadIdx.x;
  const bool live = i < n;
  const double4 x = live ? normalize4(q[i]) : make_double4(1, 0, 0, 0);
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  double lsum = 0.0, best = 4.0;
  int degenerate = 0, best_at = -1;
  const int t0 = blockIdx.y * tiles_per_chunk, t1 = min(total_tiles, t0 + tiles_per_chunk);
  for (int tid = t0; tid < t1; ++tid) {
    const PairTile pt = pair_tile(tid, jtiles, n);
    __syncthreads();
    if ((int)threadIdx.x < pt.count) {
      const double4 qj = q[pt.j0 + threadIdx.x];
      tile[threadIdx.x] = pt.k == 0 ? normalize4(qj) : normalize4(qmul(qj, c_ops64[op_off + pt.k]));
    }
    __syncthreads();
    if (!live) continue;
    double s[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (pt.j0 < i0 + kPairBlock && i0 < pt.j0 + pt.count)
      full64_tile<true>(x, tile, pt.count, i, pt.j0, pt.k, n, s, lsum, degenerate, best, best_at);
    else
      full64_tile<false>(x, tile, pt.count, i, pt.j0, pt.k, n, s, lsum, degenerate, best, best_at);
#pragma unroll
    for (int c = 0; c < 9; ++c) acc[c] += s[c];
  }
  if (!live) return;
  const size_t at = (size_t)blockIdx.y * stride + i;
  out.force[at] = make_double4(acc[0], acc[1], acc[2], acc[3]);
  out.energy[at] = acc[4];
  out.nearest[at] = best;
  out.nearest_at[at] = best_at;
  extra[at * 5 + 0] = acc[5];
  extra[at * 5 + 1] = acc[6];
  extra[at * 5 + 2] = acc[7];
  extra[at * 5 + 3] = acc[8] / (4.0 * kPi * kPi);
  extra[at * 5 + 4] = lsum;
  degen[at] = degenerate;
}

// Chunks summed as k_rows_reduce does (warp w takes chunks w, w + kReduceWarps, ...; warp 0
// adds the warps' sums in warp order), extras and degenerate flags alongside.
__global__ void __launch_bounds__(32 * kReduceWarps) k_full_reduce(Rows part, const double* __restrict__ pextra,
                                                                   const int* __restrict__ pdegen, int parts, int n,
                                                                   Rows out, double* __restrict__ extra,
                                                                   int* __restrict__ degen) {
  __shared__ double sv[kReduceWarps][6][32];  // force xyzw, energy, nearest
  __shared__ double sx[kReduceWarps][5][32];
  __shared__ int sa[kReduceWarps][32], sc[kReduceWarps][32], sd[kReduceWarps][32];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int i = blockIdx.x * 32 + lane;
  double4 f = make_double4(0, 0, 0, 0);
  double e = 0, best = 4.0, x[5] = {0, 0, 0, 0, 0};
  int best_at = -1, best_c = parts, dg = 0;
  if (i < n) {
    for (int c = w; c < parts; c += kReduceWarps) {
      const size_t at = (size_t)c * n + i;
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
        best_at = part.nearest_at[at];
      }
      for (int r = 0; r < 5; ++r) x[r] += pextra[at * 5 + r];
      dg |= pdegen[at];
    }
  }
  sv[w][0][lane] = f.x;
  sv[w][1][lane] = f.y;
  sv[w][2][lane] = f.z;
  sv[w][3][lane] = f.w;
  sv[w][4][lane] = e;
  sv[w][5][lane] = best;
  for (int r = 0; r < 5; ++r) sx[w][r][lane] = x[r];
  sa[w][lane] = best_at;
  sc[w][lane] = best_c;
  sd[w][lane] = dg;
  __syncthreads();
  if (w != 0 || i >= n) return;
  for (int k = 1; k < kReduceWarps; ++k) {
    f.x += sv[k][0][lane];
    f.y += sv[k][1][lane];
    f.z += sv[k][2][lane];
    f.w += sv[k][3][lane];
    e += sv[k][4][lane];
    const double b = sv[k][5][lane];
    if (b < best || (b == best && sc[k][lane] < best_c)) {
      best = b;
      best_c = sc[k][lane];
      best_at = sa[k][lane];
    }
    for (int r = 0; r < 5; ++r) x[r] += sx[k][r][lane];
    dg |= sd[k][lane];
  }
  out.force[i] = f;
  out.energy[i] = e;
  out.nearest[i] = best;
  out.nearest_at[i] = best_at;
  for (int r = 0; r < 5; ++r) extra[(size_t)i * 5 + r] = x[r];
  degen[i] = dg;
}

cudaError_t launch_full(int prec, const float4* q32, const double4* q64, int n, int gid, const PairsPlan& pl, Rows partial,
                        double* pextra, int* pdegen, Rows out, double* extra, int* degen, cudaStream_t s) {
  const int op_off = host_group_offset(gid);
  const dim3 grid(pl.jtiles, pl.chunks);
  const bool direct = pl.chunks == 1;
  Rows dst = direct ? out : partial;
  double* dx = direct ? extra : pextra;
  int* dd = direct ? degen : pdegen;
  if (prec == kFP64)
    k_full64<<<grid, kPairBlock, 0, s>>>(q64, n, op_off, pl.jtiles, pl.total_tiles, pl.tiles_per_chunk, dst, dx, dd, n);
  else
    k_full32<<<grid, kPairBlock, 0, s>>>(q32, n, op_off, pl.jtiles, pl.total_tiles, pl.tiles_per_chunk, dst, dx, dd, n);
  if (!direct)
    k_full_reduce<<<(n + 31) / 32, 32 * kReduceWarps, 0, s>>>(partial, pextra, pdegen, pl.chunks, n, out, extra, degen);
  return cudaGetLastError();
}

}  // namespace zo
