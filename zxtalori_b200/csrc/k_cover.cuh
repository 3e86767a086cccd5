// Covering radius: the largest empty cap of the sample's full orbit {+-q_j g_k} on S3.
//
// The spherical Delaunay triangulation of the orbit is its convex hull in R4; a hull facet
// through the orbit points x, y_a, y_b, y_c has the unit normal n and offset h = n . x with
// n . y <= h for every orbit point y, and its cap {z : n . z >= h} (centre n, angular radius
// acos h) holds no orbit point inside. The covering radius is the largest such cap
// (tests/test_covering.py:8-15 states it through Qhull). Every facet is an image of one that
// touches a representative, so it is enough to build each representative's star, the
// facets that touch it (src/covering.zig measures the same quantity with its own shell
// triangulation; this is a different construction).
//
// One warp per source x:
//  1. Collect the orbit points within a reach of x (squared chord reach2, excluding x
//     itself), from the near-field structure's sorted shell sites and chart grid (every
//     orbit point within its radius of the zone is a site) or, for small samples, from every
//     image. Positions are the float32 sample, images formed and normalised in FP64 from the
//     float32 operator table (the oracle's definition). The points are put in a canonical
//     order (by source, then image) so the result does not depend on the collection order.
//  2. Gift-wrap the star in FP64: from the tangent hyperplane at x, three pivots give a
//     first facet; each facet's three faces through x are pivoted to their neighbouring
//     facets until no new facet appears. A pivot about the face (x, y_p, y_q) of a facet
//     with normal n turns the hyperplane about that face, n(t) = cos t n + sin t v with
//     v _|_ n, y_p - x, y_q - x and v . (y_o - x) < 0 (away from the dropped vertex o); the
//     first point it meets is the one with the largest cot t_m = (v . d_m) / (-n . d_m),
//     d_m = y_m - x, and the new facet's normal is r n + v normalised (r that cot), kept
//     with the facet: recomputing it from the facet's vertices is ill-conditioned for the
//     flat facets of co-spherical points (lattices). A point already on the hyperplane
//     (co-spherical with the facet) is met at once, unless it lies on the face's own line.
//  3. Certificate: a facet whose cap has radius a lies within 2a of x (x is on its rim), so
//     when every facet of the star has 2a within the reach, no point outside the reach can
//     enter any of them and the star is exact. Otherwise the source reports the reach it
//     needs and the host runs it again with that reach.
//
// Outputs per source: the largest cap (S3 angle) of its star and the cap's centre, the
// number of distinct neighbours its star touches (the faces of its Voronoi cell), the
// number of facets, and a status (kCoverOk, or why the star is not certified).
#pragma once
#include "k_common.cuh"
#include "kernels.h"
#include "k_near.cuh"  // cell_axis, NearGrid: the chart grid the collection walks
#include "qvm_device.cuh"

namespace zo {

constexpr int kCoverWarps = 4;
constexpr int kCoverMax = 256;      // neighbours per source (the wide star)
constexpr int kCoverFacets = 256;   // facets per star (the wide star)
// The first pass over every source uses a narrow star: 64 neighbours (the reach is sized to
// hold 48 on average) and 128 facets (a star of V neighbours closes with 2V - 4 facets), so a
// warp's shared memory is 8 KB instead of 19 KB and three times as many warps stay resident;
// a source that overflows it is sent to the wide star at the same reach.
constexpr int kCoverMaxNarrow = 64;
constexpr int kCoverFacetsNarrow = 128;
// Reruns (a reach wider than the first) start in a middle star of 128 neighbours and 256
// facets (15 KB per warp), then go to the wide one.
constexpr int kCoverMaxMiddle = 128;
constexpr int kCoverFacetsMiddle = 256;

template <int NB, int NF>
struct CoverStar {
  static constexpr int kPoints = NB, kFacets = NF;
  double4 d[NB];                   // y_m - x in canonical order
  uint32_t key[NB];                // (source << 8) | image of each collected point
  uint32_t facet[NF];              // a | b << 8 | c << 16, a < b < c
  double4 normal[NF];              // each facet's unit normal, oriented to its cap
  uint32_t used[NB / 32];          // neighbours touched by some facet
  float4 image_dot[kMaxGroupOrder];  // dense collection: x g_k^-1 / |g_k| (float32)
  int total;                       // points within the reach (may exceed NB)
};
static_assert(kCoverMax <= 256 && kCoverMaxNarrow <= kCoverMaxMiddle && kCoverMaxMiddle <= kCoverMax,
              "facet keys hold 8-bit neighbour indices");

// A vector orthogonal to a, b and c (the 4-D generalised cross product).
__device__ __forceinline__ double4 cross4(double4 a, double4 b, double4 c) {
  const double m01 = b.x * c.y - b.y * c.x, m02 = b.x * c.z - b.z * c.x, m03 = b.x * c.w - b.w * c.x;
  const double m12 = b.y * c.z - b.z * c.y, m13 = b.y * c.w - b.w * c.y, m23 = b.z * c.w - b.w * c.z;
  return make_double4(a.y * m23 - a.z * m13 + a.w * m12, -(a.x * m23 - a.z * m03 + a.w * m02),
                      a.x * m13 - a.y * m03 + a.w * m01, -(a.x * m12 - a.y * m02 + a.z * m01));
}
__device__ __forceinline__ double4 unit4(double4 a) {
  const double s = dot4(a, a);
  return s > 0.0 ? scale4(a, 1.0 / sqrt(s)) : a;
}
__device__ __forceinline__ double4 sub4d(double4 a, double4 b) {
  return make_double4(a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w);
}
__device__ __forceinline__ double4 axpy4(double s, double4 x, double4 y) {  // s x + y
  return make_double4(fma(s, x.x, y.x), fma(s, x.y, y.y), fma(s, x.z, y.z), fma(s, x.w, y.w));
}

// Orbit point `key` = (source j << 8) | image (2 * operator + sign), unit, in FP64.
__device__ __forceinline__ double4 cover_point(const float4* __restrict__ q, const double4* ops, uint32_t key) {
  const uint32_t j = key >> 8, im = key & 0xffu;
  const int op = (int)(im >> 1);
  double4 y = normalize4(op == 0 ? to_d4(q[j]) : qmul(to_d4(q[j]), ops[op]));
  return (im & 1u) ? neg4(y) : y;
}

// The pivot: of the points other than the excluded ones, the first that the hyperplane
// (normal n) meets when turned towards v, and r = cot of the turn; -1 when none. Ties go to
// the lower index. A point on the hyperplane already (-n . d within rounding of 0: co-spherical
// points) is met at once (r = inf) when it lies on v's side of the face by more than rounding,
// never otherwise: a point on the face's own line would make a flat facet. Warp-uniform.
template <class Star>
__device__ __forceinline__ int cover_pivot(const Star& W, int count, double4 n, double4 v, int e0, int e1,
                                           int e2, double& r_out) {
  const unsigned full = 0xffffffffu;
  double best = -INFINITY;
  int at = -1;
  for (int m = threadIdx.x & 31; m < count; m += 32) {
    if (m == e0 || m == e1 || m == e2) continue;
    const double4 d = W.d[m];
    const double a = -dot4(n, d), b = dot4(v, d);
    double r;
    const double d2 = dot4(d, d);
    if (a > 1e-13 * d2) r = b / a;
    else if (b > 1e-10 * sqrt(d2)) r = INFINITY;
    else continue;
    if (r > best) {  // lanes visit m in increasing order: the first of equals is kept
      best = r;
      at = m;
    }
  }
  for (int o = 16; o; o >>= 1) {
    const double ob = __shfl_xor_sync(full, best, o);
    const int oa = __shfl_xor_sync(full, at, o);
    if (oa >= 0 && (at < 0 || ob > best || (ob == best && oa < at))) {
      best = ob;
      at = oa;
    }
  }
  r_out = best;
  return at;
}

// The hyperplane n turned towards v until it meets a point with cot r: r n + v, or n itself
// when the point was on it already (r = inf).
__device__ __forceinline__ double4 cover_turn(double4 n, double4 v, double r) {
  return isinf(r) ? n : unit4(axpy4(r, n, v));
}

__device__ __forceinline__ uint32_t facet_key(int a, int b, int c) {
  int t;
  if (a > b) { t = a; a = b; b = t; }
  if (b > c) { t = b; b = c; c = t; }
  if (a > b) { t = a; a = b; b = t; }
  return (uint32_t)a | ((uint32_t)b << 8) | ((uint32_t)c << 16);
}

// Collection of the points within reach2 of x into W.key (unsorted; W.total counts them all).
// Grid: the chart ball of the reach over the sorted shell sites (as k_nearest_exact walks it).
template <class Star>
__device__ __forceinline__ void cover_collect_grid(const CoverArgs& A, const double4* ops, Star& W, uint32_t i,
                                                   double4 x, double reach2) {
  const NearGrid g = *A.grid;
  const int lane = threadIdx.x & 31;
  const double kappa = 1.0 - 0.5 * reach2;
  const double den = 1.0 / (x.x + kappa);
  const double cen[3] = {x.y * den, x.z * den, x.w * den};
  const double rho = sqrt(fmax(0.0, 1.0 - kappa * kappa)) * den * 1.001 + 1e-6;
  int lo[3], hi[3];
  for (int a = 0; a < 3; ++a) {
    lo[a] = cell_axis((float)(cen[a] - rho), g.lower[a], g.cells_per_unit, g.sdim);
    hi[a] = cell_axis((float)(cen[a] + rho), g.lower[a], g.cells_per_unit, g.sdim);
  }
  const int ny = hi[1] - lo[1] + 1, rows = ny * (hi[2] - lo[2] + 1);
  for (int r = lane; r < rows; r += 32) {
    const int row = g.sdim * (lo[1] + r % ny + g.sdim * (lo[2] + r / ny));
    const uint32_t end = A.cell_off[row + hi[0] + 1];
    for (uint32_t t = A.cell_off[row + lo[0]]; t < end; ++t) {
      const uint32_t code = A.scode[t];
      if (code == (i | kIdentityBit)) continue;  // x itself
      const uint32_t key = ((code & ~kIdentityBit) << 8) | A.simg[t];
      const double4 d = sub4d(cover_point(A.q, ops, key), x);
      const double c2 = dot4(d, d);
      if (c2 <= reach2 && c2 > 1e-24) {
        const int slot = atomicAdd(&W.total, 1);
        if (slot < Star::kPoints) W.key[slot] = key;
      }
    }
  }
}

// Dense: every image of every source, screened in float32 (dot of q_j with x g_k^-1, within
// 4e-6 of the reach's cosine; the float32 error is below 1e-6), then tested in FP64.
template <class Star>
__device__ __forceinline__ void cover_collect_dense(const CoverArgs& A, const double4* ops, int order, Star& W,
                                                    uint32_t i, double4 x, double reach2) {
  const int lane = threadIdx.x & 31;
  const float lim = (float)(1.0 - 0.5 * reach2) - 4e-6f;
  for (int j = lane; j < A.n; j += 32) {
    const float4 p = A.q[j];
    const float inv = rsqrtf(fmaf(p.x, p.x, fmaf(p.y, p.y, fmaf(p.z, p.z, p.w * p.w))));
    for (int k = 0; k < order; ++k) {
      const float4 t = W.image_dot[k];
      const float dot = inv * fmaf(p.x, t.x, fmaf(p.y, t.y, fmaf(p.z, t.z, p.w * t.w)));
      for (int sign = 0; sign < 2; ++sign) {  // the image, then its antipode (both for reaches past pi/2)
        if ((sign ? -dot : dot) < lim) continue;
        const uint32_t key = ((uint32_t)j << 8) | (uint32_t)(2 * k + sign);
        if (key == (i << 8)) continue;  // x itself
        const double4 d = sub4d(cover_point(A.q, ops, key), x);
        const double c2 = dot4(d, d);
        if (c2 <= reach2 && c2 > 1e-24) {
          const int slot = atomicAdd(&W.total, 1);
          if (slot < Star::kPoints) W.key[slot] = key;
        }
      }
    }
  }
}

// NB, NF: the star's capacity (neighbours, facets). A star narrower than the wide one
// (NB < kCoverMax) that cannot hold a source's points or facets reports it short at the
// reach it was asked for, so the next width runs it again at that reach.
template <int NB, int NF>
__global__ void __launch_bounds__(kCoverWarps * 32) k_cover_star(const CoverArgs A) {
  using Star = CoverStar<NB, NF>;
  constexpr bool kNarrow = NB < kCoverMax;
  extern __shared__ __align__(16) unsigned char cover_smem[];
  __shared__ double4 ops[kMaxGroupOrder];
  const int off = c_group_offset[A.gid], order = c_group_order[A.gid];
  for (int k = threadIdx.x; k < order; k += blockDim.x) ops[k] = c_ops32[off + k];
  __syncthreads();
  Star& W = reinterpret_cast<Star*>(cover_smem)[threadIdx.x >> 5];
  const unsigned full = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int count_src = A.list ? A.count : A.n;
  const int stride = (gridDim.x * blockDim.x) >> 5;
  unsigned long long probes = 0;
  for (int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < count_src; w += stride) {
    const uint32_t i = A.list ? A.list[w] : (uint32_t)w;
    const double4 x = normalize4(to_d4(A.q[i]));
    double reach2 = A.reach2_of ? A.reach2_of[i] : A.reach2;
    if (A.grid) reach2 = fmin(reach2, A.grid_reach2);
    reach2 = fmin(reach2, 4.0);
    const double asked2 = reach2;
    if (!A.grid) {
      // x g_k^-1 / |g_k|: (q_j g_k) . x = q_j . (x conj(g_k)) for the float32 operator g_k.
      for (int k = lane; k < order; k += 32) {
        const double4 gk = ops[k];
        const double inv = 1.0 / dot4(gk, gk);
        const double4 t = qmul(x, make_double4(gk.x * inv, -gk.y * inv, -gk.z * inv, -gk.w * inv));
        W.image_dot[k] = to_f4(scale4(t, sqrt(dot4(gk, gk))));
      }
    }
    // 1. Collect; a reach that holds too many points shrinks (volume ~ chord^3).
    int count = 0;
    for (int attempt = 0; attempt < 8; ++attempt) {
      if (lane == 0) W.total = 0;
      __syncwarp();
      if (A.grid) cover_collect_grid(A, ops, W, i, x, reach2);
      else cover_collect_dense(A, ops, order, W, i, x, reach2);
      __syncwarp();
      const int total = W.total;
      if (total <= NB) {
        count = total;
        break;
      }
      reach2 *= pow(0.8 * NB / (double)total, 2.0 / 3.0);
      __syncwarp();
    }
    uint32_t status = kCoverOk;
    double alpha = 0.0;
    double4 centre = x;
    int faces = 0, nfacets = 0;
    if (count < 4) status = count == 0 && W.total > NB ? kCoverCrowded : kCoverSparse;
    if (status == kCoverOk) {
      // Canonical order: each key's rank among the collected keys (keys are distinct).
      uint32_t mine[NB / 32];
      int rank[NB / 32];
      for (int u = 0; u < NB / 32; ++u) {
        const int e = lane + 32 * u;
        mine[u] = e < count ? W.key[e] : 0xffffffffu;
        rank[u] = 0;
      }
      for (int e2 = 0; e2 < count; ++e2) {
        const uint32_t k2 = W.key[e2];
        for (int u = 0; u < NB / 32; ++u) rank[u] += k2 < mine[u];
      }
      __syncwarp();
      for (int u = 0; u < NB / 32; ++u)
        if (lane + 32 * u < count) {
          W.d[rank[u]] = sub4d(cover_point(A.q, ops, mine[u]), x);
          if (A.mesh) W.key[rank[u]] = mine[u];  // every lane has read the keys (the sync above)
        }
      if (lane < NB / 32) W.used[lane] = 0u;
      __syncwarp();
      // 2. A first facet: from the tangent hyperplane (n = x) pivot towards the nearest
      // point, then about it, then about both.
      double near = 1e300;
      int nn = -1;
      for (int m = lane; m < count; m += 32) {
        const double c2 = dot4(W.d[m], W.d[m]);
        if (c2 < near) {
          near = c2;
          nn = m;
        }
      }
      for (int o = 16; o; o >>= 1) {
        const double on = __shfl_xor_sync(full, near, o);
        const int oi = __shfl_xor_sync(full, nn, o);
        if (on < near || (on == near && oi < nn)) {
          near = on;
          nn = oi;
        }
      }
      double4 n = x;
      double4 v = unit4(axpy4(-dot4(x, W.d[nn]), x, W.d[nn]));
      double r = 0.0;
      const int a = cover_pivot(W, count, n, v, -1, -1, -1, r);
      int b = -1, c = -1;
      if (a >= 0) {
        n = cover_turn(n, v, r);
        const double4 da = W.d[a];
        const double4 ua = unit4(axpy4(-dot4(n, da), n, da));
        // Any direction orthogonal to n and d_a: the first coordinate axis that leaves enough.
        for (int e = 0; e < 4; ++e) {
          const double4 ax = make_double4(e == 0, e == 1, e == 2, e == 3);
          const double4 t = axpy4(-dot4(ax, ua), ua, axpy4(-dot4(ax, n), n, ax));
          if (dot4(t, t) > 0.09) {
            v = unit4(t);
            break;
          }
        }
        b = cover_pivot(W, count, n, v, a, -1, -1, r);
      }
      if (b >= 0) {
        n = cover_turn(n, v, r);
        v = unit4(cross4(n, W.d[a], W.d[b]));
        c = cover_pivot(W, count, n, v, a, b, -1, r);
      }
      if (c < 0) status = kCoverSparse;
      int head = 0, tail = 0;
      if (status == kCoverOk) {
        if (lane == 0) {
          W.facet[0] = facet_key(a, b, c);
          W.normal[0] = cover_turn(n, v, r);
        }
        tail = 1;
        __syncwarp();
      }
      // 3. Breadth-first over the star; the facet list is also the queue.
      while (status == kCoverOk && head < tail) {
        const uint32_t f = W.facet[head];
        const double4 fn = W.normal[head++];
        const double h = dot4(fn, x);
        if (!(h > 0.0)) {
          status = kCoverSparse;  // a cap as wide as a hemisphere: the reach is far too short
          break;
        }
        // The facet must support every collected point (n . d <= 0, up to rounding); one that
        // does not means rounding broke the star.
        double worst = -1e300;
        for (int m = lane; m < count; m += 32) worst = fmax(worst, dot4(fn, W.d[m]));
        for (int o = 16; o; o >>= 1) worst = fmax(worst, __shfl_xor_sync(full, worst, o));
        if (worst > 1e-12) {
          status = kCoverSparse;
          break;
        }
        const double cap = acos(fmin(1.0, h));
        if (cap > alpha) {
          alpha = cap;
          centre = fn;
        }
        const int vtx[3] = {(int)(f & 0xffu), (int)((f >> 8) & 0xffu), (int)((f >> 16) & 0xffu)};
        if (lane < 3) atomicOr(&W.used[vtx[lane] >> 5], 1u << (vtx[lane] & 31));
        for (int drop = 0; drop < 3 && status == kCoverOk; ++drop) {
          const int o = vtx[drop], p = vtx[(drop + 1) % 3], qv = vtx[(drop + 2) % 3];
          double4 pv = unit4(cross4(fn, W.d[p], W.d[qv]));
          if (dot4(pv, W.d[o]) > 0.0) pv = neg4(pv);
          const int m = cover_pivot(W, count, fn, pv, p, qv, o, r);
          ++probes;
          if (m < 0) {
            status = kCoverSparse;
            break;
          }
          const uint32_t key = facet_key(p, qv, m);
          bool seen = false;
          for (int t = lane; t < tail; t += 32) seen |= W.facet[t] == key;
          seen = __any_sync(full, seen);
          if (!seen) {
            if (tail == NF) {
              status = kCoverStarFull;
              break;
            }
            if (lane == 0) {
              W.facet[tail] = key;
              W.normal[tail] = cover_turn(fn, pv, r);
            }
            ++tail;
            __syncwarp();
          }
        }
      }
      nfacets = tail;
      __syncwarp();
      // Export (zo_mesh): each facet as the tetrahedron (x, y_a, y_b, y_c) of point keys, in
      // the slots the host set aside for this source (its facet count from the covering pass).
      if (A.mesh && status == kCoverOk) {
        const uint32_t first = A.mesh_offset[i], room = A.mesh_offset[i + 1] - first;
        for (int t = lane; t < tail && t < (int)room; t += 32) {
          const uint32_t f = W.facet[t];
          A.mesh[first + t] = make_uint4(i << 8, W.key[f & 0xffu], W.key[(f >> 8) & 0xffu], W.key[(f >> 16) & 0xffu]);
          if (A.mesh_normal) A.mesh_normal[first + t] = W.normal[t];
        }
      }
      if (lane < NB / 32) faces = __popc(W.used[lane]);
      for (int o = 16; o; o >>= 1) faces += __shfl_xor_sync(full, faces, o);
      faces = __shfl_sync(full, faces, 0);
    }
    // Certificate: every cap of the star lies within 2 alpha of x.
    double need2 = 0.0;
    if (status == kCoverOk) {
      const double reach = 2.0 * asin(fmin(1.0, 0.5 * sqrt(reach2)));
      if (2.0 * alpha > reach * (1.0 - 1e-12)) {
        status = kCoverShort;
        const double want = fmin(kPi, 2.0 * alpha * 1.0001 + 1e-9);
        need2 = 4.0 * sin(0.5 * want) * sin(0.5 * want);
      }
    } else if (status == kCoverSparse) {
      need2 = fmin(4.0, 4.0 * reach2);  // too few points or no closed star: twice the reach
    }
    if (kNarrow && status != kCoverOk &&
        (status == kCoverCrowded || status == kCoverStarFull || reach2 < asked2)) {
      status = kCoverShort;  // to the wide star, at least at the reach this one was asked for
      need2 = fmax(need2, asked2);
    }
    if (lane == 0) {
      A.alpha[i] = alpha;
      A.centre[i] = centre;
      A.faces[i] = (uint32_t)faces;
      A.facets[i] = (uint32_t)nfacets;
      A.status[i] = status;
      A.need2[i] = need2;
    }
    __syncwarp();
  }
  if (lane == 0 && A.probes) atomicAdd(A.probes, probes);
}

}  // namespace zo
