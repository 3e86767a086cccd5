// Device-side arithmetic of the QVM repulsion path: quaternion helpers, the Quey pair in
// FP32 (fast, hot loops) and FP64 (exact, plain method), the near-field window, and the
// fundamental-zone fold. Quaternions are scalar first and live in float4/double4 as
// (.x=w, .y=x, .z=y, .w=z); symmetry acts on the right (q*g).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "qvm_shared.h"

namespace zo {

constexpr float kPiF = 3.14159265358979323846f;
constexpr double kPi = 3.14159265358979323846;

// Operator tables of all eleven groups (rows kGroupOffset[g] .. +kGroupOrder[g]):
// c_ops64 the FP64 table, c_ops32 the float32 rounding the reference uploads (as double).
// Zone bisector planes (2|K|-1 per group, src/covering.zig:382-396): float32 rounding of the
// planes built from the f32 table (FP32 mode) and FP64 planes of the f64 table (FP64 mode).
// Defined here: every kernel is compiled in the one translation unit kernels.cu.
__constant__ double4 c_ops64[kMaxOperatorRows];
__constant__ double4 c_ops32[kMaxOperatorRows];
__constant__ float4 c_planes32[kMaxPlaneRows];
__constant__ double4 c_planes64[kMaxPlaneRows];
__constant__ int c_group_offset[11];
__constant__ int c_group_order[11];
__constant__ int c_plane_offset[11];
// Each group's planes sorted by reach (the least dot product of the plane with any zone
// point, less a margin for rounding): the group-local index of each sorted row and its
// reach. A source in the zone can be within `margin` of a plane only if its reach <= margin.
__constant__ uint8_t c_plane_order[kMaxPlaneRows];
__constant__ float c_plane_reach[kMaxPlaneRows];

// ------------------------------------------------------------------ quaternion helpers
__device__ __forceinline__ double4 qmul(double4 a, double4 b) {
  return make_double4(a.x * b.x - a.y * b.y - a.z * b.z - a.w * b.w,
                      a.x * b.y + a.y * b.x + a.z * b.w - a.w * b.z,
                      a.x * b.z - a.y * b.w + a.z * b.x + a.w * b.y,
                      a.x * b.w + a.y * b.z - a.z * b.y + a.w * b.x);
}
__device__ __forceinline__ double dot4(double4 a, double4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
__device__ __forceinline__ double4 scale4(double4 a, double s) { return make_double4(a.x * s, a.y * s, a.z * s, a.w * s); }
__device__ __forceinline__ double4 neg4(double4 a) { return make_double4(-a.x, -a.y, -a.z, -a.w); }
__device__ __forceinline__ double4 normalize4(double4 a) { return scale4(a, 1.0 / sqrt(dot4(a, a))); }
__device__ __forceinline__ double4 to_d4(float4 a) { return make_double4(a.x, a.y, a.z, a.w); }
__device__ __forceinline__ float4 to_f4(double4 a) {
  return make_float4((float)a.x, (float)a.y, (float)a.z, (float)a.w);
}

// Image y = q g_k of a source (shaders/pairs.wgsl:181): the identity image is the source
// itself bit for bit; the others are normalised. FP32 mode forms the product and the
// normalisation in FP64 and rounds once (the correctly rounded image).
__device__ __forceinline__ float4 image32(float4 q, int op_row, bool identity) {
  if (identity) return q;
  return to_f4(normalize4(qmul(to_d4(q), c_ops32[op_row])));
}
__device__ __forceinline__ double4 image64(double4 q, int op_row, bool identity) {
  if (identity) return q;
  return normalize4(qmul(q, c_ops64[op_row]));
}

// ------------------------------------------------------------------ approximate SFU ops
// PTX rcp.approx / sqrt.approx: the documented MUFU approximations (max error ~1 ulp).
__device__ __forceinline__ float rcp_approx(float x) {
  float r;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}
__device__ __forceinline__ float sqrt_approx(float x) {
  float r;
  asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

// 2 atan(t) for t in [0,1]: t * P(t^2), P the degree-8 minimax fit of fit_atan.py (max
// relative error 1.5e-8 with exact coefficients, 6.4e-8 - about one float ulp - with these
// float32 ones), doubled.
__device__ __forceinline__ float two_atan_unit(float t, float t2) {
  float p = 0x1.758a10p-8f;
  p = fmaf(p, t2, -0x1.07448cp-5f);
  p = fmaf(p, t2, 0x1.5dba7cp-4f);
  p = fmaf(p, t2, -0x1.336030p-3f);
  p = fmaf(p, t2, 0x1.b3da44p-3f);
  p = fmaf(p, t2, -0x1.22e400p-2f);
  p = fmaf(p, t2, 0x1.9972e8p-2f);
  p = fmaf(p, t2, -0x1.5554a6p-1f);
  p = fmaf(p, t2, 2.0f);
  return t * p;
}

// 2 atan(t) for t in [0, 0.21] (near-field cutoffs r <= 0.4 rad, t = tan(a/2) <= tan 0.2):
// degree-3 minimax fit in t^2 from fit_atan.py, max relative error 3.0e-9 (6.0e-9 with these
// float32 coefficients).
__device__ __forceinline__ float two_atan_short(float t, float t2) {
  float p = -0x1.117a86p-2f;
  p = fmaf(p, t2, 0x1.991528p-2f);
  p = fmaf(p, t2, -0x1.5554c2p-1f);
  p = fmaf(p, t2, 2.0f);
  return t * p;
}

// Vector part of y * conj(x): the left-tangent direction of a pair (shaders/pairs.wgsl:258).
template <class T, class V>
__device__ __forceinline__ void pair_direction(const V& x, const V& y, T& d1, T& d2, T& d3) {
  d1 = x.x * y.y - y.x * x.y + (x.z * y.w - x.w * y.z);
  d2 = x.x * y.z - y.x * x.z + (x.w * y.y - x.y * y.w);
  d3 = x.x * y.w - y.x * x.w + (x.y * y.z - x.z * y.y);
}

// One Quey pair (shaders/pairs.wgsl:250-262), FP32. With a = 2 atan(sqrt(near/far)) the
// nearer S3 angle and b = pi - a:
//   force = -sign (1/(a^2+e) - 1/(b^2+e)) / (sin a + e) * dir,  curvature = 1/(a^3+e) + 1/(b^3+e),
//   energy = 1/a + 1/b = pi/(ab),  e = 1e-9,  sin a = 2t/(1+t^2).
// The four divisions share two approximate reciprocals; `coef` multiplies the direction.
struct PairF {
  float coef, curv, energy, a, inv_sine;
};
__device__ __forceinline__ PairF quey_pair32(float dm2, float dp2) {
  const float nearv = fmaxf(fminf(dm2, dp2), 1e-30f);
  const float farv = fmaxf(fmaxf(dm2, dp2), 1e-30f);
  const float t2 = nearv * rcp_approx(farv);
  const float t = sqrt_approx(t2);
  const float a = fmaxf(two_atan_unit(t, t2), 1e-12f);
  const float b = kPiF - a;
  const float aa = a * a, bb = b * b;
  const float a2 = aa + 1e-9f, b2 = bb + 1e-9f;
  const float a3 = fmaf(aa, a, 1e-9f), b3 = fmaf(bb, b, 1e-9f);
  const float onept2 = 1.0f + t2;
  const float sp = fmaf(1e-9f, onept2, t + t);  // (sine + 1e-9) * (1 + t^2)
  const float a2b2 = a2 * b2;
  const float r1 = rcp_approx(a2b2 * sp);
  const float along = (b2 - a2) * onept2 * r1;
  const float ab = a * b;
  const float a3b3 = a3 * b3;
  const float r2 = rcp_approx(a3b3 * ab);
  PairF p;
  p.coef = (dm2 <= dp2) ? -along : along;
  p.curv = (a3 + b3) * ab * r2;
  p.energy = kPiF * a3b3 * r2;
  p.a = a;
  p.inv_sine = onept2 * a2b2 * r1;
  return p;
}

// ------------------------------------------------------------------ asynchronous copies
// cp.async: a 16-byte global-to-shared copy that bypasses the registers (cached in L2
// only), committed as a group and awaited with wait_group; both addresses 16-byte aligned.
__device__ __forceinline__ void copy_async16(void* shared, const void* global) {
  const unsigned to = (unsigned)__cvta_generic_to_shared(shared);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(to), "l"(global) : "memory");
}
__device__ __forceinline__ void copy_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// Waits until at most `pending` of this thread's committed groups are still in flight.
template <int pending>
__device__ __forceinline__ void copy_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(pending) : "memory");
}

// ------------------------------------------------------------------ packed FP32 (two pairs)
// sm_100 f32x2 arithmetic: one instruction does the same add, multiply or fused
// multiply-add on two lanes of a float2, each rounded exactly as its scalar counterpart.
// The hot loops evaluate two pairs per thread this way, halving their issue slots.
__device__ __forceinline__ float2 splat(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 rcp2(float2 a) { return make_float2(rcp_approx(a.x), rcp_approx(a.y)); }
__device__ __forceinline__ float2 sqrt2(float2 a) { return make_float2(sqrt_approx(a.x), sqrt_approx(a.y)); }
__device__ __forceinline__ float2 max2(float2 a, float b) { return make_float2(fmaxf(a.x, b), fmaxf(a.y, b)); }

__device__ __forceinline__ float2 two_atan_unit2(float2 t, float2 t2) {
  float2 p = splat(0x1.758a10p-8f);
  p = fma2(p, t2, splat(-0x1.07448cp-5f));
  p = fma2(p, t2, splat(0x1.5dba7cp-4f));
  p = fma2(p, t2, splat(-0x1.336030p-3f));
  p = fma2(p, t2, splat(0x1.b3da44p-3f));
  p = fma2(p, t2, splat(-0x1.22e400p-2f));
  p = fma2(p, t2, splat(0x1.9972e8p-2f));
  p = fma2(p, t2, splat(-0x1.5554a6p-1f));
  p = fma2(p, t2, splat(2.0f));
  return mul2(t, p);
}
__device__ __forceinline__ float2 two_atan_short2(float2 t, float2 t2) {
  float2 p = splat(-0x1.117a86p-2f);
  p = fma2(p, t2, splat(0x1.991528p-2f));
  p = fma2(p, t2, splat(-0x1.5554c2p-1f));
  p = fma2(p, t2, splat(2.0f));
  return mul2(t, p);
}

// Two Quey pairs given near = |x - y~|^2 (clamped to >= 1e-30) and far = |x + y~|^2 of
// each, y~ the near twin: the coefficient of (x - y~) in the force sum (minus the force
// magnitude over sin a; sign included), the curvature 1/a3 + 1/b3 = cs * cr and the energy
// pi / (a b) = pi * rab, left as factors so the caller accumulates each with one FMA (and
// multiplies the energy sum by pi once). The arithmetic of quey_pair32 lane by lane.
struct QueyPair2 {
  float2 coef, cs, cr, rab;
};
__device__ __forceinline__ QueyPair2 quey_pair32x2(float2 nearv, float2 farv) {
  const float2 t2 = mul2(nearv, rcp2(farv));
  const float2 t = sqrt2(t2);
  const float2 a = max2(two_atan_unit2(t, t2), 1e-12f);
  const float2 b = fma2(a, splat(-1.0f), splat(kPiF));
  const float2 aa = mul2(a, a), bb = mul2(b, b);
  // b >= pi/2 (a is the near twin's angle), so b^2 + 1e-9 rounds to b^2: b2 = bb.
  const float2 a2 = add2(aa, splat(1e-9f));
  const float2 a3 = fma2(aa, a, splat(1e-9f)), b3 = fma2(bb, b, splat(1e-9f));
  const float2 onept2 = add2(t2, splat(1.0f));
  const float2 sp = fma2(splat(1e-9f), onept2, add2(t, t));  // (sine + 1e-9) (1 + t^2)
  const float2 r1 = rcp2(mul2(mul2(a2, bb), sp));
  QueyPair2 p;
  p.coef = mul2(mul2(fma2(bb, splat(-1.0f), a2), onept2), r1);  // -(b2 - a2)(1 + t^2) / (a2 b2 sp)
  p.cs = add2(a3, b3);
  p.cr = rcp2(mul2(a3, b3));
  p.rab = rcp2(mul2(a, b));
  return p;
}

// The terms of two windowed near-field pairs, left as factors for FMA accumulation: the
// coefficient of (x - y~), the curvature q w and the energy pi (rab w), with the window w.
struct NearPair2 {
  float2 coef, q, w, rab;
};

// near_pair32 (below) on two sites at once: dm2 and dp2 of each, the window's start cz and
// inverse width cw, czw = cz * cw and pk = -6 pi cw (the window's slope factor times pi).
// Regrouped as coefficient = (1 + t^2) [w (a2 - b2) + pi slope a2 b2 / (a b)] / (a2 b2 sp).
// Beyond the cutoff the window is exactly zero, so such a site contributes nothing.
template <bool SHORT>
__device__ __forceinline__ NearPair2 near_pair32x2(float2 dm2, float2 dp2, float cw, float czw, float pk) {
  const float2 t2 = mul2(max2(dm2, 1e-30f), rcp2(dp2));
  const float2 t = sqrt2(t2);
  const float2 a = max2(SHORT ? two_atan_short2(t, t2) : two_atan_unit2(t, t2), 1e-12f);
  const float2 b = fma2(a, splat(-1.0f), splat(kPiF));
  const float2 aa = mul2(a, a), bb = mul2(b, b);
  // b >= pi/2 (the site is the near twin), so b^2 + 1e-9 rounds to b^2: b2 = bb.
  const float2 a2 = add2(aa, splat(1e-9f));
  const float2 a3 = fma2(aa, a, splat(1e-9f)), b3 = fma2(bb, b, splat(1e-9f));
  const float2 onept2 = add2(t2, splat(1.0f));
  const float2 sp = fma2(splat(1e-9f), onept2, add2(t, t));
  const float2 a2b2 = mul2(a2, bb);
  const float2 r1 = rcp2(mul2(a2b2, sp));
  NearPair2 p;
  p.rab = rcp2(mul2(a, b));
  const float2 sr = fma2(a, splat(cw), splat(-czw));
  const float2 s = make_float2(__saturatef(sr.x), __saturatef(sr.y));
  const float2 ss = mul2(s, s);
  p.w = fma2(ss, fma2(s, splat(2.0f), splat(-3.0f)), splat(1.0f));  // 1 - s^2 (3 - 2s)
  const float2 slope = fma2(ss, splat(-pk), mul2(s, splat(pk)));   // pi * (-6 cw) s (1 - s)
  const float2 g = mul2(mul2(p.rab, slope), a2b2);
  p.coef = mul2(fma2(p.w, fma2(bb, splat(-1.0f), a2), g), mul2(onept2, r1));
  p.q = mul2(add2(a3, b3), rcp2(mul2(a3, b3)));
  return p;
}

// near_pair32x2 from the squared chords d alone, for cutoffs r <= 0.4 rad (d <= 0.25 after
// the clamp at 1.25 r). For unit quaternions the angle a = 2 atan(sqrt(near/far)) of
// quey_pair is also 2 asin(c/2), c = sqrt(d) the chord, and sin a = c sqrt(1 - d/4):
// a = c (1 + d Pa(d)) and sin a = c (1 + d Ps(d)) with Pa, Ps the quadratic fits of
// fit_atan.py (relative error below 1e-8 on [0, 0.25]). Neither the far chord nor its
// reciprocal is needed: coefficient = [w (a2 - b2) + pi slope a2 b2 / (a b)] /
// (a2 b2 (sin a + 1e-9)).
__device__ __forceinline__ NearPair2 near_chord_pair32x2(float2 d, float cw, float czw, float pk) {
  const float2 c = sqrt2(d);
  const float2 cd = mul2(c, d);
  const float2 pa = fma2(fma2(splat(0x1.8d9f56p-11f), d, splat(0x1.329be0p-8f)), d, splat(0x1.555620p-5f));
  const float2 ps = fma2(fma2(splat(-0x1.147feap-10f), d, splat(-0x1.ff3d12p-8f)), d, splat(-0x1.000042p-3f));
  const float2 a = max2(fma2(cd, pa, c), 1e-12f);
  const float2 sn = fma2(cd, ps, add2(c, splat(1e-9f)));  // sin a + 1e-9
  const float2 b = fma2(a, splat(-1.0f), splat(kPiF));
  const float2 aa = mul2(a, a), bb = mul2(b, b);
  // b >= pi/2 (the site is the near twin), so b^2 + 1e-9 rounds to b^2: b2 = bb.
  const float2 a2 = add2(aa, splat(1e-9f));
  const float2 a3 = fma2(aa, a, splat(1e-9f)), b3 = fma2(bb, b, splat(1e-9f));
  const float2 a2b2 = mul2(a2, bb);
  const float2 r1 = rcp2(mul2(a2b2, sn));  // 1 / (a2 b2 (sin a + 1e-9))
  NearPair2 p;
  p.rab = rcp2(mul2(a, b));
  const float2 sr = fma2(a, splat(cw), splat(-czw));
  const float2 s = make_float2(__saturatef(sr.x), __saturatef(sr.y));
  const float2 ss = mul2(s, s);
  p.w = fma2(ss, fma2(s, splat(2.0f), splat(-3.0f)), splat(1.0f));  // 1 - s^2 (3 - 2s)
  const float2 slope = fma2(ss, splat(-pk), mul2(s, splat(pk)));   // pi * (-6 cw) s (1 - s)
  const float2 g = mul2(mul2(p.rab, slope), a2b2);
  p.coef = mul2(fma2(p.w, fma2(bb, splat(-1.0f), a2), g), r1);
  p.q = mul2(add2(a3, b3), rcp2(mul2(a3, b3)));
  return p;
}

// Windowed near-field pair, FP32, for a site that is the near twin (dm2 <= cut < 2 <= dp2,
// so the sign is +1, near = dm2 and far = dp2): the coefficient c of the pair's direction
// (force contribution c * dir), its windowed curvature and energy. Same arithmetic as
// quey_pair32 followed by window32. SHORT: the cutoff is at most 0.4 rad (two_atan_short).
template <bool SHORT>
__device__ __forceinline__ void near_pair32(float dm2, float dp2, float cut_z, float cut_w, float& coef, float& curv,
                                            float& energy) {
  const float t2 = fmaxf(dm2, 1e-30f) * rcp_approx(dp2);
  const float t = sqrt_approx(t2);
  const float a = fmaxf(SHORT ? two_atan_short(t, t2) : two_atan_unit(t, t2), 1e-12f);
  const float b = kPiF - a;
  const float aa = a * a, bb = b * b;
  const float a2 = aa + 1e-9f, b2 = bb + 1e-9f;
  const float a3 = fmaf(aa, a, 1e-9f), b3 = fmaf(bb, b, 1e-9f);
  const float onept2 = 1.0f + t2;
  const float sp = fmaf(1e-9f, onept2, t + t);
  const float a2b2 = a2 * b2;
  const float r1 = rcp_approx(a2b2 * sp);
  const float along = (b2 - a2) * onept2 * r1;
  const float ab = a * b;
  const float a3b3 = a3 * b3;
  const float r2 = rcp_approx(a3b3 * ab);
  const float e = kPiF * a3b3 * r2;
  const float s = __saturatef((a - cut_z) * cut_w);
  const float w = fmaf(-s * s, fmaf(-2.0f, s, 3.0f), 1.0f);
  const float slope = -6.0f * s * (1.0f - s) * cut_w;
  coef = fmaf(-w, along, e * slope * (onept2 * a2b2 * r1));
  curv = (a3 + b3) * ab * r2 * w;
  energy = e * w;
}

// The force of a source from the accumulated sum Y = sum_k c_k (x - y_k): the direction
// vec(y x^-1) is linear in y and vanishes at y = x, so sum_k c_k dir_k = -dir(Y). Summing
// the short difference vectors keeps the precision of summing the directions themselves.
__device__ __forceinline__ double3 force_from_differences(double4 x, double4 y) {
  double d1, d2, d3;
  pair_direction(x, y, d1, d2, d3);
  return make_double3(-d1, -d2, -d3);
}

// The same pair in FP64 with IEEE division, sqrt and atan: the plain method's arithmetic.
struct PairD {
  double coef, curv, energy, a;
};
__device__ __forceinline__ PairD quey_pair64(double dm2, double dp2) {
  const double nearv = fmax(fmin(dm2, dp2), 1e-30);
  const double farv = fmax(fmax(dm2, dp2), 1e-30);
  const double t = sqrt(nearv / farv);
  const double a = fmax(2.0 * atan(t), 1e-12);
  const double b = kPi - a;
  const double a2 = a * a + 1e-9, b2 = b * b + 1e-9;
  const double a3 = a * a * a + 1e-9, b3 = b * b * b + 1e-9;
  const double sine = 2.0 * t / (1.0 + t * t) + 1e-9;
  const double sign = (dm2 <= dp2) ? 1.0 : -1.0;
  const double along = sign * (b2 - a2) / (a2 * b2 * sine);
  PairD p;
  p.coef = -along;
  p.curv = (a3 + b3) / (a3 * b3);
  p.energy = kPi / (a * b);
  p.a = a;
  return p;
}

// Near-field window (shaders/pairs.wgsl:352-361): the pair potential times
// w = 1 - s^2 (3 - 2s), s = clamp((a - taper r) / ((1 - taper) r), 0, 1), and its exact force
// (the window's slope adds sign E w'(a) / sin a along the direction). `cut_z` is taper*r,
// `cut_w` 1/((1-taper) r). Evaluated branch-free: at s = 0 it is the plain pair.
__device__ __forceinline__ void window32(PairF& p, float dm2, float dp2, float cut_z, float cut_w) {
  const float s = __saturatef((p.a - cut_z) * cut_w);
  const float w = fmaf(-s * s, fmaf(-2.0f, s, 3.0f), 1.0f);
  const float slope = -6.0f * s * (1.0f - s) * cut_w;
  float extra = p.energy * slope * p.inv_sine;
  extra = (dm2 <= dp2) ? extra : -extra;
  p.coef = fmaf(w, p.coef, extra);
  p.curv *= w;
  p.energy *= w;
}
__device__ __forceinline__ void window64(PairD& p, double dm2, double dp2, double cut_z, double cut_w) {
  const double s = fmin(fmax((p.a - cut_z) * cut_w, 0.0), 1.0);
  if (s <= 0.0) return;
  const double w = 1.0 - s * s * (3.0 - 2.0 * s);
  const double slope = -6.0 * s * (1.0 - s) * cut_w;
  const double sign = (dm2 <= dp2) ? 1.0 : -1.0;
  const double extra = sign * p.energy * slope / fmax(sin(p.a), 1e-9);
  p.coef = w * p.coef + extra;
  p.curv *= w;
  p.energy *= w;
}

// ------------------------------------------------------------------ fundamental-zone fold
// Homogeneous zone inequalities (shaders/state.wgsl:6-29) on a unit quaternion with w >= 0.
__device__ __forceinline__ bool in_zone(double4 p, int gid, bool f32_ops) {
  const double ax = fabs(p.y), ay = fabs(p.z), az = fabs(p.w), w = p.x;
  const double t6 = 0.5773502691896258, t8 = 0.4142135623730951, t12 = 0.2679491924311227;
  const double c6 = 0.8660254037844386, s45 = 0.7071067811865476;
  switch (gid) {
    case 0: return az <= w;
    case 1: return az <= t6 * w;
    case 2: return az <= t8 * w;
    case 3: return az <= t12 * w;
    case 4: return fmax(fmax(ax, ay), az) <= w;
    case 5: return az <= t6 * w && fmax(ax, 0.5 * ax + c6 * ay) <= w;
    case 6: return az <= t8 * w && fmax(fmax(ax, ay), s45 * (ax + ay)) <= w;
    case 7: {
      const double m = fmax(ax, ay), n = fmin(ax, ay);
      return az <= t12 * w && fmax(m, c6 * m + 0.5 * n) <= w;
    }
    case 8: return ax + ay + az <= w;
    case 9: return fmax(fmax(ax, ay), az) <= t8 * w && ax + ay + az <= w;
    default: {
      if (w > 0.9510566) return true;
      if (w < 0.9256147) return false;
      const int off = c_group_offset[gid], order = c_group_order[gid];
      for (int k = 1; k < order; ++k) {
        const double4 g = f32_ops ? c_ops32[off + k] : c_ops64[off + k];
        if (fabs(fabs(g.x) - 0.8090169943749475) < 1e-5 && fabs(dot4(p, g)) > w) return false;
      }
      return true;
    }
  }
}

// Fold a unit quaternion into the zone (shaders/state.wgsl:30-46), FP64: w >= 0, keep it if
// in the zone, else the image p g_k of largest |w| (first maximum), sign fixed, normalised.
// `f32_ops` picks the float32 table (FP32 mode) or the FP64 one.
__device__ __forceinline__ double4 fold64(double4 p, int gid, bool f32_ops) {
  if (p.x < 0.0) p = neg4(p);
  if (in_zone(p, gid, f32_ops)) return p;
  const int off = c_group_offset[gid], order = c_group_order[gid];
  double4 best = p;
  double w = p.x;
  for (int k = 0; k < order; ++k) {
    const double4 c = qmul(p, f32_ops ? c_ops32[off + k] : c_ops64[off + k]);
    if (fabs(c.x) > w) {
      best = c.x >= 0.0 ? c : neg4(c);
      w = fabs(c.x);
    }
  }
  return normalize4(best);
}

}  // namespace zo
