// CPU restatement of the reference crate's geometry, used ONLY as a test oracle.
//
// This file is test infrastructure.  Nothing in the shipped library includes it;
// only tests/, bench.py's CPU-baseline leg and __graft_entry__.smoke() reach it
// (through liboracle's C ABI).
//
// Every function restates a function of the Rust crate `mesh_to_sdf` with the
// same f32 operation order.  Rust never contracts a*b+c into an FMA, so this file
// must be compiled with -ffp-contract=off and without -ffast-math (the Makefile
// beside it does so); x86-64 SSE arithmetic then rounds every step to f32 exactly
// as the reference does.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

namespace m2s_oracle {

struct V3 {
  float x, y, z;
};

// Default `Point` arithmetic (mesh_to_sdf/src/point.rs:80-153): component-wise,
// left to right, no FMA.
static inline V3 v_add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline V3 v_sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
// point.rs:100-102 — (x*x' + y*y') + z*z'
static inline float v_dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// point.rs:105-111
static inline V3 v_cross(V3 a, V3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// point.rs:131-133
static inline V3 v_fmul(V3 a, float s) { return {a.x * s, a.y * s, a.z * s}; }
// point.rs:119-127
static inline float v_dist2(V3 a, V3 b) {
  V3 d = v_sub(a, b);
  return v_dot(d, d);
}
static inline float v_dist(V3 a, V3 b) { return std::sqrt(v_dist2(a, b)); }
// PartialEq of [f32; 3]: element-wise IEEE equality.
static inline bool v_eq(V3 a, V3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
static inline float v_get(V3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

// Rust f32::clamp (returns NaN for a NaN input; no min/max NaN-dropping).
static inline float rs_clamp(float v, float lo, float hi) {
  if (v < lo) v = lo;
  if (v > hi) v = hi;
  return v;
}
// Rust f32::min / f32::max: IEEE minNum/maxNum (a NaN operand is ignored).
static inline float rs_min(float a, float b) {
  if (std::isnan(a)) return b;
  if (std::isnan(b)) return a;
  return a < b ? a : b;
}
static inline float rs_max(float a, float b) {
  if (std::isnan(a)) return b;
  if (std::isnan(b)) return a;
  return a > b ? a : b;
}

// geo.rs:4-22 — triangle AABB padded by 1e-4 on every side.
static inline void triangle_bounding_box(V3 a, V3 b, V3 c, V3* mn, V3* mx) {
  const float eps = 0.0001f;
  V3 lo = {rs_min(a.x, rs_min(b.x, c.x)), rs_min(a.y, rs_min(b.y, c.y)),
           rs_min(a.z, rs_min(b.z, c.z))};
  V3 hi = {rs_max(a.x, rs_max(b.x, c.x)), rs_max(a.y, rs_max(b.y, c.y)),
           rs_max(a.z, rs_max(b.z, c.z))};
  V3 e = {eps, eps, eps};
  *mn = v_sub(lo, e);
  *mx = v_add(hi, e);
}

// geo.rs:141-151 — projection of p on the segment [a, b].
static inline V3 closest_point_segment(V3 p, V3 a, V3 b) {
  V3 ab = v_sub(b, a);
  float m = v_dot(ab, ab);
  V3 ap = v_sub(p, a);
  float s = v_dot(ab, ap) / m;
  s = rs_clamp(s, 0.0f, 1.0f);
  return v_add(a, v_fmul(ab, s));
}

// geo.rs:70-138 — Voronoi-region closest point (Embree formulation), with the
// degenerate-triangle fallbacks of geo.rs:73-88.
static inline V3 closest_point_triangle(V3 p, V3 a, V3 b, V3 c) {
  bool ab_eq = v_eq(a, b), bc_eq = v_eq(b, c), ac_eq = v_eq(a, c);
  if (ab_eq && bc_eq && ac_eq) return a;
  if (ab_eq) return closest_point_segment(p, a, c);
  if (bc_eq) return closest_point_segment(p, a, b);
  if (ac_eq) return closest_point_segment(p, a, b);

  V3 ab = v_sub(b, a);
  V3 ac = v_sub(c, a);
  V3 ap = v_sub(p, a);
  float d1 = v_dot(ab, ap);
  float d2 = v_dot(ac, ap);
  if (d1 <= 0.0f && d2 <= 0.0f) return a;

  V3 bp = v_sub(p, b);
  float d3 = v_dot(ab, bp);
  float d4 = v_dot(ac, bp);
  if (d3 >= 0.0f && d4 <= d3) return b;

  V3 cp = v_sub(p, c);
  float d5 = v_dot(ab, cp);
  float d6 = v_dot(ac, cp);
  if (d6 >= 0.0f && d5 <= d6) return c;

  float vc = d1 * d4 - d3 * d2;
  if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
    float v = d1 / (d1 - d3);
    return v_add(a, v_fmul(ab, v));
  }

  float vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
    float v = d2 / (d2 - d6);
    return v_add(a, v_fmul(ac, v));
  }

  float va = d3 * d6 - d5 * d4;
  if (va <= 0.0f && d4 - d3 >= 0.0f && d5 - d6 >= 0.0f) {
    float v = (d4 - d3) / ((d4 - d3) + (d5 - d6));
    V3 bc = v_sub(c, b);
    return v_add(b, v_fmul(bc, v));
  }

  float denom = 1.0f / (va + vb + vc);
  float v = vb * denom;
  float w = vc * denom;
  return v_add(v_add(a, v_fmul(ab, v)), v_fmul(ac, w));
}

// geo.rs:26-30
static inline float point_triangle_distance(V3 p, V3 a, V3 b, V3 c) {
  return v_dist(p, closest_point_triangle(p, a, b, c));
}
// geo.rs:33-37
static inline float point_triangle_distance2(V3 p, V3 a, V3 b, V3 c) {
  return v_dist2(p, closest_point_triangle(p, a, b, c));
}
// geo.rs:43-56 and geo.rs:60-64 — sign of (p - closest) . (ab x ac); zero counts
// as inside (negative), so a zero distance comes back as -0.0.
static inline float point_triangle_signed_distance(V3 p, V3 a, V3 b, V3 c) {
  V3 nearest = closest_point_triangle(p, a, b, c);
  V3 dir = v_sub(p, nearest);
  V3 n = v_cross(v_sub(b, a), v_sub(c, a));
  float d = v_dist(p, nearest);
  return v_dot(dir, n) > 0.0f ? d : -d;
}

// geo.rs:165-216 — ray from `o` along +axis (0 = X, 1 = Y, 2 = Z).  The (y, z)
// projection plane rotates with the axis exactly as the reference's get_y/get_z.
// Returns true and writes t on a hit with t > 0.
static inline bool ray_triangle_intersection_aligned(V3 o, V3 t0, V3 t1, V3 t2, int axis,
                                                     float* t_out) {
  V3 e01 = v_sub(t1, t0);
  V3 e12 = v_sub(t2, t1);
  V3 e20 = v_sub(t0, t2);
  V3 p0 = v_sub(o, t0);
  V3 p1 = v_sub(o, t1);
  V3 p2 = v_sub(o, t2);
  const int ix = axis, iy = (axis + 1) % 3, iz = (axis + 2) % 3;
  float w0 = v_get(p1, iz) * v_get(e12, iy) - v_get(p1, iy) * v_get(e12, iz);
  float w1 = v_get(p2, iz) * v_get(e20, iy) - v_get(p2, iy) * v_get(e20, iz);
  float w2 = v_get(p0, iz) * v_get(e01, iy) - v_get(p0, iy) * v_get(e01, iz);
  if ((w0 < 0.0f && w1 < 0.0f && w2 < 0.0f) || (w0 > 0.0f && w1 > 0.0f && w2 > 0.0f)) {
    float t = -(w0 * v_get(p0, ix) + w2 * v_get(p2, ix) + w1 * v_get(p1, ix)) / (w0 + w1 + w2);
    if (t > 0.0f) {
      if (t_out) *t_out = t;
      return true;
    }
  }
  return false;
}

// float-cmp 0.9 `approx_eq!(f32, a, b, ulps = 2, epsilon = 1e-6)`, restated from
// its documented meaning: equal, or |a - b| <= epsilon, or the distance between
// the two bit patterns read as i32 (wrapping subtraction, saturating abs) <= ulps.
static inline bool approx_eq_ulps2_eps1e6(float a, float b) {
  if (a == b) return true;
  if (std::fabs(a - b) <= 1e-6f) return true;
  int32_t ai, bi;
  std::memcpy(&ai, &a, 4);
  std::memcpy(&bi, &b, 4);
  int32_t diff = (int32_t)((uint32_t)ai - (uint32_t)bi);
  int32_t ad = diff == INT32_MIN ? INT32_MAX : (diff < 0 ? -diff : diff);
  return ad <= 2;
}

// lib.rs:315-332 — returns -1 (Less), 0 (Equal) or 1 (Greater).  Sets *nan when
// the reference would panic on a NaN distance.
static inline int compare_distances(float a, float b, bool* nan) {
  float A = std::fabs(a), B = std::fabs(b);
  if (approx_eq_ulps2_eps1e6(A, B)) {
    bool an = std::signbit(a), bn = std::signbit(b);
    if (an && !bn) return 1;
    if (!an && bn) return -1;
  }
  if (A < B) return -1;
  if (A > B) return 1;
  if (A == B) return 0;
  if (nan) *nan = true;
  return 0;
}

}  // namespace m2s_oracle
