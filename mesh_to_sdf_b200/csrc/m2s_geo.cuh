// Device geometry for mesh_to_sdf_b200 (sm_100a).
//
// The arithmetic follows the Rust crate `mesh_to_sdf` operation by operation:
// Rust never fuses a*b+c, so every add / sub / mul / div / sqrt here goes
// through a round-to-nearest intrinsic (__fadd_rn and friends), which the
// compiler may not contract into an FMA whatever -fmad says.  With the same
// inputs the results are therefore bit-identical to the reference's f32 code.
#pragma once

#include <cstdint>

namespace m2s {

__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fd(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ float fsqrt(float a) { return __fsqrt_rn(a); }

struct P3 {
  float x, y, z;
};

__device__ __forceinline__ P3 p3(float4 v) { return {v.x, v.y, v.z}; }
__device__ __forceinline__ P3 vsub(P3 a, P3 b) { return {fs(a.x, b.x), fs(a.y, b.y), fs(a.z, b.z)}; }
__device__ __forceinline__ P3 vadd(P3 a, P3 b) { return {fa(a.x, b.x), fa(a.y, b.y), fa(a.z, b.z)}; }
__device__ __forceinline__ P3 vmul(P3 a, float s) { return {fm(a.x, s), fm(a.y, s), fm(a.z, s)}; }
// point.rs:100-102 — (x*x' + y*y') + z*z'
__device__ __forceinline__ float vdot(P3 a, P3 b) { return fa(fa(fm(a.x, b.x), fm(a.y, b.y)), fm(a.z, b.z)); }
// point.rs:105-111
__device__ __forceinline__ P3 vcross(P3 a, P3 b) {
  return {fs(fm(a.y, b.z), fm(a.z, b.y)), fs(fm(a.z, b.x), fm(a.x, b.z)), fs(fm(a.x, b.y), fm(a.y, b.x))};
}
__device__ __forceinline__ float vget(P3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }

// Arithmetic of the closest-point and distance computations.  The default
// (strict) build rounds every operation like the reference; the fast build
// (M2S_FAST_MATH) lets the compiler fuse multiply-adds there, and only there:
// ray-triangle tests, cell centres and the Normal sign's dot product stay
// strict, so Raycast signs are the strict build's.  Division and square root
// are IEEE in both.
#ifdef M2S_FAST_MATH
__device__ __forceinline__ float da(float a, float b) { return a + b; }
__device__ __forceinline__ float ds(float a, float b) { return a - b; }
__device__ __forceinline__ float dm(float a, float b) { return a * b; }
#else
__device__ __forceinline__ float da(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float ds(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float dm(float a, float b) { return __fmul_rn(a, b); }
#endif
__device__ __forceinline__ P3 dvsub(P3 a, P3 b) { return {ds(a.x, b.x), ds(a.y, b.y), ds(a.z, b.z)}; }
__device__ __forceinline__ P3 dvadd(P3 a, P3 b) { return {da(a.x, b.x), da(a.y, b.y), da(a.z, b.z)}; }
__device__ __forceinline__ P3 dvmul(P3 a, float s) { return {dm(a.x, s), dm(a.y, s), dm(a.z, s)}; }
__device__ __forceinline__ float dvdot(P3 a, P3 b) { return da(da(dm(a.x, b.x), dm(a.y, b.y)), dm(a.z, b.z)); }

// Rust f32::clamp: a NaN stays NaN.
__device__ __forceinline__ float rs_clamp01(float v) {
  if (v < 0.0f) v = 0.0f;
  if (v > 1.0f) v = 1.0f;
  return v;
}

// Degenerate-triangle cases of geo.rs:73-88, decided once per triangle and kept
// in the record: 0 = proper triangle, 1 = a point (all equal), 2 = segment a..c
// (a == b), 3 = segment a..b (b == c or a == c).
enum : int { TRI_PROPER = 0, TRI_POINT = 1, TRI_SEG_AC = 2, TRI_SEG_AB = 3 };

__host__ __device__ __forceinline__ int degenerate_kind(float ax, float ay, float az, float bx, float by,
                                                        float bz, float cx, float cy, float cz) {
  bool ab = ax == bx && ay == by && az == bz;
  bool bc = bx == cx && by == cy && bz == cz;
  bool ac = ax == cx && ay == cy && az == cz;
  if (ab && bc && ac) return TRI_POINT;
  if (ab) return TRI_SEG_AC;
  if (bc || ac) return TRI_SEG_AB;
  return TRI_PROPER;
}

// geo.rs:141-151
__device__ __forceinline__ P3 closest_point_segment(P3 p, P3 a, P3 b) {
  P3 ab = dvsub(b, a);
  float m = dvdot(ab, ab);
  P3 ap = dvsub(p, a);
  float s = rs_clamp01(fd(dvdot(ab, ap), m));
  return dvadd(a, dvmul(ab, s));
}

// geo.rs:70-138 (Embree Voronoi regions) for a proper triangle.
__device__ __forceinline__ P3 closest_point_proper(P3 p, P3 a, P3 b, P3 c) {
  P3 ab = dvsub(b, a);
  P3 ac = dvsub(c, a);
  P3 ap = dvsub(p, a);
  float d1 = dvdot(ab, ap);
  float d2 = dvdot(ac, ap);
  if (d1 <= 0.0f && d2 <= 0.0f) return a;
  P3 bp = dvsub(p, b);
  float d3 = dvdot(ab, bp);
  float d4 = dvdot(ac, bp);
  if (d3 >= 0.0f && d4 <= d3) return b;
  P3 cp = dvsub(p, c);
  float d5 = dvdot(ab, cp);
  float d6 = dvdot(ac, cp);
  if (d6 >= 0.0f && d5 <= d6) return c;
  float vc = ds(dm(d1, d4), dm(d3, d2));
  if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) return dvadd(a, dvmul(ab, fd(d1, ds(d1, d3))));
  float vb = ds(dm(d5, d2), dm(d1, d6));
  if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) return dvadd(a, dvmul(ac, fd(d2, ds(d2, d6))));
  float va = ds(dm(d3, d6), dm(d5, d4));
  float d43 = ds(d4, d3), d56 = ds(d5, d6);
  if (va <= 0.0f && d43 >= 0.0f && d56 >= 0.0f) return dvadd(b, dvmul(dvsub(c, b), fd(d43, da(d43, d56))));
  float denom = fd(1.0f, da(da(va, vb), vc));
  float v = dm(vb, denom);
  float w = dm(vc, denom);
  return dvadd(dvadd(a, dvmul(ab, v)), dvmul(ac, w));
}

// geo.rs:70-138 including the degenerate fallbacks (kind from degenerate_kind).
__device__ __forceinline__ P3 closest_point_triangle(P3 p, P3 a, P3 b, P3 c, int kind) {
  if (kind == TRI_PROPER) return closest_point_proper(p, a, b, c);
  if (kind == TRI_POINT) return a;
  if (kind == TRI_SEG_AC) return closest_point_segment(p, a, c);
  return closest_point_segment(p, a, b);
}

// geo.rs:33-37
__device__ __forceinline__ float point_triangle_distance2(P3 p, P3 a, P3 b, P3 c, int kind) {
  P3 d = dvsub(p, closest_point_triangle(p, a, b, c, kind));
  return dvdot(d, d);
}

// closest_point_proper without branches: every dot product is formed, the
// first region whose test holds (in the reference's order) is chosen by
// selects, and the one division that region needs is done once.  Each
// region's value comes from the same operations as above, so the result is
// bit-identical; lanes of a warp in different regions no longer run every
// region's path and division one after another.
// The region choice and result of closest_point_proper_sel from the six dot
// products d1..d6 (ab.ap, ac.ap, ab.bp, ac.bp, ab.cp, ac.cp).
__device__ __forceinline__ P3 closest_from_dots(P3 a, P3 b, P3 c, P3 ab, P3 ac, float d1, float d2, float d3,
                                                float d4, float d5, float d6) {
  const float vc = ds(dm(d1, d4), dm(d3, d2));
  const float vb = ds(dm(d5, d2), dm(d1, d6));
  const float va = ds(dm(d3, d6), dm(d5, d4));
  const float d43 = ds(d4, d3), d56 = ds(d5, d6);
  const bool rA = d1 <= 0.0f && d2 <= 0.0f;
  const bool rB = d3 >= 0.0f && d4 <= d3;
  const bool rC = d6 >= 0.0f && d5 <= d6;
  const bool eAB = vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f;
  const bool eAC = !eAB && vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f;
  const bool eBC = !eAB && !eAC && va <= 0.0f && d43 >= 0.0f && d56 >= 0.0f;
  const bool face = !eAB && !eAC && !eBC;
  const float num = eAB ? d1 : (eAC ? d2 : (eBC ? d43 : 1.0f));
  const float den = eAB ? ds(d1, d3) : (eAC ? ds(d2, d6) : (eBC ? da(d43, d56) : da(da(va, vb), vc)));
  const float q = fd(num, den);
  const P3 cb = dvsub(c, b);
  const P3 base = eBC ? b : a;
  const P3 e1 = eAC ? ac : (eBC ? cb : ab);
  const float s1 = face ? dm(vb, q) : q;
  P3 x = dvadd(base, dvmul(e1, s1));
  const P3 x2 = dvadd(x, dvmul(ac, dm(vc, q)));
  if (face) x = x2;
  if (rA || rB || rC) x = rA ? a : (rB ? b : c);
  return x;
}

__device__ __forceinline__ P3 closest_point_proper_sel(P3 p, P3 a, P3 b, P3 c) {
  const P3 ab = dvsub(b, a), ac = dvsub(c, a);
  const P3 ap = dvsub(p, a), bp = dvsub(p, b), cp = dvsub(p, c);
  return closest_from_dots(a, b, c, ab, ac, dvdot(ab, ap), dvdot(ac, ap), dvdot(ab, bp), dvdot(ac, bp),
                           dvdot(ab, cp), dvdot(ac, cp));
}

// Points that share x and y (the cells of one grid row along z) share the x
// and y parts of the six dot products, (e.x q.x + e.y q.y) in the reference's
// order (x*x' + y*y') + z*z': RowXY holds them, formed once per row, and
// row_distance2 adds each point's z terms.  Same operations, same rounding:
// bit-identical to point_triangle_distance2_sel of a proper triangle.
struct RowXY {
  float d1, d2, d3, d4, d5, d6;
};
__device__ __forceinline__ RowXY row_xy(float px, float py, P3 a, P3 b, P3 c) {
  const P3 ab = dvsub(b, a), ac = dvsub(c, a);
  const float apx = ds(px, a.x), apy = ds(py, a.y), bpx = ds(px, b.x), bpy = ds(py, b.y);
  const float cpx = ds(px, c.x), cpy = ds(py, c.y);
  return {da(dm(ab.x, apx), dm(ab.y, apy)), da(dm(ac.x, apx), dm(ac.y, apy)), da(dm(ab.x, bpx), dm(ab.y, bpy)),
          da(dm(ac.x, bpx), dm(ac.y, bpy)), da(dm(ab.x, cpx), dm(ab.y, cpy)), da(dm(ac.x, cpx), dm(ac.y, cpy))};
}
__device__ __forceinline__ float row_distance2(const RowXY& r, P3 p, P3 a, P3 b, P3 c) {
  const P3 ab = dvsub(b, a), ac = dvsub(c, a);
  const float apz = ds(p.z, a.z), bpz = ds(p.z, b.z), cpz = ds(p.z, c.z);
  const P3 x = closest_from_dots(a, b, c, ab, ac, da(r.d1, dm(ab.z, apz)), da(r.d2, dm(ac.z, apz)),
                                 da(r.d3, dm(ab.z, bpz)), da(r.d4, dm(ac.z, bpz)), da(r.d5, dm(ab.z, cpz)),
                                 da(r.d6, dm(ac.z, cpz)));
  const P3 d = dvsub(p, x);
  return dvdot(d, d);
}

// point_triangle_distance2 with the branch-free proper case.
__device__ __forceinline__ float point_triangle_distance2_sel(P3 p, P3 a, P3 b, P3 c, int kind) {
  const P3 cp = kind == TRI_PROPER ? closest_point_proper_sel(p, a, b, c) : closest_point_triangle(p, a, b, c, kind);
  const P3 d = dvsub(p, cp);
  return dvdot(d, d);
}

// geo.rs:43-56: positive when (p - closest) . (ab x ac) > 0, else -distance.
__device__ __forceinline__ float point_triangle_signed_distance(P3 p, P3 a, P3 b, P3 c, int kind) {
  P3 cp = closest_point_triangle(p, a, b, c, kind);
  P3 dir = dvsub(p, cp);
  P3 n = vcross(vsub(b, a), vsub(c, a));
  float d = fsqrt(dvdot(dir, dir));
  return vdot(dir, n) > 0.0f ? d : -d;
}

// signed distance with the branch-free proper case.
__device__ __forceinline__ float point_triangle_signed_distance_sel(P3 p, P3 a, P3 b, P3 c, int kind) {
  P3 cp = kind == TRI_PROPER ? closest_point_proper_sel(p, a, b, c) : closest_point_triangle(p, a, b, c, kind);
  P3 dir = dvsub(p, cp);
  P3 n = vcross(vsub(b, a), vsub(c, a));
  float d = fsqrt(dvdot(dir, dir));
  return vdot(dir, n) > 0.0f ? d : -d;
}


// geo.rs:165-216 for a +axis ray; (y, z) of the projection rotate with the axis
// as in the reference (X: y,z; Y: z,x; Z: x,y).  Returns true with *t on a hit.
template <int AXIS>
__device__ __forceinline__ bool ray_hit_aligned(P3 o, P3 t0, P3 t1, P3 t2, float* t_out) {
  constexpr int IX = AXIS, IY = (AXIS + 1) % 3, IZ = (AXIS + 2) % 3;
  P3 e01 = vsub(t1, t0), e12 = vsub(t2, t1), e20 = vsub(t0, t2);
  P3 p0 = vsub(o, t0), p1 = vsub(o, t1), p2 = vsub(o, t2);
  float w0 = fs(fm(vget(p1, IZ), vget(e12, IY)), fm(vget(p1, IY), vget(e12, IZ)));
  float w1 = fs(fm(vget(p2, IZ), vget(e20, IY)), fm(vget(p2, IY), vget(e20, IZ)));
  float w2 = fs(fm(vget(p0, IZ), vget(e01, IY)), fm(vget(p0, IY), vget(e01, IZ)));
  if ((w0 < 0.0f && w1 < 0.0f && w2 < 0.0f) || (w0 > 0.0f && w1 > 0.0f && w2 > 0.0f)) {
    float num = fa(fa(fm(w0, vget(p0, IX)), fm(w2, vget(p2, IX))), fm(w1, vget(p1, IX)));
    float t = fd(-num, fa(fa(w0, w1), w2));
    if (t > 0.0f) {
      *t_out = t;
      return true;
    }
  }
  return false;
}

__device__ __forceinline__ bool ray_hit_axis(int axis, P3 o, P3 t0, P3 t1, P3 t2, float* t) {
  if (axis == 0) return ray_hit_aligned<0>(o, t0, t1, t2, t);
  if (axis == 1) return ray_hit_aligned<1>(o, t0, t1, t2, t);
  return ray_hit_aligned<2>(o, t0, t1, t2, t);
}

// float-cmp 0.9 approx_eq!(f32, a, b, ulps = 2, epsilon = 1e-6): equal, or
// |a - b| <= epsilon, or the i32 bit patterns (wrapping difference, saturating
// abs) within 2.
__device__ __forceinline__ bool approx_eq_band(float a, float b) {
  if (a == b) return true;
  if (fabsf(fs(a, b)) <= 1e-6f) return true;
  int32_t diff = (int32_t)((uint32_t)__float_as_int(a) - (uint32_t)__float_as_int(b));
  int32_t ad = diff == INT32_MIN ? INT32_MAX : (diff < 0 ? -diff : diff);
  return ad <= 2;
}

// lib.rs:315-332: -1 Less, 0 Equal, 1 Greater; *nan set where the crate panics.
__device__ __forceinline__ int compare_distances(float a, float b, bool* nan) {
  float A = fabsf(a), B = fabsf(b);
  if (approx_eq_band(A, B)) {
    bool an = signbit(a), bn = signbit(b);
    if (an && !bn) return 1;
    if (!an && bn) return -1;
  }
  if (A < B) return -1;
  if (A > B) return 1;
  if (A == B) return 0;
  *nan = true;
  return 0;
}

// A fold under compare_distances (`best` replaced by each d it puts before
// it) only takes a d with |d| <= B + one tie band, B = |best|: a larger
// magnitude can win only by the sign rule inside the band.  A replacement
// that raises the magnitude leaves a positive best, which the next such
// raise needs to be negative, so no fold from |best| = B ever holds a value
// above B + one band (at most max(1e-6, 2 ulps of B)).  fold_reach(B) is B
// plus two bands with room for rounding: a d with |d| > fold_reach(B) is
// before no value of such a fold.  `!(|d| > reach)` keeps NaN distances.
__device__ __forceinline__ float fold_reach(float B) { return fmaf(B, 1.0f + 0x1p-19f, 4.0e-6f); }

// Plane bound.  Whatever Voronoi region the reference's f32 closest point x
// takes (closest_point_proper), x lies within rounding of the triangle's
// plane: a vertex; a point a + s e of an edge with s in [0, 1] (the region
// tests make the computed s so); or, in the face region, a + ab v + ac w,
// whose rounding is at most ~2^-22 (|a| + |ab||v| + |ac||w|).  If the weights
// are so inaccurate that |ab||v| + |ac||w| is large, then so is |x - a| (at
// least that sum over sqrt(2 / (1 - |cos A|)), A the angle at a: 32 when
// sin A >= 1/16), and x is far from p anyway.  Either way the reference's
// distance from p is at least
//     |h| (1 - 2^-13) - 2^-11 (|p|max + |triangle|max),
// h the distance from p to the plane, for a proper triangle with
// sin^2 A >= 1/200 and coordinates below 2^30 (a margin of some 64x over the
// error terms).  So a triangle whose bound exceeds a search's best distance
// cannot be strictly nearer.  TriPlane holds the unit normal (n.w = n . a)
// and the triangle's share of the slack, +inf where the bound does not apply
// (the normal is then zero).  Float arithmetic suffices: for the triangles
// kept the normal's rounding is a few ulps, far inside the slack, and the
// shape test asks sin^2 A >= 1/200 so that its own rounding cannot admit
// sin A < 1/16.
struct TriPlane {
  float4 n;
  float slack;
};
__device__ __forceinline__ TriPlane tri_plane(P3 a, P3 b, P3 c, int kind) {
  const float abx = b.x - a.x, aby = b.y - a.y, abz = b.z - a.z;
  const float acx = c.x - a.x, acy = c.y - a.y, acz = c.z - a.z;
  const float nx = aby * acz - abz * acy, ny = abz * acx - abx * acz, nz = abx * acy - aby * acx;
  const float nn2 = nx * nx + ny * ny + nz * nz;
  const float lab2 = abx * abx + aby * aby + abz * abz, lac2 = acx * acx + acy * acy + acz * acz;
  const float vmax = fmaxf(fmaxf(fmaxf(fabsf(a.x), fabsf(a.y)), fmaxf(fabsf(a.z), fabsf(b.x))),
                           fmaxf(fmaxf(fabsf(b.y), fabsf(b.z)), fmaxf(fmaxf(fabsf(c.x), fabsf(c.y)), fabsf(c.z))));
  const bool ok = kind == TRI_PROPER && vmax < 0x1p30f && nn2 > 0.0f && 200.0f * nn2 >= lab2 * lac2;
  if (!ok) return {make_float4(0.f, 0.f, 0.f, 0.f), INFINITY};
  const float inv = rsqrtf(nn2);
  const float ux = nx * inv, uy = ny * inv, uz = nz * inv;
  return {make_float4(ux, uy, uz, ux * a.x + uy * a.y + uz * a.z), 0x1p-11f * vmax};
}
// The query's share of the slack.
__device__ __forceinline__ float plane_query_slack(P3 p) {
  return 0x1p-11f * fmaxf(fabsf(p.x), fmaxf(fabsf(p.y), fabsf(p.z)));
}
// The lower bound of the reference's distance from p (-inf where it does not apply).
__device__ __forceinline__ float plane_bound(float4 n, float slack, P3 p, float pslack) {
  const float h = fabsf(fmaf(n.x, p.x, fmaf(n.y, p.y, fmaf(n.z, p.z, -n.w))));
  return fmaf(h, 1.0f - 0x1p-13f, -(slack + pslack));
}
// A bound above this proves the triangle's squared distance exceeds d2.
__device__ __forceinline__ float plane_above(float d2) { return sqrtf(d2) * (1.0f + 0x1p-18f); }

// geo.rs:4-22: AABB grown by 1e-4 on every side (f32 min/max then -/+ 1e-4).
__device__ __forceinline__ void padded_box(P3 a, P3 b, P3 c, P3* lo, P3* hi) {
  const float e = 0.0001f;
  *lo = {fs(fminf(a.x, fminf(b.x, c.x)), e), fs(fminf(a.y, fminf(b.y, c.y)), e), fs(fminf(a.z, fminf(b.z, c.z)), e)};
  *hi = {fa(fmaxf(a.x, fmaxf(b.x, c.x)), e), fa(fmaxf(a.y, fmaxf(b.y, c.y)), e), fa(fmaxf(a.z, fmaxf(b.z, c.z)), e)};
}

}  // namespace m2s
