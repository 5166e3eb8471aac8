// FP64 re-decision of the f32 tests whose outcome rounding could have
// changed — a report, never a change of output.
//
// The results of this library are the reference's f32 arithmetic, decision
// for decision.  Two kinds of decision steer a result:
//  * the aligned ray test (geo.rs:165-216): the signs of the three edge
//    functions w0, w1, w2 and of t decide whether a ray crosses a triangle,
//    and the crossings' parities decide Raycast signs;
//  * the Voronoi-region tests of closest_point_triangle (geo.rs:97-128): the
//    signs of d1..d6, va, vb, vc and of d4 - d3, d5 - d6 pick the region, and
//    so the closest point.
// A decision is flagged ambiguous when the quantity it compares lies within
// a forward-error bound of the threshold: the bound is 8 units of roundoff
// (2^-24) times the sum of the magnitudes of the terms the f32 operations
// combine, plus the propagated bounds of their operands — above what the
// operations can accumulate.  Only flagged decisions are re-decided in FP64
// from the same f32 inputs (differences and products of f32 values are
// exact or nearly so in double), and the counts of flagged decisions and of
// those FP64 decides the other way are reported.
#pragma once

#include "m2s_geo.cuh"

namespace m2s {

constexpr float kAuditGamma = 8.0f * 5.9604645e-8f;  // 8 x 2^-24

struct RayAudit {
  bool hit32;      // the f32 decision (the reference's, what the results use)
  bool ambiguous;  // some sign it depends on lies within its error bound
  bool hit64;      // the FP64 decision (= hit32 unless ambiguous)
  float t32;       // the f32 hit distance (when hit32)
  double t64;      // the FP64 hit distance (when hit64 and ambiguous)
};

// geo.rs:165-216 for a +AXIS ray from o, audited.
template <int AXIS>
__device__ __forceinline__ RayAudit ray_audit(P3 o, P3 t0, P3 t1, P3 t2) {
  constexpr int IX = AXIS, IY = (AXIS + 1) % 3, IZ = (AXIS + 2) % 3;
  RayAudit r;
  r.t32 = 0.0f;
  r.t64 = 0.0;
  r.hit32 = ray_hit_aligned<AXIS>(o, t0, t1, t2, &r.t32);
  const P3 e01 = vsub(t1, t0), e12 = vsub(t2, t1), e20 = vsub(t0, t2);
  const P3 p0 = vsub(o, t0), p1 = vsub(o, t1), p2 = vsub(o, t2);
  const float a0 = fm(vget(p1, IZ), vget(e12, IY)), b0 = fm(vget(p1, IY), vget(e12, IZ));
  const float a1 = fm(vget(p2, IZ), vget(e20, IY)), b1 = fm(vget(p2, IY), vget(e20, IZ));
  const float a2 = fm(vget(p0, IZ), vget(e01, IY)), b2 = fm(vget(p0, IY), vget(e01, IZ));
  const float w0 = fs(a0, b0), w1 = fs(a1, b1), w2 = fs(a2, b2);
  const float bw0 = kAuditGamma * (fabsf(a0) + fabsf(b0)), bw1 = kAuditGamma * (fabsf(a1) + fabsf(b1));
  const float bw2 = kAuditGamma * (fabsf(a2) + fabsf(b2));
  r.ambiguous = fabsf(w0) <= bw0 || fabsf(w1) <= bw1 || fabsf(w2) <= bw2;
  if (!r.ambiguous && ((w0 < 0.0f && w1 < 0.0f && w2 < 0.0f) || (w0 > 0.0f && w1 > 0.0f && w2 > 0.0f))) {
    // t > 0 exactly when the numerator's sign is opposite the common sign
    // of the weights; the numerator's bound adds the weights' own bounds.
    const float c0 = fm(w0, vget(p0, IX)), c2 = fm(w2, vget(p2, IX)), c1 = fm(w1, vget(p1, IX));
    const float num = fa(fa(c0, c2), c1);
    const float bn = kAuditGamma * (fabsf(c0) + fabsf(c1) + fabsf(c2)) + bw0 * fabsf(vget(p0, IX)) +
                     bw1 * fabsf(vget(p1, IX)) + bw2 * fabsf(vget(p2, IX));
    r.ambiguous = fabsf(num) <= bn;
  }
  r.hit64 = r.hit32;
  if (r.ambiguous) {
    const double ox = vget(o, IX), oy = vget(o, IY), oz = vget(o, IZ);
    const double x0 = vget(t0, IX), y0 = vget(t0, IY), z0 = vget(t0, IZ);
    const double x1 = vget(t1, IX), y1 = vget(t1, IY), z1 = vget(t1, IZ);
    const double x2 = vget(t2, IX), y2 = vget(t2, IY), z2 = vget(t2, IZ);
    const double W0 = (oz - z1) * (y2 - y1) - (oy - y1) * (z2 - z1);
    const double W1 = (oz - z2) * (y0 - y2) - (oy - y2) * (z0 - z2);
    const double W2 = (oz - z0) * (y1 - y0) - (oy - y0) * (z1 - z0);
    bool hit = false;
    if ((W0 < 0 && W1 < 0 && W2 < 0) || (W0 > 0 && W1 > 0 && W2 > 0)) {
      const double t = -(W0 * (ox - x0) + W2 * (ox - x2) + W1 * (ox - x1)) / (W0 + W1 + W2);
      hit = t > 0;
      r.t64 = t;
    }
    r.hit64 = hit;
  }
  return r;
}

struct RegionAudit {
  int region32;    // 0 = vertex a, 1 = vertex b, 2 = vertex c, 3 = edge ab, 4 = edge ac, 5 = edge bc, 6 = face
  bool ambiguous;  // a test on the way to it lies within its error bound
  int region64;    // the FP64 choice (= region32 unless ambiguous)
};

// The region closest_point_triangle picks for p on a proper triangle
// (geo.rs:97-128, tests in the reference's order), audited.  The strict
// build's arithmetic; the fast build's fused multiply-adds err less.
__device__ __forceinline__ RegionAudit region_audit(P3 p, P3 a, P3 b, P3 c) {
  auto dotb = [](P3 x, P3 y, float* bound) {
    const float m0 = fm(x.x, y.x), m1 = fm(x.y, y.y), m2 = fm(x.z, y.z);
    *bound = kAuditGamma * (fabsf(m0) + fabsf(m1) + fabsf(m2));
    return fa(fa(m0, m1), m2);
  };
  const P3 ab = vsub(b, a), ac = vsub(c, a), ap = vsub(p, a), bp = vsub(p, b), cp = vsub(p, c);
  float e1, e2, e3, e4, e5, e6;
  const float d1 = dotb(ab, ap, &e1), d2 = dotb(ac, ap, &e2);
  const float d3 = dotb(ab, bp, &e3), d4 = dotb(ac, bp, &e4);
  const float d5 = dotb(ab, cp, &e5), d6 = dotb(ac, cp, &e6);
  // differences of two quantities with bounds ea, eb
  auto near0 = [](float v, float e) { return fabsf(v) <= e; };
  auto prodb = [](float x, float ex, float y, float ey) { return fabsf(x) * ey + fabsf(y) * ex + ex * ey; };
  const float vc = fs(fm(d1, d4), fm(d3, d2));
  const float evc = prodb(d1, e1, d4, e4) + prodb(d3, e3, d2, e2) + kAuditGamma * (fabsf(fm(d1, d4)) + fabsf(fm(d3, d2)));
  const float vb = fs(fm(d5, d2), fm(d1, d6));
  const float evb = prodb(d5, e5, d2, e2) + prodb(d1, e1, d6, e6) + kAuditGamma * (fabsf(fm(d5, d2)) + fabsf(fm(d1, d6)));
  const float va = fs(fm(d3, d6), fm(d5, d4));
  const float eva = prodb(d3, e3, d6, e6) + prodb(d5, e5, d4, e4) + kAuditGamma * (fabsf(fm(d3, d6)) + fabsf(fm(d5, d4)));
  const float d43 = fs(d4, d3), d56 = fs(d5, d6);
  const float e43 = e4 + e3 + kAuditGamma * fabsf(d43), e56 = e5 + e6 + kAuditGamma * fabsf(d56);
  RegionAudit r;
  bool amb = false;
  // The decision chain, flagging every comparison it makes on the way.
  amb |= near0(d1, e1) || near0(d2, e2);
  if (d1 <= 0.0f && d2 <= 0.0f) {
    r.region32 = 0;
  } else {
    amb |= near0(d3, e3) || near0(d4 - d3, e4 + e3);
    if (d3 >= 0.0f && d4 <= d3) {
      r.region32 = 1;
    } else {
      amb |= near0(d6, e6) || near0(d5 - d6, e5 + e6);
      if (d6 >= 0.0f && d5 <= d6) {
        r.region32 = 2;
      } else {
        amb |= near0(vc, evc);
        if (vc <= 0.0f && d1 >= 0.0f && d3 <= 0.0f) {
          r.region32 = 3;
        } else {
          amb |= near0(vb, evb);
          if (vb <= 0.0f && d2 >= 0.0f && d6 <= 0.0f) {
            r.region32 = 4;
          } else {
            amb |= near0(va, eva) || near0(d43, e43) || near0(d56, e56);
            r.region32 = (va <= 0.0f && d43 >= 0.0f && d56 >= 0.0f) ? 5 : 6;
          }
        }
      }
    }
  }
  r.ambiguous = amb;
  r.region64 = r.region32;
  if (amb) {
    const double ABx = (double)b.x - a.x, ABy = (double)b.y - a.y, ABz = (double)b.z - a.z;
    const double ACx = (double)c.x - a.x, ACy = (double)c.y - a.y, ACz = (double)c.z - a.z;
    auto dd = [](double x0, double y0, double z0, double x1, double y1, double z1) { return x0 * x1 + y0 * y1 + z0 * z1; };
    const double APx = (double)p.x - a.x, APy = (double)p.y - a.y, APz = (double)p.z - a.z;
    const double BPx = (double)p.x - b.x, BPy = (double)p.y - b.y, BPz = (double)p.z - b.z;
    const double CPx = (double)p.x - c.x, CPy = (double)p.y - c.y, CPz = (double)p.z - c.z;
    const double D1 = dd(ABx, ABy, ABz, APx, APy, APz), D2 = dd(ACx, ACy, ACz, APx, APy, APz);
    const double D3 = dd(ABx, ABy, ABz, BPx, BPy, BPz), D4 = dd(ACx, ACy, ACz, BPx, BPy, BPz);
    const double D5 = dd(ABx, ABy, ABz, CPx, CPy, CPz), D6 = dd(ACx, ACy, ACz, CPx, CPy, CPz);
    const double VC = D1 * D4 - D3 * D2, VB = D5 * D2 - D1 * D6, VA = D3 * D6 - D5 * D4;
    if (D1 <= 0 && D2 <= 0) r.region64 = 0;
    else if (D3 >= 0 && D4 <= D3) r.region64 = 1;
    else if (D6 >= 0 && D5 <= D6) r.region64 = 2;
    else if (VC <= 0 && D1 >= 0 && D3 <= 0) r.region64 = 3;
    else if (VB <= 0 && D2 >= 0 && D6 <= 0) r.region64 = 4;
    else if (VA <= 0 && D4 - D3 >= 0 && D5 - D6 >= 0) r.region64 = 5;
    else r.region64 = 6;
  }
  return r;
}

}  // namespace m2s
