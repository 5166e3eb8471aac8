// CPU oracle for mesh_to_sdf_b200 — test infrastructure, never shipped.
//
// A restatement of the Rust crate `mesh_to_sdf` (file:line citations are to that
// crate, `mesh_to_sdf/src/...`).  The CUDA library is checked against this file
// and bench.py times it as the CPU baseline.  Geometry lives in geo_ref.hpp.
//
// Third-party pieces the reference leans on are restated from their documented
// behaviour, not copied:
//   * bvh 0.10 / rstar 0.12 trees only pre-filter candidates.  Any tree whose
//     boxes hold the 1e-4-padded triangle AABBs gives the same exact-test
//     results, so a small median-split BVH (CpuBvh below) stands in for both.
//   * float-cmp 0.9 approx_eq — geo_ref.hpp:approx_eq_ulps2_eps1e6.
//   * rayon's thread count — the n_threads argument.
#include "m2s_oracle.h"

#include <omp.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <limits>
#include <mutex>
#include <queue>
#include <thread>
#include <array>
#include <set>
#include <vector>

#include "geo_ref.hpp"

using namespace m2s_oracle;

namespace {

enum {
  ST_OK = 0,
  ST_INVALID_ARGUMENT = 1,
  ST_NONFINITE_QUERY = 2,
  ST_INDEX_COUNT = 3,
  ST_INDEX_RANGE = 4,
  ST_NAN_DISTANCE = 5,
  ST_EMPTY_MESH = 6,
};

const float F32_MAX = std::numeric_limits<float>::max();

inline V3 load3(const float* p) { return {p[0], p[1], p[2]}; }

int threads_or_all(int n) { return n > 0 ? n : (int)std::thread::hardware_concurrency(); }

struct Tri {
  uint32_t i, j, k;
};

// Topology::get_triangles (lib.rs:193-215): lists take indices three at a time
// (itertools tuples, lib.rs:204/208); strips take every window of three with no
// winding flip (tuple_windows, lib.rs:211/213).
int expand_topology(uint64_t nv, const void* idx, uint64_t ni, int bits, int topo,
                    std::vector<Tri>* out) {
  auto get = [&](uint64_t k) -> uint64_t {
    if (bits == 16) return ((const uint16_t*)idx)[k];
    if (bits == 32) return ((const uint32_t*)idx)[k];
    return k;
  };
  if (bits != 0 && bits != 16 && bits != 32) return ST_INVALID_ARGUMENT;
  if (topo != 0 && topo != 1) return ST_INVALID_ARGUMENT;
  uint64_t n = bits == 0 ? nv : ni;
  if (bits != 0 && ni > 0 && idx == nullptr) return ST_INVALID_ARGUMENT;
  out->clear();
  if (topo == 0) {
    if (n % 3 != 0) return ST_INDEX_COUNT;  // lib.rs:203, lib.rs:207
    out->reserve(n / 3);
    for (uint64_t t = 0; t + 2 < n; t += 3) out->push_back({(uint32_t)get(t), (uint32_t)get(t + 1), (uint32_t)get(t + 2)});
  } else {
    if (n >= 3) {
      out->reserve(n - 2);
      for (uint64_t t = 0; t + 2 < n; ++t) out->push_back({(uint32_t)get(t), (uint32_t)get(t + 1), (uint32_t)get(t + 2)});
    }
  }
  // Out-of-range indices panic in the reference through slice indexing.
  for (uint64_t k = 0; k < n; ++k)
    if (get(k) >= nv) return ST_INDEX_RANGE;
  return ST_OK;
}

struct Mesh {
  std::vector<V3> a, b, c;  // triangle corners in triangle order
  std::vector<Tri> tris;
  size_t size() const { return tris.size(); }
};

int make_mesh(const float* v, uint64_t nv, const void* idx, uint64_t ni, int bits, int topo, Mesh* m) {
  int st = expand_topology(nv, idx, ni, bits, topo, &m->tris);
  if (st) return st;
  size_t T = m->tris.size();
  m->a.resize(T);
  m->b.resize(T);
  m->c.resize(T);
  for (size_t t = 0; t < T; ++t) {
    m->a[t] = load3(v + 3 * (size_t)m->tris[t].i);
    m->b[t] = load3(v + 3 * (size_t)m->tris[t].j);
    m->c[t] = load3(v + 3 * (size_t)m->tris[t].k);
  }
  return ST_OK;
}

// ---------------------------------------------------------------------------
// Candidate filter standing in for the bvh / rstar trees.  Boxes are the
// reference's padded triangle AABBs (geo.rs:4-22), widened once more by a
// relative 1e-6 in double so the filter stays conservative at any scale.
struct CpuBvh {
  struct Node {
    double lo[3], hi[3];
    int left = -1, right = -1;
    int start = 0, count = 0;
  };
  std::vector<Node> nodes;
  std::vector<uint32_t> order;
  std::vector<double> tlo, thi;  // per-triangle padded box

  void build(const Mesh& m) {
    size_t T = m.size();
    nodes.clear();
    order.resize(T);
    tlo.resize(3 * T);
    thi.resize(3 * T);
    std::vector<double> cen(3 * T);
    for (size_t t = 0; t < T; ++t) {
      V3 mn, mx;
      triangle_bounding_box(m.a[t], m.b[t], m.c[t], &mn, &mx);
      for (int d = 0; d < 3; ++d) {
        double lo = v_get(mn, d), hi = v_get(mx, d);
        tlo[3 * t + d] = lo - 1e-6 * std::fabs(lo);
        thi[3 * t + d] = hi + 1e-6 * std::fabs(hi);
        cen[3 * t + d] = 0.5 * (lo + hi);
      }
      order[t] = (uint32_t)t;
    }
    if (T == 0) return;
    nodes.reserve(2 * T);
    build_rec(0, (int)T, cen);
  }

  int build_rec(int start, int count, const std::vector<double>& cen) {
    int id = (int)nodes.size();
    nodes.emplace_back();
    Node nd;
    for (int d = 0; d < 3; ++d) {
      nd.lo[d] = std::numeric_limits<double>::infinity();
      nd.hi[d] = -std::numeric_limits<double>::infinity();
    }
    double clo[3], chi[3];
    for (int d = 0; d < 3; ++d) {
      clo[d] = std::numeric_limits<double>::infinity();
      chi[d] = -std::numeric_limits<double>::infinity();
    }
    for (int k = start; k < start + count; ++k) {
      uint32_t t = order[k];
      for (int d = 0; d < 3; ++d) {
        nd.lo[d] = std::min(nd.lo[d], tlo[3 * t + d]);
        nd.hi[d] = std::max(nd.hi[d], thi[3 * t + d]);
        clo[d] = std::min(clo[d], cen[3 * t + d]);
        chi[d] = std::max(chi[d], cen[3 * t + d]);
      }
    }
    if (count <= 4) {
      nd.start = start;
      nd.count = count;
      nodes[id] = nd;
      return id;
    }
    int axis = 0;
    for (int d = 1; d < 3; ++d)
      if (chi[d] - clo[d] > chi[axis] - clo[axis]) axis = d;
    int mid = start + count / 2;
    std::nth_element(order.begin() + start, order.begin() + mid, order.begin() + start + count,
                     [&](uint32_t x, uint32_t y) {
                       double cx = cen[3 * x + axis], cy = cen[3 * y + axis];
                       return cx < cy || (cx == cy && x < y);
                     });
    nodes[id] = nd;
    int l = build_rec(start, mid - start, cen);
    int r = build_rec(mid, start + count - mid, cen);
    nodes[id].left = l;
    nodes[id].right = r;
    return id;
  }

  static double box_dist2(const double* lo, const double* hi, V3 p) {
    double s = 0;
    for (int d = 0; d < 3; ++d) {
      double x = v_get(p, d);
      double e = x < lo[d] ? lo[d] - x : (x > hi[d] ? x - hi[d] : 0.0);
      s += e * e;
    }
    return s;
  }

  // Exact nearest triangle under the f32 point_triangle_distance2 of geo.rs:33-37,
  // ties going to the lowest triangle index.  Returns -1 on an empty mesh.
  long nearest(const Mesh& m, V3 p, float* d2_out) const {
    if (nodes.empty()) return -1;
    float best = std::numeric_limits<float>::infinity();
    long best_t = std::numeric_limits<long>::max();
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
      const Node& nd = nodes[stack[--sp]];
      if (box_dist2(nd.lo, nd.hi, p) > (double)best) continue;
      if (nd.count) {
        for (int k = nd.start; k < nd.start + nd.count; ++k) {
          uint32_t t = order[k];
          if (box_dist2(&tlo[3 * t], &thi[3 * t], p) > (double)best) continue;
          float d2 = point_triangle_distance2(p, m.a[t], m.b[t], m.c[t]);
          if (!(d2 <= best)) continue;  // NaN distances never win
          if (d2 < best || (long)t < best_t) {
            best = d2;
            best_t = t;
          }
        }
        continue;
      }
      double dl = box_dist2(nodes[nd.left].lo, nodes[nd.left].hi, p);
      double dr = box_dist2(nodes[nd.right].lo, nodes[nd.right].hi, p);
      if (dl < dr) {
        stack[sp++] = nd.right;
        stack[sp++] = nd.left;
      } else {
        stack[sp++] = nd.left;
        stack[sp++] = nd.right;
      }
    }
    if (best_t == std::numeric_limits<long>::max()) {
      // Every distance was NaN: report triangle 0 so the index is defined.
      best_t = 0;
      best = point_triangle_distance2(p, m.a[0], m.b[0], m.c[0]);
    }
    *d2_out = best;
    return best_t;
  }

  // Triangles whose padded box lies within `r` of p (r in distance units).
  void within(V3 p, double r, std::vector<uint32_t>* out) const {
    out->clear();
    if (nodes.empty()) return;
    double r2 = r * r;
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
      const Node& nd = nodes[stack[--sp]];
      if (box_dist2(nd.lo, nd.hi, p) > r2) continue;
      if (nd.count) {
        for (int k = nd.start; k < nd.start + nd.count; ++k) {
          uint32_t t = order[k];
          if (box_dist2(&tlo[3 * t], &thi[3 * t], p) <= r2) out->push_back(t);
        }
        continue;
      }
      stack[sp++] = nd.left;
      stack[sp++] = nd.right;
    }
  }

  // Number of triangles that the +axis ray from o hits under geo.rs:165-216.
  // The box test only discards triangles that cannot be hit; every survivor is
  // decided by the reference's own aligned test.
  template <class F>
  void ray_hits(const Mesh& m, V3 o, int axis, F&& on_hit) const {
    if (nodes.empty()) return;
    const int iy = (axis + 1) % 3, iz = (axis + 2) % 3;
    double oy = v_get(o, iy), oz = v_get(o, iz), ox = v_get(o, axis);
    auto hit_box = [&](const double* lo, const double* hi) {
      return oy >= lo[iy] && oy <= hi[iy] && oz >= lo[iz] && oz <= hi[iz] && hi[axis] >= ox;
    };
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp) {
      const Node& nd = nodes[stack[--sp]];
      if (!hit_box(nd.lo, nd.hi)) continue;
      if (nd.count) {
        for (int k = nd.start; k < nd.start + nd.count; ++k) {
          uint32_t t = order[k];
          if (!hit_box(&tlo[3 * t], &thi[3 * t])) continue;
          float tt;
          if (ray_triangle_intersection_aligned(o, m.a[t], m.b[t], m.c[t], axis, &tt)) on_hit(t, tt);
        }
        continue;
      }
      stack[sp++] = nd.left;
      stack[sp++] = nd.right;
    }
  }
};

// 3-ray vote of bvh.rs:141-176 / rtree_bvh.rs:163-199: inside when at least two
// of the +X, +Y, +Z rays cross the mesh an odd number of times.
bool ray_vote_inside(const Mesh& m, const CpuBvh& bvh, V3 p) {
  int insides = 0;
  for (int axis = 0; axis < 3; ++axis) {
    uint32_t count = 0;
    bvh.ray_hits(m, p, axis, [&](uint32_t, float) { ++count; });
    if (count % 2 == 1) ++insides;
  }
  return insides > 1;
}

bool finite3(const float* q) { return std::isfinite(q[0]) && std::isfinite(q[1]) && std::isfinite(q[2]); }

// Bvh + Normal (bvh.rs:117-129) folds compare_distances over the tree's
// candidate list in the tree's traversal order.  The fold can only move within
// the near-tie band of the nearest distance, so this restatement folds that band
// in triangle-index order (the same order generate_sdf_default uses).
float normal_fold_near(const Mesh& m, const CpuBvh& bvh, V3 p, bool* nan) {
  float d2;
  long nn = bvh.nearest(m, p, &d2);
  if (nn < 0) return F32_MAX;
  double dstar = std::sqrt((double)d2);
  double band = dstar * (1.0 + 1e-5) + 4e-6;
  std::vector<uint32_t> cand;
  bvh.within(p, band + 2e-4, &cand);
  std::sort(cand.begin(), cand.end());
  float best = F32_MAX;
  for (uint32_t t : cand) {
    float d = point_triangle_signed_distance(p, m.a[t], m.b[t], m.c[t]);
    if (!(std::fabs((double)d) <= band)) continue;
    if (compare_distances(best, d, nan) == 1) best = d;
  }
  return best;
}

}  // namespace

extern "C" {

void orc_closest_point_triangle(const float* p, const float* a, const float* b, const float* c, float* out) {
  V3 r = closest_point_triangle(load3(p), load3(a), load3(b), load3(c));
  out[0] = r.x;
  out[1] = r.y;
  out[2] = r.z;
}
float orc_point_triangle_distance(const float* p, const float* a, const float* b, const float* c) {
  return point_triangle_distance(load3(p), load3(a), load3(b), load3(c));
}
float orc_point_triangle_distance2(const float* p, const float* a, const float* b, const float* c) {
  return point_triangle_distance2(load3(p), load3(a), load3(b), load3(c));
}
float orc_point_triangle_signed_distance(const float* p, const float* a, const float* b, const float* c) {
  return point_triangle_signed_distance(load3(p), load3(a), load3(b), load3(c));
}
int orc_ray_triangle_intersection_aligned(const float* o, const float* a, const float* b, const float* c, int axis,
                                          float* t) {
  return ray_triangle_intersection_aligned(load3(o), load3(a), load3(b), load3(c), axis, t) ? 1 : 0;
}
void orc_triangle_bounding_box(const float* a, const float* b, const float* c, float* mn, float* mx) {
  V3 lo, hi;
  triangle_bounding_box(load3(a), load3(b), load3(c), &lo, &hi);
  mn[0] = lo.x, mn[1] = lo.y, mn[2] = lo.z;
  mx[0] = hi.x, mx[1] = hi.y, mx[2] = hi.z;
}
int orc_compare_distances(float a, float b) {
  bool nan = false;
  int r = compare_distances(a, b, &nan);
  return nan ? 2 : r;
}

int orc_expand_topology(uint64_t nv, const void* idx, uint64_t ni, int bits, int topo, uint32_t* tris_out,
                        uint64_t* n_tris) {
  std::vector<Tri> tris;
  int st = expand_topology(nv, idx, ni, bits, topo, &tris);
  if (n_tris) *n_tris = tris.size();
  if (tris_out)
    for (size_t t = 0; t < tris.size(); ++t) {
      tris_out[3 * t] = tris[t].i;
      tris_out[3 * t + 1] = tris[t].j;
      tris_out[3 * t + 2] = tris[t].k;
    }
  return st;
}

int orc_generate_sdf(const float* v, uint64_t nv, const void* idx, uint64_t ni, int bits, int topo, const float* q,
                     uint64_t nq, int accel, int sign, float* out, uint64_t* out_len, int n_threads) {
  if (out_len) *out_len = 0;
  if (accel < 0 || accel > 3 || sign < 0 || sign > 1) return ST_INVALID_ARGUMENT;
  // lib.rs:374-376
  for (uint64_t i = 0; i < nq; ++i)
    if (!finite3(q + 3 * i)) return ST_NONFINITE_QUERY;
  Mesh m;
  int st = make_mesh(v, nv, idx, ni, bits, topo, &m);
  // generate_sdf_default never touches a triangle when there is no query.
  if (st == ST_INDEX_RANGE && accel == 0 && nq == 0) st = ST_OK;
  if (st) return st;
  const size_t T = m.size();
  const int nt = threads_or_all(n_threads);
  std::atomic<int> nan_seen{0};

  if (accel == 0) {
    // generate_sdf_default (default.rs:38-84).
#pragma omp parallel for num_threads(nt) schedule(dynamic, 16)
    for (int64_t i = 0; i < (int64_t)nq; ++i) {
      V3 p = load3(q + 3 * i);
      float best = F32_MAX;
      uint32_t hits = 0;
      bool nan = false;
      for (size_t t = 0; t < T; ++t) {
        if (sign == 0) {
          float d = point_triangle_distance(p, m.a[t], m.b[t], m.c[t]);
          best = rs_min(best, d);
          hits += ray_triangle_intersection_aligned(p, m.a[t], m.b[t], m.c[t], 0, nullptr) ? 1u : 0u;
        } else {
          float d = point_triangle_signed_distance(p, m.a[t], m.b[t], m.c[t]);
          if (compare_distances(d, best, &nan) == -1) best = d;
        }
      }
      if (nan) nan_seen = 1;
      out[i] = hits % 2 == 0 ? best : -best;
    }
    if (nan_seen) return ST_NAN_DISTANCE;
    if (out_len) *out_len = nq;
    return ST_OK;
  }

  if (T == 0) {
    if (accel == 3) return ST_OK;  // rtree_bvh.rs:96-97, 124-126: empty Vec
    if (nq == 0) {
      if (out_len) *out_len = 0;
      return ST_OK;
    }
    return ST_EMPTY_MESH;  // rtree.rs:148 unwrap on None; bvh has no root node
  }
  CpuBvh bvh;
  bvh.build(m);
  // RtreeBvh's query loop is serial in the reference (rtree_bvh.rs:150-151).
  const int nt_q = nt;
#pragma omp parallel for num_threads(nt_q) schedule(dynamic, 64)
  for (int64_t i = 0; i < (int64_t)nq; ++i) {
    V3 p = load3(q + 3 * i);
    bool nan = false;
    float r;
    if (accel == 1 && sign == 1) {
      r = normal_fold_near(m, bvh, p, &nan);
    } else {
      float d2;
      long t = bvh.nearest(m, p, &d2);
      if (accel == 2) {
        // query_sdf_rtree (rtree.rs:137-157)
        r = point_triangle_signed_distance(p, m.a[t], m.b[t], m.c[t]);
      } else {
        // query_sdf_bvh Raycast (bvh.rs:283-328), query_sdf_rtree_bvh (rtree_bvh.rs:150-199)
        float d = point_triangle_distance(p, m.a[t], m.b[t], m.c[t]);
        r = ray_vote_inside(m, bvh, p) ? -d : d;
      }
    }
    if (nan) nan_seen = 1;
    out[i] = r;
  }
  if (nan_seen) return ST_NAN_DISTANCE;
  if (out_len) *out_len = nq;
  return ST_OK;
}

int orc_query_vector_to_closest_point(const float* v, uint64_t nv, const void* idx, uint64_t ni, int bits, int topo,
                                      const float* q, uint64_t nq, float* out_vec, uint8_t* out_inside,
                                      uint64_t* out_len, int n_threads) {
  if (out_len) *out_len = 0;
  Mesh m;
  int st = make_mesh(v, nv, idx, ni, bits, topo, &m);
  if (st) return st;
  if (m.size() == 0) return ST_EMPTY_MESH;  // build_sdf_acceleration_rtree_bvh returns None
  for (uint64_t i = 0; i < nq; ++i)
    if (!finite3(q + 3 * i)) return ST_NONFINITE_QUERY;
  CpuBvh bvh;
  bvh.build(m);
  const int nt = threads_or_all(n_threads);
#pragma omp parallel for num_threads(nt) schedule(dynamic, 64)
  for (int64_t i = 0; i < (int64_t)nq; ++i) {
    V3 p = load3(q + 3 * i);
    float d2;
    long t = bvh.nearest(m, p, &d2);
    V3 cp = closest_point_triangle(p, m.a[t], m.b[t], m.c[t]);
    V3 vec = v_sub(cp, p);  // rtree_bvh.rs:273
    out_vec[3 * i] = vec.x;
    out_vec[3 * i + 1] = vec.y;
    out_vec[3 * i + 2] = vec.z;
    out_inside[i] = ray_vote_inside(m, bvh, p) ? 1 : 0;
  }
  if (out_len) *out_len = nq;
  return ST_OK;
}

// ---------------------------------------------------------------------------
// Grid helpers (grid.rs).

void orc_grid_from_bounding_box(const float* mn, const float* mx, const uint64_t* n, float* first, float* size) {
  // grid.rs:59-74
  V3 fc = {(float)n[0], (float)n[1], (float)n[2]};
  V3 d = v_sub(load3(mx), load3(mn));
  V3 s = {d.x / fc.x, d.y / fc.y, d.z / fc.z};
  V3 f = v_add(load3(mn), v_fmul(s, 0.5f));
  first[0] = f.x, first[1] = f.y, first[2] = f.z;
  size[0] = s.x, size[1] = s.y, size[2] = s.z;
}

void orc_grid_cell_center(const float* first, const float* size, const uint64_t* cell, float* out) {
  // grid.rs:135-141
  for (int d = 0; d < 3; ++d) out[d] = first[d] + (float)cell[d] * size[d];
}

namespace {
struct GridD {
  V3 first, size;
  uint64_t n[3];
  V3 center(uint64_t x, uint64_t y, uint64_t z) const {
    return {first.x + (float)x * size.x, first.y + (float)y * size.y, first.z + (float)z * size.z};
  }
  uint64_t idx(uint64_t x, uint64_t y, uint64_t z) const { return z + y * n[2] + x * n[1] * n[2]; }
};

// Rust `f as isize` saturates and maps NaN to 0.
int64_t sat_isize(float f) {
  if (std::isnan(f)) return 0;
  if (f >= 9.2233720368547758e18f) return INT64_MAX;
  if (f <= -9.2233720368547758e18f) return INT64_MIN;
  return (int64_t)f;
}
uint64_t sat_usize(float f) {
  if (std::isnan(f) || f <= 0.0f) return 0;
  if (f >= 1.8446744073709552e19f) return UINT64_MAX;
  return (uint64_t)f;
}

// grid.rs:145-170; returns Inside (1) / Outside (0).
int snap(const GridD& g, V3 p, uint64_t* cell) {
  V3 half = v_fmul(g.size, 0.5f);
  V3 bbmin = v_sub(g.first, half);  // get_bounding_box().0, grid.rs:111
  V3 r = v_sub(p, bbmin);
  r = {r.x / g.size.x, r.y / g.size.y, r.z / g.size.z};
  int inside = 1;
  for (int d = 0; d < 3; ++d) {
    int64_t c = sat_isize(std::floor(v_get(r, d)));
    int64_t hi = (int64_t)g.n[d] - 1;
    int64_t cl = c < 0 ? 0 : (c > hi ? hi : c);
    if (cl != c) inside = 0;
    cell[d] = (uint64_t)cl;
  }
  return inside;
}

struct State {
  float dist;
  uint64_t cell[3];
  Tri tri;
};

// State ordering of generate/grid.rs:27-35: compare_distances(other, self), then
// cell, then the triangle's vertex-index tuple.  std::priority_queue pops the
// greatest, as Rust's BinaryHeap does.
struct StateLess {
  bool operator()(const State& s, const State& o) const {
    bool nan = false;
    int c = compare_distances(o.dist, s.dist, &nan);
    if (c == 0) {
      for (int d = 0; d < 3; ++d)
        if (s.cell[d] != o.cell[d]) return s.cell[d] < o.cell[d];
      if (s.tri.i != o.tri.i) return s.tri.i < o.tri.i;
      if (s.tri.j != o.tri.j) return s.tri.j < o.tri.j;
      return s.tri.k < o.tri.k;
    }
    return c < 0;
  }
};

float not_nan_or_max(float d) { return std::isnan(d) ? F32_MAX : d; }
}  // namespace

int orc_grid_snap_point(const float* first, const float* size, const uint64_t* n, const float* p, uint64_t* cell_out) {
  GridD g{load3(first), load3(size), {n[0], n[1], n[2]}};
  return snap(g, load3(p), cell_out);
}

int orc_generate_grid_sdf(const float* v, uint64_t nv, const void* idx, uint64_t ni, int bits, int topo,
                          const float* first, const float* size, const uint64_t* n, int sign, float* out,
                          uint64_t* out_len, int n_threads, uint64_t* stats) {
  if (out_len) *out_len = 0;
  if (sign < 0 || sign > 1) return ST_INVALID_ARGUMENT;
  Mesh m;
  int st = make_mesh(v, nv, idx, ni, bits, topo, &m);
  if (st) return st;
  GridD g{load3(first), load3(size), {n[0], n[1], n[2]}};
  const uint64_t N = n[0] * n[1] * n[2];
  const size_t T = m.size();
  if (N == 0) {
    // A zero cell count panics in the reference's clamp once a triangle is snapped.
    return T ? ST_INVALID_ARGUMENT : ST_OK;
  }
  const int nt = threads_or_all(n_threads);
  const bool raycast = sign == 0;
  std::atomic<uint64_t> st_seed{0}, st_pops{0}, st_cand{0}, st_hits{0};
  std::atomic<int> nan_seen{0};

  // Striped locks stand in for the per-cell RwLock of grid.rs:118-143.
  const size_t NLOCK = 1 << 16;
  std::vector<std::mutex> locks(nt > 1 ? NLOCK : 1);
  auto lock_of = [&](uint64_t c) -> std::mutex& { return locks[nt > 1 ? (c * 0x9E3779B97F4A7C15ull >> 48) : 0]; };

  // ---- generate_preheap (grid.rs:383-457)
  std::vector<float> pre_d(N, F32_MAX);
  std::vector<Tri> pre_t(N, Tri{0, 0, 0});
  auto seed_triangle = [&](size_t t) {
    V3 a = m.a[t], b = m.b[t], c = m.c[t];
    V3 bmn, bmx;
    triangle_bounding_box(a, b, c, &bmn, &bmx);
    uint64_t lo[3], hi[3];
    snap(g, bmn, lo);
    snap(g, bmx, hi);
    V3 lof = g.center(lo[0], lo[1], lo[2]);
    for (int d = 0; d < 3; ++d)
      if (lo[d] > 0 && v_get(lof, d) > v_get(bmn, d)) lo[d] -= 1;
    V3 hif = g.center(hi[0], hi[1], hi[2]);
    for (int d = 0; d < 3; ++d)
      if (hi[d] < g.n[d] - 1 && v_get(hif, d) < v_get(bmx, d)) hi[d] += 1;
    bool nan = false;
    for (uint64_t x = lo[0]; x <= hi[0]; ++x)
      for (uint64_t y = lo[1]; y <= hi[1]; ++y)
        for (uint64_t z = lo[2]; z <= hi[2]; ++z) {
          uint64_t ci = g.idx(x, y, z);
          V3 pos = g.center(x, y, z);
          float d = raycast ? point_triangle_distance(pos, a, b, c) : point_triangle_signed_distance(pos, a, b, c);
          std::lock_guard<std::mutex> lk(lock_of(ci));
          if (compare_distances(d, pre_d[ci], &nan) == -1) {
            pre_d[ci] = d;
            pre_t[ci] = m.tris[t];
            st_seed.fetch_add(1, std::memory_order_relaxed);
          }
        }
    if (nan) nan_seen = 1;
  };
  if (nt > 1) {
#pragma omp parallel for num_threads(nt) schedule(dynamic, 64)
    for (int64_t t = 0; t < (int64_t)T; ++t) seed_triangle((size_t)t);
  } else {
    for (size_t t = 0; t < T; ++t) seed_triangle(t);
  }

  // ---- generate_heap (grid.rs:464-490)
  std::vector<float> dist(N, F32_MAX);
  std::vector<State> heap;
  for (uint64_t ci = 0; ci < N; ++ci) {
    if (pre_d[ci] < F32_MAX) {
      dist[ci] = pre_d[ci];
      State s;
      s.dist = not_nan_or_max(pre_d[ci]);
      s.cell[2] = ci % g.n[2];
      s.cell[1] = (ci / g.n[2]) % g.n[1];
      s.cell[0] = ci / (g.n[1] * g.n[2]);
      s.tri = pre_t[ci];
      heap.push_back(s);
    }
  }
  // sorted_unstable (grid.rs:488).  compare_distances is not transitive inside
  // its tie band, so a merge sort keeps the ordering well-defined in memory.
  std::stable_sort(heap.begin(), heap.end(), StateLess());

  // ---- propagation (grid.rs:318-339, propagate_heap grid.rs:495-558)
  std::vector<std::vector<State>> parts(nt);
  for (size_t i = 0; i < heap.size(); ++i) parts[i % nt].push_back(heap[i]);
  heap.clear();
  heap.shrink_to_fit();
  auto propagate = [&](std::vector<State> init) {
    std::priority_queue<State, std::vector<State>, StateLess> pq(StateLess(), std::move(init));
    bool nan = false;
    uint64_t pops = 0;
    while (!pq.empty()) {
      State s = pq.top();
      pq.pop();
      ++pops;
      V3 a = load3(v + 3 * (size_t)s.tri.i), b = load3(v + 3 * (size_t)s.tri.j), c = load3(v + 3 * (size_t)s.tri.k);
      for (int dx = -1; dx <= 1; ++dx)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dz = -1; dz <= 1; ++dz) {
            int64_t x = (int64_t)s.cell[0] + dx, y = (int64_t)s.cell[1] + dy, z = (int64_t)s.cell[2] + dz;
            if (x < 0 || y < 0 || z < 0 || x >= (int64_t)g.n[0] || y >= (int64_t)g.n[1] || z >= (int64_t)g.n[2])
              continue;
            V3 pos = g.center(x, y, z);
            uint64_t ci = g.idx(x, y, z);
            float d = raycast ? point_triangle_distance(pos, a, b, c) : point_triangle_signed_distance(pos, a, b, c);
            bool push = false;
            {
              std::lock_guard<std::mutex> lk(lock_of(ci));
              if (compare_distances(d, dist[ci], &nan) == -1) {
                dist[ci] = d;
                push = true;
              }
            }
            if (push) {
              State ns;
              ns.dist = not_nan_or_max(d);
              ns.cell[0] = x, ns.cell[1] = y, ns.cell[2] = z;
              ns.tri = s.tri;
              pq.push(ns);
            }
          }
    }
    st_pops.fetch_add(pops);
    if (nan) nan_seen = 1;
  };
  if (nt > 1) {
    std::vector<std::thread> th;
    for (int k = nt - 1; k >= 0; --k) th.emplace_back(propagate, std::move(parts[k]));
    for (auto& t : th) t.join();
  } else {
    propagate(std::move(parts[0]));
  }

  // ---- compute_raycasts (grid.rs:568-642)
  if (raycast && T > 0) {
    CpuBvh bvh;
    bvh.build(m);
    std::vector<std::atomic<uint32_t>> inter(3 * N);
    for (auto& x : inter) x.store(0, std::memory_order_relaxed);
    // generate_raycasts (grid.rs:648-684): X rays from (0,y,z), Y from (x,0,z), Z from (x,y,0).
    struct Ray {
      int axis;
      uint64_t cell[3];
    };
    std::vector<Ray> rays;
    rays.reserve(n[1] * n[2] + n[0] * n[2] + n[0] * n[1]);
    for (uint64_t y = 0; y < n[1]; ++y)
      for (uint64_t z = 0; z < n[2]; ++z) rays.push_back({0, {0, y, z}});
    for (uint64_t x = 0; x < n[0]; ++x)
      for (uint64_t z = 0; z < n[2]; ++z) rays.push_back({1, {x, 0, z}});
    for (uint64_t x = 0; x < n[0]; ++x)
      for (uint64_t y = 0; y < n[1]; ++y) rays.push_back({2, {x, y, 0}});
#pragma omp parallel for num_threads(nt) schedule(dynamic, 64)
    for (int64_t r = 0; r < (int64_t)rays.size(); ++r) {
      const Ray& ray = rays[r];
      V3 o = g.center(ray.cell[0], ray.cell[1], ray.cell[2]);
      const int ax = ray.axis;
      uint64_t hits = 0;
      bvh.ray_hits(m, o, ax, [&](uint32_t, float t) {
        ++hits;
        float cc = t / v_get(g.size, ax);
        uint64_t k = std::min(sat_usize(std::floor(cc)), g.n[ax] - 1);
        uint64_t cell[3] = {ray.cell[0], ray.cell[1], ray.cell[2]};
        for (uint64_t i = 0; i <= k; ++i) {
          cell[ax] = i;
          inter[3 * g.idx(cell[0], cell[1], cell[2]) + ax].fetch_add(1, std::memory_order_relaxed);
        }
      });
      st_hits.fetch_add(hits, std::memory_order_relaxed);
      st_cand.fetch_add(1, std::memory_order_relaxed);
    }
    for (uint64_t ci = 0; ci < N; ++ci) {
      int odd = (inter[3 * ci] & 1) + (inter[3 * ci + 1] & 1) + (inter[3 * ci + 2] & 1);
      if (odd >= 2) dist[ci] = -dist[ci];
    }
  }
  if (stats) {
    stats[0] = st_seed;
    stats[1] = st_pops;
    stats[2] = st_cand;
    stats[3] = st_hits;
  }
  if (nan_seen) return ST_NAN_DISTANCE;
  std::memcpy(out, dist.data(), N * sizeof(float));
  if (out_len) *out_len = N;
  return ST_OK;
}

// ---------------------------------------------------------------------------
// FP64 brute force (error reports only).

namespace {
struct D3 {
  double x, y, z;
};
inline D3 d_sub(D3 a, D3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline D3 d_add(D3 a, D3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline D3 d_mul(D3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double d_dot(D3 a, D3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double d_get(D3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
inline D3 d_load(V3 v) { return {v.x, v.y, v.z}; }

D3 d_seg(D3 p, D3 a, D3 b) {
  D3 ab = d_sub(b, a);
  double m = d_dot(ab, ab);
  double s = m > 0 ? d_dot(ab, d_sub(p, a)) / m : 0.0;
  s = std::min(1.0, std::max(0.0, s));
  return d_add(a, d_mul(ab, s));
}
// Nearest of the three edges: the closest point of a zero-area triangle.
D3 d_closest_edges(D3 p, D3 a, D3 b, D3 c) {
  D3 e[3] = {d_seg(p, a, b), d_seg(p, b, c), d_seg(p, a, c)};
  D3 best = e[0];
  double bd = d_dot(d_sub(p, e[0]), d_sub(p, e[0]));
  for (int k = 1; k < 3; ++k) {
    double dd = d_dot(d_sub(p, e[k]), d_sub(p, e[k]));
    if (dd < bd) bd = dd, best = e[k];
  }
  return best;
}
D3 d_closest(D3 p, D3 a, D3 b, D3 c) {
  D3 ab = d_sub(b, a), ac = d_sub(c, a), ap = d_sub(p, a);
  // A zero-area triangle (repeated or collinear vertices, like a strip's
  // connector windows) is its edges; the region formulas below would divide
  // by zero on it.
  D3 n = {ab.y * ac.z - ab.z * ac.y, ab.z * ac.x - ab.x * ac.z, ab.x * ac.y - ab.y * ac.x};
  if (d_dot(n, n) == 0) return d_closest_edges(p, a, b, c);
  double d1 = d_dot(ab, ap), d2 = d_dot(ac, ap);
  if (d1 <= 0 && d2 <= 0) return a;
  D3 bp = d_sub(p, b);
  double d3 = d_dot(ab, bp), d4 = d_dot(ac, bp);
  if (d3 >= 0 && d4 <= d3) return b;
  D3 cp = d_sub(p, c);
  double d5 = d_dot(ab, cp), d6 = d_dot(ac, cp);
  if (d6 >= 0 && d5 <= d6) return c;
  double vc = d1 * d4 - d3 * d2;
  if (vc <= 0 && d1 >= 0 && d3 <= 0) return d_add(a, d_mul(ab, d1 / (d1 - d3)));
  double vb = d5 * d2 - d1 * d6;
  if (vb <= 0 && d2 >= 0 && d6 <= 0) return d_add(a, d_mul(ac, d2 / (d2 - d6)));
  double va = d3 * d6 - d5 * d4;
  if (va <= 0 && d4 - d3 >= 0 && d5 - d6 >= 0)
    return d_add(b, d_mul(d_sub(c, b), (d4 - d3) / ((d4 - d3) + (d5 - d6))));
  double den = va + vb + vc;
  if (!(den != 0)) return d_closest_edges(p, a, b, c);
  return d_add(d_add(a, d_mul(ab, vb / den)), d_mul(ac, vc / den));
}
bool d_ray(D3 o, D3 t0, D3 t1, D3 t2, int axis) {
  const int ix = axis, iy = (axis + 1) % 3, iz = (axis + 2) % 3;
  D3 e01 = d_sub(t1, t0), e12 = d_sub(t2, t1), e20 = d_sub(t0, t2);
  D3 p0 = d_sub(o, t0), p1 = d_sub(o, t1), p2 = d_sub(o, t2);
  double w0 = d_get(p1, iz) * d_get(e12, iy) - d_get(p1, iy) * d_get(e12, iz);
  double w1 = d_get(p2, iz) * d_get(e20, iy) - d_get(p2, iy) * d_get(e20, iz);
  double w2 = d_get(p0, iz) * d_get(e01, iy) - d_get(p0, iy) * d_get(e01, iz);
  if ((w0 < 0 && w1 < 0 && w2 < 0) || (w0 > 0 && w1 > 0 && w2 > 0)) {
    double t = -(w0 * d_get(p0, ix) + w2 * d_get(p2, ix) + w1 * d_get(p1, ix)) / (w0 + w1 + w2);
    return t > 0;
  }
  return false;
}
}  // namespace

int orc_generate_sdf_f64(const float* v, uint64_t nv, const void* idx, uint64_t ni, int bits, int topo,
                         const float* q, uint64_t nq, double* out_unsigned, uint8_t* out_inside, int n_threads) {
  Mesh m;
  int st = make_mesh(v, nv, idx, ni, bits, topo, &m);
  if (st) return st;
  const size_t T = m.size();
  CpuBvh bvh;
  bvh.build(m);
  const int nt = threads_or_all(n_threads);
#pragma omp parallel for num_threads(nt) schedule(dynamic, 16)
  for (int64_t i = 0; i < (int64_t)nq; ++i) {
    V3 pf = load3(q + 3 * i);
    D3 p = d_load(pf);
    // Start from the f32 nearest and scan every triangle whose box could beat it.
    double best = std::numeric_limits<double>::infinity();
    if (T) {
      float d2f;
      long t0 = bvh.nearest(m, pf, &d2f);
      D3 cp = d_closest(p, d_load(m.a[t0]), d_load(m.b[t0]), d_load(m.c[t0]));
      best = std::sqrt(d_dot(d_sub(p, cp), d_sub(p, cp)));
      std::vector<uint32_t> cand;
      bvh.within(pf, best * (1 + 1e-6) + 2e-4, &cand);
      for (uint32_t t : cand) {
        D3 c2 = d_closest(p, d_load(m.a[t]), d_load(m.b[t]), d_load(m.c[t]));
        best = std::min(best, std::sqrt(d_dot(d_sub(p, c2), d_sub(p, c2))));
      }
    }
    out_unsigned[i] = best;
    int insides = 0;
    for (int axis = 0; axis < 3; ++axis) {
      uint32_t cnt = 0;
      // Every triangle whose padded box the ray meets is decided in double.
      const int iy = (axis + 1) % 3, iz = (axis + 2) % 3;
      for (size_t t = 0; t < T; ++t) {
        const double* lo = &bvh.tlo[3 * t];
        const double* hi = &bvh.thi[3 * t];
        double oy = v_get(pf, iy), oz = v_get(pf, iz);
        if (oy < lo[iy] || oy > hi[iy] || oz < lo[iz] || oz > hi[iz] || hi[axis] < v_get(pf, axis)) continue;
        if (d_ray(p, d_load(m.a[t]), d_load(m.b[t]), d_load(m.c[t]), axis)) ++cnt;
      }
      if (cnt % 2 == 1) ++insides;
    }
    out_inside[i] = insides > 1 ? 1 : 0;
  }
  return ST_OK;
}

// check_mesh_triangle_list (generate/mesh_check.rs:24-81), restated step by
// step.  The crate compares vertices by their `{:?}` text, which is the same
// as comparing the f32 bit patterns except that every NaN prints "NaN": the
// key below merges the NaNs.  Faces compare as ordered index triples.  The
// edge loop is the crate's: pop the last edge, fail if another copy remains
// or if its reverse is missing, drop every copy of the reverse.
// kind: 0 ok, 1 length not a multiple of 3, 2 duplicate vertex (detail[0] =
// vertex index), 3 duplicate face (detail[0] = face index), 4 duplicate edge,
// 5 edge without its reverse (detail = from, to).
int orc_check_mesh_triangle_list(const float* vertices, uint64_t nv, const uint32_t* faces, uint64_t n_idx,
                                 int* kind, uint64_t* detail) {
  detail[0] = detail[1] = 0;
  if (n_idx % 3 != 0) {
    *kind = 1;
    return ST_OK;
  }
  auto vkey = [&](uint64_t i, int d) {
    float f = vertices[3 * i + d];
    uint32_t b;
    std::memcpy(&b, &f, 4);
    return std::isnan(f) ? 0x7FC00000u : b;
  };
  {
    std::set<std::array<uint32_t, 3>> seen;
    for (uint64_t i = 0; i < nv; ++i) {
      if (!seen.insert({vkey(i, 0), vkey(i, 1), vkey(i, 2)}).second) {
        *kind = 2;
        detail[0] = i;
        return ST_OK;
      }
    }
  }
  const uint64_t F = n_idx / 3;
  {
    std::set<std::array<uint32_t, 3>> seen;
    for (uint64_t f = 0; f < F; ++f) {
      if (!seen.insert({faces[3 * f], faces[3 * f + 1], faces[3 * f + 2]}).second) {
        *kind = 3;
        detail[0] = f;
        return ST_OK;
      }
    }
  }
  std::vector<std::pair<uint32_t, uint32_t>> edges;
  edges.reserve(3 * F);
  for (uint64_t f = 0; f < F; ++f) {
    const uint32_t* t = faces + 3 * f;
    edges.push_back({t[0], t[1]});
    edges.push_back({t[1], t[2]});
    edges.push_back({t[2], t[0]});
  }
  while (!edges.empty()) {
    const auto e = edges.back();
    edges.pop_back();
    const std::pair<uint32_t, uint32_t> opp{e.second, e.first};
    if (std::count(edges.begin(), edges.end(), e) > 0) {
      *kind = 4;
      detail[0] = e.first;
      detail[1] = e.second;
      return ST_OK;
    }
    if (std::find(edges.begin(), edges.end(), opp) == edges.end()) {
      *kind = 5;
      detail[0] = e.first;
      detail[1] = e.second;
      return ST_OK;
    }
    edges.erase(std::remove(edges.begin(), edges.end(), opp), edges.end());
  }
  *kind = 0;
  return ST_OK;
}

}  // extern "C"
