// Point queries: generate_sdf / query_sdf for every AccelerationMethod.
//
//  * None  (generate/generic/default.rs:22-85): k_brute — every query against
//    every triangle.  Triangle tiles are staged in shared memory by the bulk
//    copy engine (cp.async.bulk + mbarrier, double-buffered); each thread owns
//    one query and folds the tile in triangle order, exactly the reference's
//    fold order; batches of 2^28 pairs or more are visited in Morton order.
//    Normal batches of fewer than 2^17 queries take k_brute_normal_warp: a
//    warp per query, the same fold in the same order.
//  * Bvh(Raycast) / RtreeBvh (bvh.rs:104-180, rtree_bvh.rs:143-201): exact
//    nearest triangle on the LBVH, then the 3-axis ray vote.
//  * Rtree (rtree.rs:137-157): the nearest triangle's signed distance.
//  * Bvh(Normal) (bvh.rs:117-129): compare_distances folded over the near-tie
//    band of the nearest distance, in triangle order.
//  * query_vector_to_closest_point_rtree_bvh (rtree_bvh.rs:217-276).
#include <cuda_runtime.h>

#include <type_traits>

#include <algorithm>
#include <cfloat>

#include "m2s_audit.cuh"
#include "m2s_internal.cuh"
#include "m2s_tma.cuh"

namespace m2s {
namespace {

constexpr float F32_MAX = 3.40282347e+38f;

__device__ __forceinline__ P3 load_query(const float* q, uint64_t i) { return {q[3 * i], q[3 * i + 1], q[3 * i + 2]}; }

// ---------------------------------------------------------------------------
// K1: brute force over all triangles (AccelerationMethod::None).
constexpr int kBfThreads = 128;
constexpr int kBfTile = 256;  // triangles per stage: 256 * 48 B = 12 KiB

// Raycast splits the triangle range into gridDim.y chunks (min and hit parity
// commute): each chunk folds its part and merges into `part` (atomicMin on the
// squared distance bits, atomicXor on the parity).  Normal folds all
// triangles in order in one chunk (compare_distances ties depend on order).
//
// Raycast: a triangle whose plane bound (tri_plane in m2s_geo.cuh) exceeds
// the query's best distance so far cannot lower the minimum, so its closest
// point is not evaluated; its +X ray test always is (the parity counts every
// triangle).  Rust's f32::min ignores a NaN distance (default.rs:58), so a
// skipped triangle changes nothing even then.  The planes of a tile are
// formed in shared memory as it lands.
template <int SIGN>
__global__ void __launch_bounds__(kBfThreads) k_brute(const TriRec* __restrict__ tris, uint32_t T,
                                                      const float* __restrict__ q, uint64_t nq,
                                                      float* __restrict__ out, uint32_t* status,
                                                      uint2* __restrict__ part, const uint32_t* __restrict__ order) {
  __shared__ __align__(128) TriRec tile[2][kBfTile];
  __shared__ __align__(16) float4 plane_n[2][SIGN == 0 ? kBfTile : 1];  // TriPlane::n
  __shared__ float plane_s[2][SIGN == 0 ? kBfTile : 1];                  // TriPlane::slack
  __shared__ __align__(8) uint64_t bar[2];
  const int tid = threadIdx.x;
  const uint64_t k = (uint64_t)blockIdx.x * kBfThreads + tid;
  const bool valid = k < nq;
  const uint64_t qi = valid && order ? order[k] : k;  // Morton order: a warp's queries share region branches
  const P3 p = valid ? load_query(q, qi) : P3{0.0f, 0.0f, 0.0f};
  // this block's chunk of triangles: whole tiles [t_begin, t_end)
  const uint32_t all_tiles = (T + kBfTile - 1) / kBfTile;
  const uint32_t per = (all_tiles + gridDim.y - 1) / gridDim.y;
  const uint32_t t_begin = min(all_tiles, blockIdx.y * per), t_end = min(all_tiles, t_begin + per);
  const uint32_t ntile = t_end - t_begin;
  tris += (uint64_t)t_begin * kBfTile;
  T = ntile == 0 ? 0u : (t_end == all_tiles ? T - t_begin * kBfTile : ntile * kBfTile);

  if (tid == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_barrier_init();
  }
  __syncthreads();
  auto issue = [&](uint32_t i) {
    uint32_t cnt = min((uint32_t)kBfTile, T - i * kBfTile);
    uint32_t bytes = cnt * (uint32_t)sizeof(TriRec);
    mbar_arrive_expect_tx(&bar[i & 1], bytes);
    bulk_g2s(&tile[i & 1][0], tris + (uint64_t)i * kBfTile, bytes, &bar[i & 1]);
  };
  if (tid == 0) {
    if (ntile > 0) issue(0);
    if (ntile > 1) issue(1);
  }

  float best = SIGN == 0 ? INFINITY : F32_MAX;  // Raycast keeps the squared distance
  float reach = INFINITY;                         // Normal: fold_reach(|best|)
  // Raycast: a triangle's plane bound must exceed `above` to skip it;
  // `pslack` is the query's share of the bound's slack.
  float above = INFINITY;
  const float pslack = plane_query_slack(p);
  uint32_t hits = 0;
  bool nan = false, lost = false;
  for (uint32_t i = 0; i < ntile; ++i) {
    const int buf = i & 1;
    if (!mbar_wait_bounded(&bar[buf], (i >> 1) & 1)) lost = true;
    const uint32_t cnt = min((uint32_t)kBfTile, T - i * kBfTile);
    const TriRec* tl = tile[buf];
    if (SIGN == 0) {
      lost = __syncthreads_or(lost);  // the planes are only formed from a tile every thread has
      if (!lost)
        for (uint32_t j = tid; j < cnt; j += kBfThreads) {
          const TriPlane pl = tri_plane(p3(tl[j].a), p3(tl[j].b), p3(tl[j].c), __float_as_int(tl[j].a.w));
          plane_n[buf][j] = pl.n;
          plane_s[buf][j] = pl.slack;
        }
      __syncthreads();
    }
    if (!lost) {
#pragma unroll 2
      for (uint32_t j = 0; j < cnt; ++j) {
        const float4 ra = tl[j].a, rb = tl[j].b, rc = tl[j].c;
        const P3 a = p3(ra), b = p3(rb), c = p3(rc);
        const int kind = __float_as_int(ra.w);
        if (SIGN == 0) {
          // default.rs:45-49 then :59-62 — min of distances, count of +X hits.
          if (!(plane_bound(plane_n[buf][SIGN == 0 ? j : 0], plane_s[buf][SIGN == 0 ? j : 0], p, pslack) > above)) {
            const float d2 = point_triangle_distance2(p, a, b, c, kind);
            if (d2 < best) {  // fminf: a NaN distance is ignored
              best = d2;
              above = plane_above(best);
            }
          }
          float t;
          hits += ray_hit_aligned<0>(p, a, b, c, &t) ? 1u : 0u;
        } else {
          // default.rs:51-53 then :63-70 — compare_distances fold; a d
          // beyond the fold's reach cannot be before best.
          float d = point_triangle_signed_distance(p, a, b, c, kind);
          if (!(fabsf(d) > reach) && compare_distances(d, best, &nan) == -1) {
            best = d;
            reach = fold_reach(fabsf(best));
          }
        }
      }
    }
    __syncthreads();
    if (tid == 0 && i + 2 < ntile) {
      fence_proxy_async_smem();
      issue(i + 2);
    }
  }
  if (lost) atomicOr(status, bit(M2S_ERR_LIMIT));
  if (nan) atomicOr(status, bit(M2S_ERR_NAN_DISTANCE));
  if (!valid) return;
  if (SIGN == 0 && part) {
    atomicMin(&part[qi].x, __float_as_uint(best));  // non-negative floats order like their bits
    if (hits & 1u) atomicXor(&part[qi].y, 1u);
    return;
  }
  float r;
  if (SIGN == 0) {
    // sqrt(min d2) == min sqrt(d2) (IEEE sqrt is monotone); f32::MAX start value.
    float d = fminf(F32_MAX, fsqrt(best));
    r = (hits & 1u) ? -d : d;
  } else {
    r = best;
  }
  out[qi] = r;
}

__global__ void k_brute_init(uint2* part, uint64_t nq) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += (uint64_t)gridDim.x * blockDim.x)
    part[i] = make_uint2(0x7F800000u, 0u);  // +inf, even
}

__global__ void k_brute_finish(const uint2* __restrict__ part, uint64_t nq, float* __restrict__ out) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += (uint64_t)gridDim.x * blockDim.x) {
    const uint2 pp = part[i];
    const float d = fminf(F32_MAX, fsqrt(__uint_as_float(pp.x)));
    out[i] = pp.y ? -d : d;
  }
}

// Normal sign, one warp per query: lane k evaluates triangle t0 + k of each
// group of 32, then the warp folds the group's distances into `best` in
// triangle order — the first lane whose distance compare_distances puts
// before `best` replaces it, and only the lanes after it are tested again,
// against the new value, until none is before it.  That is the reference's
// sequential fold (default.rs:63-70) step for step, with 32 triangles
// evaluated at a time, so a batch of few queries still fills the GPU.  Lanes
// whose |d| lies beyond fold_reach of the group's first best cannot be
// before any value the group's fold takes and are left out at once; most
// groups then need no compare_distances at all.
constexpr int kBwThreads = 256;                 // 8 queries per block
constexpr uint64_t kBruteWarpMaxQueries = 1u << 17;  // below: one warp per query
constexpr uint64_t kBruteSortMinPairs = 1ull << 28;  // from here the thread kernels visit queries in Morton order
__global__ void __launch_bounds__(kBwThreads) k_brute_normal_warp(const TriRec* __restrict__ tris, uint32_t T,
                                                                  const float* __restrict__ q, uint64_t nq,
                                                                  float* __restrict__ out, uint32_t* status) {
  __shared__ __align__(128) TriRec tile[2][kBfTile];
  __shared__ __align__(8) uint64_t bar[2];
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t qi = (uint64_t)blockIdx.x * (kBwThreads / 32) + (threadIdx.x >> 5);
  const bool valid = qi < nq;  // warp-uniform
  const P3 p = valid ? load_query(q, qi) : P3{0.0f, 0.0f, 0.0f};
  const uint32_t ntile = (T + kBfTile - 1) / kBfTile;
  if (threadIdx.x == 0) {
    mbar_init(&bar[0], 1);
    mbar_init(&bar[1], 1);
    fence_barrier_init();
  }
  __syncthreads();
  auto issue = [&](uint32_t i) {
    uint32_t cnt = min((uint32_t)kBfTile, T - i * kBfTile);
    uint32_t bytes = cnt * (uint32_t)sizeof(TriRec);
    mbar_arrive_expect_tx(&bar[i & 1], bytes);
    bulk_g2s(&tile[i & 1][0], tris + (uint64_t)i * kBfTile, bytes, &bar[i & 1]);
  };
  if (threadIdx.x == 0) {
    if (ntile > 0) issue(0);
    if (ntile > 1) issue(1);
  }
  float best = F32_MAX;
  bool nan = false, lost = false;
  for (uint32_t i = 0; i < ntile; ++i) {
    const int buf = i & 1;
    if (!mbar_wait_bounded(&bar[buf], (i >> 1) & 1)) lost = true;
    const uint32_t cnt = min((uint32_t)kBfTile, T - i * kBfTile);
    const TriRec* tl = tile[buf];
    if (valid && !__any_sync(0xFFFFFFFFu, lost)) {
      for (uint32_t j0 = 0; j0 < cnt; j0 += 32u) {
        const uint32_t j = j0 + lane;
        const bool have = j < cnt;
        float d = 0.0f;
        if (have) {
          const float4 ra = tl[j].a, rb = tl[j].b, rc = tl[j].c;
          d = point_triangle_signed_distance(p, p3(ra), p3(rb), p3(rc), __float_as_int(ra.w));
        }
        // lanes not folded yet; none beyond the reach of the group's first best
        uint32_t todo = __ballot_sync(0xFFFFFFFFu, have && !(fabsf(d) > fold_reach(fabsf(best))));
        while (todo) {
          const bool before = ((todo >> lane) & 1u) && compare_distances(d, best, &nan) == -1;
          const uint32_t m = __ballot_sync(0xFFFFFFFFu, before);
          if (!m) break;
          const int w = __ffs(m) - 1;
          best = __shfl_sync(0xFFFFFFFFu, d, w);
          todo &= ~((2u << w) - 1u);  // lanes up to w are folded (w = 31 clears all)
        }
      }
    }
    __syncthreads();
    if (threadIdx.x == 0 && i + 2 < ntile) {
      fence_proxy_async_smem();
      issue(i + 2);
    }
  }
  if (lost) atomicOr(status, bit(M2S_ERR_LIMIT));
  if (nan) atomicOr(status, bit(M2S_ERR_NAN_DISTANCE));
  if (valid && lane == 0) out[qi] = best;
}

// ---------------------------------------------------------------------------
// LBVH traversals.
constexpr int kStack = 64;

__device__ __forceinline__ float box_dist2(P3 p, float4 lo, float4 hi) {
  float dx = fmaxf(fmaxf(lo.x - p.x, p.x - hi.x), 0.0f);
  float dy = fmaxf(fmaxf(lo.y - p.y, p.y - hi.y), 0.0f);
  float dz = fmaxf(fmaxf(lo.z - p.z, p.z - hi.z), 0.0f);
  return dx * dx + dy * dy + dz * dz;
}

__device__ __forceinline__ BvhNode load_node(const BvhNode* nodes, uint32_t i) {
  const float4* f = reinterpret_cast<const float4*>(nodes + i);
  BvhNode n;
  n.l_lo = __ldg(f);
  n.l_hi = __ldg(f + 1);
  n.r_lo = __ldg(f + 2);
  n.r_hi = __ldg(f + 3);
  return n;
}

__device__ __forceinline__ TriRec load_tri(const TriRec* t, uint32_t i) {
  const float4* f = reinterpret_cast<const float4*>(t + i);
  return {__ldg(f), __ldg(f + 1), __ldg(f + 2)};
}

struct Nearest {
  float d2;
  uint32_t tri;   // crate triangle index
  uint32_t leaf;  // LBVH leaf position
};

// Traversal counts of one query, kept only by the STATS instantiations
// (profiling): nearest-triangle search node fetches and triangle tests, and
// the same for the sign step (the three axis rays, or the Normal tie band).
struct QCount {
  uint32_t visits = 0, tests = 0, sign_visits = 0, sign_tests = 0;
  // FP64 audit (m2s_audit.cuh): ray tests, ambiguous, FP64 decides
  // otherwise; whether the FP64 decisions flip the query's vote; whether its
  // nearest triangle's region was audited, ambiguous, FP64 picks another.
  uint32_t ray_tests = 0, ray_ambiguous = 0, ray_disagree = 0, vote_flip = 0, region = 0, region_ambiguous = 0,
           region_disagree = 0;
};
constexpr int kQueryCounters = 11;

// Exact nearest triangle under the f32 point_triangle_distance2 (geo.rs:33-37),
// ties to the lowest triangle index.  Boxes are padded by 1e-4 (geo.rs:4-22),
// which keeps the f32 box test conservative.  Starts from `best` (an upper
// bound from an earlier, unfinished search, or +inf).  With a budget, the
// search gives up after `budget` node visits and clears *finished; `best` is
// then still a valid upper bound for a second pass.
template <bool STATS = false>
__device__ Nearest nearest_triangle(const MeshView& m, P3 p, bool* overflow, Nearest best = {INFINITY, 0xFFFFFFFFu, 0},
                                    uint32_t budget = 0xFFFFFFFFu, bool* finished = nullptr, QCount* qc = nullptr) {
  auto eval = [&](uint32_t leaf) {
    if constexpr (STATS) ++qc->tests;
    TriRec r = load_tri(m.stris, leaf);
    float d2 = point_triangle_distance2(p, p3(r.a), p3(r.b), p3(r.c), __float_as_int(r.a.w));
    uint32_t idx = __float_as_uint(r.b.w);
    if (d2 < best.d2 || (d2 == best.d2 && idx < best.tri)) best = {d2, idx, leaf};
  };
  if (finished) *finished = true;
  if (m.root & LEAF_BIT) {
    eval(m.root & ~LEAF_BIT);
    return best;
  }
  uint32_t st_node[kStack];
  float st_dist[kStack];
  int sp = 0;
  uint32_t node = 0;
  uint32_t visits = 0;
  while (true) {
    if (++visits > budget) {
      *finished = false;
      break;
    }
    if constexpr (STATS) ++qc->visits;
    BvhNode nd = load_node(m.nodes, node);
    float dl = box_dist2(p, nd.l_lo, nd.l_hi), dr = box_dist2(p, nd.r_lo, nd.r_hi);
    uint32_t L = __float_as_uint(nd.l_lo.w), R = __float_as_uint(nd.l_hi.w);
    bool goL = dl <= best.d2, goR = dr <= best.d2;
    if (goL && (L & LEAF_BIT)) {
      eval(L & ~LEAF_BIT);
      goL = false;
    }
    if (goR && (R & LEAF_BIT)) {
      eval(R & ~LEAF_BIT);
      goR = false;
    }
    goL = goL && dl <= best.d2;
    goR = goR && dr <= best.d2;
    if (goL && goR) {
      bool lfirst = dl <= dr;
      if (sp < kStack) {
        st_node[sp] = lfirst ? R : L;
        st_dist[sp] = lfirst ? dr : dl;
        ++sp;
      } else {
        *overflow = true;
      }
      node = lfirst ? L : R;
      continue;
    }
    if (goL) {
      node = L;
      continue;
    }
    if (goR) {
      node = R;
      continue;
    }
    bool found = false;
    while (sp > 0) {
      --sp;
      if (st_dist[sp] <= best.d2) {
        node = st_node[sp];
        found = true;
        break;
      }
    }
    if (!found) break;
  }
  return best;
}

// The same search for the 32 queries of a warp at once (Morton-adjacent
// queries reach mostly the same nodes): the warp walks one node sequence,
// every node fetched once for all lanes, and each lane takes a node only
// while its own box distance is within its own best; the order of the two
// children follows the majority of lanes.  A lane's result is the one the
// single-thread search gives (exhaustive under its own bound, ties to the
// lowest triangle index); `budget` counts the nodes a lane took, and a lane
// over it stops taking nodes and clears *finished.
template <bool STATS = false>
__device__ Nearest nearest_triangle_packet(const MeshView& m, P3 p, bool active, bool* overflow, uint32_t budget,
                                           bool* finished, QCount* qc = nullptr) {
  Nearest best{INFINITY, 0xFFFFFFFFu, 0};
  auto eval = [&](uint32_t leaf) {
    if constexpr (STATS) ++qc->tests;
    TriRec r = load_tri(m.stris, leaf);
    float d2 = point_triangle_distance2(p, p3(r.a), p3(r.b), p3(r.c), __float_as_int(r.a.w));
    uint32_t idx = __float_as_uint(r.b.w);
    if (d2 < best.d2 || (d2 == best.d2 && idx < best.tri)) best = {d2, idx, leaf};
  };
  *finished = true;
  bool live = active;  // still taking nodes
  if (m.root & LEAF_BIT) {
    if (live) eval(m.root & ~LEAF_BIT);
    return best;
  }
  uint32_t st_node[kStack];
  float st_dist[kStack];
  int sp = 0;
  uint32_t node = 0;
  uint32_t visits = 0;
  bool take = live;  // this lane wants `node`
  while (true) {
    if (take) {
      if (++visits > budget) {
        *finished = false;
        live = false;
      } else if constexpr (STATS) {
        ++qc->visits;
      }
    }
    take = take && live;
    if (__any_sync(0xFFFFFFFFu, take)) {
      BvhNode nd = load_node(m.nodes, node);
      float dl = box_dist2(p, nd.l_lo, nd.l_hi), dr = box_dist2(p, nd.r_lo, nd.r_hi);
      uint32_t L = __float_as_uint(nd.l_lo.w), R = __float_as_uint(nd.l_hi.w);
      bool goL = take && dl <= best.d2, goR = take && dr <= best.d2;
      if (L & LEAF_BIT) {
        if (goL) eval(L & ~LEAF_BIT);
        goL = false;
      }
      if (R & LEAF_BIT) {
        if (goR) eval(R & ~LEAF_BIT);
        goR = false;
      }
      goL = goL && dl <= best.d2;
      goR = goR && dr <= best.d2;
      const bool anyL = __any_sync(0xFFFFFFFFu, goL), anyR = __any_sync(0xFFFFFFFFu, goR);
      if (anyL && anyR) {
        const uint32_t nl = __popc(__ballot_sync(0xFFFFFFFFu, goL && (!goR || dl <= dr)));
        const uint32_t nr = __popc(__ballot_sync(0xFFFFFFFFu, goR && (!goL || dr < dl)));
        const bool lfirst = nl >= nr;
        if (sp < kStack) {
          st_node[sp] = lfirst ? R : L;
          st_dist[sp] = (lfirst ? goR : goL) ? (lfirst ? dr : dl) : INFINITY;
          ++sp;
        } else if (lfirst ? goR : goL) {
          *overflow = true;
        }
        node = lfirst ? L : R;
        take = lfirst ? goL : goR;
        continue;
      }
      if (anyL || anyR) {
        node = anyL ? L : R;
        take = anyL ? goL : goR;
        continue;
      }
    }
    // pop the next entry some lane still wants
    bool found = false;
    while (sp > 0) {
      --sp;
      const bool want = live && st_dist[sp] <= best.d2;
      if (__any_sync(0xFFFFFFFFu, want)) {
        node = st_node[sp];
        take = want;
        found = true;
        break;
      }
    }
    if (!found) break;
  }
  return best;
}

// (d2, triangle) packed so that the unsigned order is the search order.
__device__ __forceinline__ unsigned long long nn_key(float d2, uint32_t tri) {
  return ((unsigned long long)__float_as_uint(d2) << 32) | tri;
}
__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
  for (int o = 16; o; o >>= 1) {
    unsigned long long w = __shfl_xor_sync(0xFFFFFFFFu, v, o);
    v = w < v ? w : v;
  }
  return v;
}

// One warp per query: the 32 lanes pop the 32 top entries of a shared-memory
// stack of (node, box distance), test both children of each, evaluate child
// leaves in parallel and share the running best through a warp minimum.  Used
// for the queries whose single-thread search ran over its node budget (points
// deep inside a closed mesh, where many triangles are nearly equidistant).
// Returns false if the stack would overflow (the caller then finishes the
// search on one lane).  512 entries (4 KB a warp): the warp pass's blocks are
// bound by shared memory, and 2048 entries left room for 12 warps per SM
// against 56 now (star s6, mixed points, warp pass 1.67 -> 1.14 ms at
// 100,000 Rtree queries; whole queries 16,384 to 400,000 points 18-27 %
// faster; results bit-identical, the rare overflow finishing on one lane).
constexpr int kWarpStack = 512;

template <bool STATS = false, int CAP = kWarpStack>
__device__ bool nearest_triangle_warp(const MeshView& m, P3 p, Nearest* io, uint32_t* s_node, float* s_dist,
                                      QCount* qc = nullptr) {
  const int lane = threadIdx.x & 31;
  // Non-negative d2 (or +inf / NaN-free boxes) order like their bits.
  unsigned long long best = nn_key(io->d2, io->tri);
  uint32_t best_leaf = io->leaf;
  int sp = 0;
  if (lane == 0) {
    s_node[0] = 0;
    s_dist[0] = 0.0f;
  }
  sp = 1;
  __syncwarp();
  while (sp > 0) {
    const int take = min(sp, 32);
    const int base = sp - take;
    uint32_t node = 0xFFFFFFFFu;
    float nd2 = INFINITY;
    if (lane < take) {
      node = s_node[base + lane];
      nd2 = s_dist[base + lane];
    }
    __syncwarp();
    sp = base;
    const float bound = __uint_as_float((uint32_t)(best >> 32));
    uint32_t push_ref[2] = {0, 0};
    float push_d[2] = {0.0f, 0.0f};
    int npush = 0;
    unsigned long long cand = ~0ull;
    uint32_t cand_leaf = 0;
    if (node != 0xFFFFFFFFu && nd2 <= bound) {
      if constexpr (STATS) ++qc->visits;
      BvhNode nd = load_node(m.nodes, node);
      const uint32_t ch[2] = {__float_as_uint(nd.l_lo.w), __float_as_uint(nd.l_hi.w)};
      const float cd[2] = {box_dist2(p, nd.l_lo, nd.l_hi), box_dist2(p, nd.r_lo, nd.r_hi)};
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        if (!(cd[c] <= bound)) continue;
        if (ch[c] & LEAF_BIT) {
          const uint32_t leaf = ch[c] & ~LEAF_BIT;
          if constexpr (STATS) ++qc->tests;
          TriRec r = load_tri(m.stris, leaf);
          float d2 = point_triangle_distance2(p, p3(r.a), p3(r.b), p3(r.c), __float_as_int(r.a.w));
          if (!(d2 <= d2)) continue;  // NaN distances never win
          unsigned long long k = nn_key(d2, __float_as_uint(r.b.w));
          if (k < cand) {
            cand = k;
            cand_leaf = leaf;
          }
        } else {
          push_ref[npush] = ch[c];
          push_d[npush] = cd[c];
          ++npush;
        }
      }
    }
    // share the best of this step
    const unsigned long long wmin = warp_min_u64(cand);
    if (wmin < best) {
      const uint32_t who = __ffs(__ballot_sync(0xFFFFFFFFu, cand == wmin)) - 1;
      best_leaf = __shfl_sync(0xFFFFFFFFu, cand_leaf, who);
      best = wmin;
    }
    // push surviving children (deepest first: they go on top)
    const float nb = __uint_as_float((uint32_t)(best >> 32));
    int keep = 0;
    for (int c = 0; c < npush; ++c) keep += push_d[c] <= nb ? 1 : 0;
    int incl = keep;
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= o) incl += y;
    }
    const int total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    if (sp + total > CAP) return false;
    int pos = sp + incl - keep;
    for (int c = 0; c < npush; ++c)
      if (push_d[c] <= nb) {
        s_node[pos] = push_ref[c];
        s_dist[pos] = push_d[c];
        ++pos;
      }
    sp += total;
    __syncwarp();
  }
  io->d2 = __uint_as_float((uint32_t)(best >> 32));
  io->tri = (uint32_t)best;
  io->leaf = best_leaf;
  return true;
}

// Number of triangles the +AXIS ray from o crosses (geo.rs:165-216).  A box is
// entered when the ray's (y, z) lies inside it and its far side is ahead of o.
// The counting (STATS) instantiation also audits every ray test and counts
// the crossings the FP64 decisions give in *count64.
template <int AXIS, bool STATS = false>
__device__ uint32_t ray_crossings(const MeshView& m, P3 o, bool* overflow, QCount* qc = nullptr,
                                  uint32_t* count64 = nullptr) {
  constexpr int IY = (AXIS + 1) % 3, IZ = (AXIS + 2) % 3;
  const float oy = vget(o, IY), oz = vget(o, IZ), ox = vget(o, AXIS);
  uint32_t count = 0;
  auto test = [&](uint32_t leaf) {
    TriRec r = load_tri(m.stris, leaf);
    if constexpr (STATS) {
      ++qc->sign_tests;
      const RayAudit ra = ray_audit<AXIS>(o, p3(r.a), p3(r.b), p3(r.c));
      ++qc->ray_tests;
      qc->ray_ambiguous += ra.ambiguous;
      qc->ray_disagree += ra.hit64 != ra.hit32;
      count += ra.hit32 ? 1u : 0u;
      *count64 += ra.hit64 ? 1u : 0u;
    } else {
      float t;
      count += ray_hit_aligned<AXIS>(o, p3(r.a), p3(r.b), p3(r.c), &t) ? 1u : 0u;
    }
  };
  auto inside = [&](float4 lo, float4 hi) {
    float loy = IY == 0 ? lo.x : (IY == 1 ? lo.y : lo.z), hiy = IY == 0 ? hi.x : (IY == 1 ? hi.y : hi.z);
    float loz = IZ == 0 ? lo.x : (IZ == 1 ? lo.y : lo.z), hiz = IZ == 0 ? hi.x : (IZ == 1 ? hi.y : hi.z);
    float hix = AXIS == 0 ? hi.x : (AXIS == 1 ? hi.y : hi.z);
    return oy >= loy && oy <= hiy && oz >= loz && oz <= hiz && hix >= ox;
  };
  if (m.root & LEAF_BIT) {
    test(m.root & ~LEAF_BIT);
    return count;
  }
  uint32_t stack[kStack];
  int sp = 0;
  uint32_t node = 0;
  while (true) {
    if constexpr (STATS) ++qc->sign_visits;
    BvhNode nd = load_node(m.nodes, node);
    uint32_t L = __float_as_uint(nd.l_lo.w), R = __float_as_uint(nd.l_hi.w);
    bool goL = inside(nd.l_lo, nd.l_hi), goR = inside(nd.r_lo, nd.r_hi);
    if (goL && (L & LEAF_BIT)) {
      test(L & ~LEAF_BIT);
      goL = false;
    }
    if (goR && (R & LEAF_BIT)) {
      test(R & ~LEAF_BIT);
      goR = false;
    }
    if (goL && goR) {
      if (sp < kStack) stack[sp++] = R;
      else *overflow = true;
      node = L;
      continue;
    }
    if (goL) {
      node = L;
      continue;
    }
    if (goR) {
      node = R;
      continue;
    }
    if (sp == 0) break;
    node = stack[--sp];
  }
  return count;
}

// bvh.rs:293-328 / rtree_bvh.rs:163-199: inside when >= 2 of 3 axis rays are odd.
template <bool STATS = false>
__device__ __forceinline__ bool vote_inside(const MeshView& m, P3 p, bool* overflow, QCount* qc = nullptr) {
  uint32_t c64[3] = {0u, 0u, 0u};
  int insides = (ray_crossings<0, STATS>(m, p, overflow, qc, &c64[0]) & 1u) +
                (ray_crossings<1, STATS>(m, p, overflow, qc, &c64[1]) & 1u) +
                (ray_crossings<2, STATS>(m, p, overflow, qc, &c64[2]) & 1u);
  if constexpr (STATS) {
    const int insides64 = (c64[0] & 1u) + (c64[1] & 1u) + (c64[2] & 1u);
    qc->vote_flip += (insides > 1) != (insides64 > 1);
  }
  return insides > 1;
}

// The +AXIS ray's crossings from o counted by a whole warp (one query): the
// lanes pop up to 32 nodes of a shared stack, test both children's boxes as
// ray_crossings does, test child leaves with the aligned ray test and push
// child nodes.  Every leaf the box test admits is tested exactly once, so the
// count (and *count64, the FP64 audit's count, in the counting instantiation)
// is the single-thread one.  Returns false if the stack would overflow.
template <int AXIS, int CAP, bool STATS = false>
__device__ bool ray_crossings_warp(const MeshView& m, P3 o, uint32_t* s_stack, uint32_t* count_out, QCount* qc,
                                   uint32_t* count64_out) {
  constexpr int IY = (AXIS + 1) % 3, IZ = (AXIS + 2) % 3;
  const int lane = threadIdx.x & 31;
  const float oy = vget(o, IY), oz = vget(o, IZ), ox = vget(o, AXIS);
  auto inside = [&](float4 lo, float4 hi) {
    float loy = IY == 0 ? lo.x : (IY == 1 ? lo.y : lo.z), hiy = IY == 0 ? hi.x : (IY == 1 ? hi.y : hi.z);
    float loz = IZ == 0 ? lo.x : (IZ == 1 ? lo.y : lo.z), hiz = IZ == 0 ? hi.x : (IZ == 1 ? hi.y : hi.z);
    float hix = AXIS == 0 ? hi.x : (AXIS == 1 ? hi.y : hi.z);
    return oy >= loy && oy <= hiy && oz >= loz && oz <= hiz && hix >= ox;
  };
  uint32_t count = 0, count64 = 0;
  auto test = [&](uint32_t leaf) {
    TriRec r = load_tri(m.stris, leaf);
    if constexpr (STATS) {
      ++qc->sign_tests;
      const RayAudit ra = ray_audit<AXIS>(o, p3(r.a), p3(r.b), p3(r.c));
      ++qc->ray_tests;
      qc->ray_ambiguous += ra.ambiguous;
      qc->ray_disagree += ra.hit64 != ra.hit32;
      count += ra.hit32 ? 1u : 0u;
      count64 += ra.hit64 ? 1u : 0u;
    } else {
      float t;
      count += ray_hit_aligned<AXIS>(o, p3(r.a), p3(r.b), p3(r.c), &t) ? 1u : 0u;
    }
  };
  if (lane == 0) s_stack[0] = 0;
  int sp = 1;
  __syncwarp();
  while (sp > 0) {
    const int take = min(sp, 32);
    const int base = sp - take;
    const uint32_t node = lane < take ? s_stack[base + lane] : 0xFFFFFFFFu;
    __syncwarp();
    sp = base;
    uint32_t push[2] = {0u, 0u};
    int npush = 0;
    if (node != 0xFFFFFFFFu) {
      if constexpr (STATS) ++qc->sign_visits;
      const BvhNode nd = load_node(m.nodes, node);
      const uint32_t ch[2] = {__float_as_uint(nd.l_lo.w), __float_as_uint(nd.l_hi.w)};
      const bool go[2] = {inside(nd.l_lo, nd.l_hi), inside(nd.r_lo, nd.r_hi)};
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        if (!go[c]) continue;
        if (ch[c] & LEAF_BIT) test(ch[c] & ~LEAF_BIT);
        else push[npush++] = ch[c];
      }
    }
    int incl = npush;
    for (int o2 = 1; o2 < 32; o2 <<= 1) {
      const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o2);
      if (lane >= o2) incl += y;
    }
    const int total = __shfl_sync(0xFFFFFFFFu, incl, 31);
    if (sp + total > CAP) return false;
    int pos = sp + incl - npush;
    for (int c = 0; c < npush; ++c) s_stack[pos++] = push[c];
    sp += total;
    __syncwarp();
  }
  for (int o2 = 16; o2; o2 >>= 1) {
    count += __shfl_xor_sync(0xFFFFFFFFu, count, o2);
    if constexpr (STATS) count64 += __shfl_xor_sync(0xFFFFFFFFu, count64, o2);
  }
  *count_out = count;
  if constexpr (STATS) *count64_out = count64;
  return true;
}

// The 3-ray vote by a whole warp (every lane returns it).  A ray whose stack
// would overflow is counted by lane 0 alone.
template <int CAP, bool STATS = false>
__device__ bool vote_inside_warp(const MeshView& m, P3 p, uint32_t* s_stack, bool* overflow, QCount* qc) {
  uint32_t c[3] = {0u, 0u, 0u}, c64[3] = {0u, 0u, 0u};
  bool ok[3];
  ok[0] = ray_crossings_warp<0, CAP, STATS>(m, p, s_stack, &c[0], qc, &c64[0]);
  ok[1] = ray_crossings_warp<1, CAP, STATS>(m, p, s_stack, &c[1], qc, &c64[1]);
  ok[2] = ray_crossings_warp<2, CAP, STATS>(m, p, s_stack, &c[2], qc, &c64[2]);
  if (!(ok[0] && ok[1] && ok[2])) {  // warp-uniform
    if ((threadIdx.x & 31) == 0) {
      if (!ok[0]) c[0] = ray_crossings<0, STATS>(m, p, overflow, qc, &c64[0]);
      if (!ok[1]) c[1] = ray_crossings<1, STATS>(m, p, overflow, qc, &c64[1]);
      if (!ok[2]) c[2] = ray_crossings<2, STATS>(m, p, overflow, qc, &c64[2]);
    }
    for (int a = 0; a < 3; ++a) {
      c[a] = __shfl_sync(0xFFFFFFFFu, c[a], 0);
      c64[a] = __shfl_sync(0xFFFFFFFFu, c64[a], 0);
    }
  }
  const int insides = (c[0] & 1u) + (c[1] & 1u) + (c[2] & 1u);
  if constexpr (STATS) {
    const int insides64 = (c64[0] & 1u) + (c64[1] & 1u) + (c64[2] & 1u);
    if ((threadIdx.x & 31) == 0) qc->vote_flip += (insides > 1) != (insides64 > 1);
  }
  return insides > 1;
}

// The counting instantiation's audit of the Voronoi region of the query's
// nearest triangle (the closest point every method's result comes from).
template <bool STATS>
__device__ __forceinline__ void audit_region(const MeshView& m, P3 p, uint32_t tri, QCount* qc) {
  if constexpr (STATS) {
    if (tri == 0xFFFFFFFFu) return;
    const TriRec r = load_tri(m.tris, tri);
    if (__float_as_int(r.a.w) != TRI_PROPER) return;
    const RegionAudit ra = region_audit(p, p3(r.a), p3(r.b), p3(r.c));
    ++qc->region;
    qc->region_ambiguous += ra.ambiguous;
    qc->region_disagree += ra.region64 != ra.region32;
  }
}

// Bvh(Normal): compare_distances over every triangle whose |signed distance|
// lies in the near-tie band of the nearest distance, folded in triangle order
// from f32::MAX with the rule of bvh.rs:125-127.
constexpr int kBand = 32;

// With a budget, the traversal gives up after `budget` node visits and clears
// *finished (the caller then hands the query to the warp pass).
template <bool STATS = false>
__device__ float normal_band_fold(const MeshView& m, P3 p, float d2min, bool* nan, bool* overflow, QCount* qc = nullptr,
                                  uint32_t budget = 0xFFFFFFFFu, bool* finished = nullptr) {
  const double band = sqrt((double)d2min) * (1.0 + 1e-5) + 4e-6;
  const float reach = (float)((band + 2e-4) * (1.0 + 1e-6));
  const float reach2 = reach * reach;
  uint32_t c_idx[kBand];
  float c_d[kBand];
  int n = 0;
  bool full = false;
  auto consider = [&](const TriRec& r) {
    if constexpr (STATS) ++qc->sign_tests;
    float d = point_triangle_signed_distance(p, p3(r.a), p3(r.b), p3(r.c), __float_as_int(r.a.w));
    if (!(fabs((double)d) <= band)) return;
    if (n < kBand) {
      c_idx[n] = __float_as_uint(r.b.w);
      c_d[n] = d;
      ++n;
    } else {
      full = true;
    }
  };
  if (m.root & LEAF_BIT) {
    consider(load_tri(m.stris, m.root & ~LEAF_BIT));
  } else {
    uint32_t stack[kStack];
    int sp = 0;
    uint32_t node = 0;
    uint32_t visits = 0;
    while (true) {
      if (++visits > budget) {
        *finished = false;
        return 0.0f;
      }
      if constexpr (STATS) ++qc->sign_visits;
      BvhNode nd = load_node(m.nodes, node);
      uint32_t L = __float_as_uint(nd.l_lo.w), R = __float_as_uint(nd.l_hi.w);
      bool goL = box_dist2(p, nd.l_lo, nd.l_hi) <= reach2, goR = box_dist2(p, nd.r_lo, nd.r_hi) <= reach2;
      if (goL && (L & LEAF_BIT)) {
        consider(load_tri(m.stris, L & ~LEAF_BIT));
        goL = false;
      }
      if (goR && (R & LEAF_BIT)) {
        consider(load_tri(m.stris, R & ~LEAF_BIT));
        goR = false;
      }
      if (goL && goR) {
        if (sp < kStack) stack[sp++] = R;
        else *overflow = true;
        node = L;
        continue;
      }
      if (goL) {
        node = L;
        continue;
      }
      if (goR) {
        node = R;
        continue;
      }
      if (sp == 0) break;
      node = stack[--sp];
    }
  }
  float best = F32_MAX;
  if (full) {
    // More ties than the register list holds: scan the band in triangle order.
    for (uint32_t t = 0; t < m.n_tris; ++t) {
      TriRec r = load_tri(m.tris, t);
      float d = point_triangle_signed_distance(p, p3(r.a), p3(r.b), p3(r.c), __float_as_int(r.a.w));
      if (!(fabs((double)d) <= band)) continue;
      if (compare_distances(best, d, nan) == 1) best = d;
    }
    return best;
  }
  for (int i = 1; i < n; ++i) {  // insertion sort by triangle index
    uint32_t ki = c_idx[i];
    float di = c_d[i];
    int j = i - 1;
    while (j >= 0 && c_idx[j] > ki) {
      c_idx[j + 1] = c_idx[j];
      c_d[j + 1] = c_d[j];
      --j;
    }
    c_idx[j + 1] = ki;
    c_d[j + 1] = di;
  }
  for (int i = 0; i < n; ++i)
    if (compare_distances(best, c_d[i], nan) == 1) best = c_d[i];
  return best;
}

// normal_band_fold for one query on a whole warp: the same band and reach,
// so the same candidates (every leaf within reach whose |d| lies in the band),
// found by a traversal that takes up to 32 nodes a step from a shared stack;
// lane 0 then sorts them by triangle index and folds them exactly as above.
// The result is normal_band_fold's bit for bit.  Returns false (and leaves
// *result alone) when the stack (CAP entries) or the candidate list
// (kBandWarp) would overflow: the caller runs normal_band_fold instead.
constexpr int kBandWarp = 64;
template <bool STATS = false, int CAP = kWarpStack>
__device__ bool normal_band_fold_warp(const MeshView& m, P3 p, float d2min, uint32_t* s_node, uint32_t* s_cidx,
                                      float* s_cd, uint32_t* s_count, float* result, bool* nan, QCount* qc) {
  const int lane = threadIdx.x & 31;
  const double band = sqrt((double)d2min) * (1.0 + 1e-5) + 4e-6;
  const float reach = (float)((band + 2e-4) * (1.0 + 1e-6));
  const float reach2 = reach * reach;
  if (lane == 0) *s_count = 0;
  __syncwarp();
  bool over = false;
  auto consider = [&](uint32_t leaf) {
    if constexpr (STATS) ++qc->sign_tests;
    const TriRec r = load_tri(m.stris, leaf);
    const float d = point_triangle_signed_distance(p, p3(r.a), p3(r.b), p3(r.c), __float_as_int(r.a.w));
    if (!(fabs((double)d) <= band)) return;
    const uint32_t pos = atomicAdd(s_count, 1u);
    if (pos < (uint32_t)kBandWarp) {
      s_cidx[pos] = __float_as_uint(r.b.w);
      s_cd[pos] = d;
    } else {
      over = true;
    }
  };
  if (m.root & LEAF_BIT) {
    if (lane == 0) consider(m.root & ~LEAF_BIT);
  } else {
    if (lane == 0) s_node[0] = 0;
    int sp = 1;
    __syncwarp();
    while (sp > 0) {
      const int take = min(sp, 32), base = sp - take;
      const uint32_t node = lane < take ? s_node[base + lane] : 0xFFFFFFFFu;
      __syncwarp();
      sp = base;
      uint32_t push[2] = {0u, 0u};
      int npush = 0;
      if (node != 0xFFFFFFFFu) {
        if constexpr (STATS) ++qc->sign_visits;
        const BvhNode nd = load_node(m.nodes, node);
        const uint32_t ch[2] = {__float_as_uint(nd.l_lo.w), __float_as_uint(nd.l_hi.w)};
        const bool go[2] = {box_dist2(p, nd.l_lo, nd.l_hi) <= reach2, box_dist2(p, nd.r_lo, nd.r_hi) <= reach2};
#pragma unroll
        for (int c = 0; c < 2; ++c) {
          if (!go[c]) continue;
          if (ch[c] & LEAF_BIT) consider(ch[c] & ~LEAF_BIT);
          else push[npush++] = ch[c];
        }
      }
      int incl = npush;
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
        if (lane >= o) incl += y;
      }
      const int total = __shfl_sync(0xFFFFFFFFu, incl, 31);
      if (sp + total > CAP) return false;  // warp-uniform
      int pos = sp + incl - npush;
      for (int c = 0; c < npush; ++c) s_node[pos++] = push[c];
      sp += total;
      __syncwarp();
    }
  }
  __syncwarp();
  if (__any_sync(0xFFFFFFFFu, over)) return false;
  if (lane == 0) {
    const int n = (int)*s_count;
    for (int i = 1; i < n; ++i) {  // insertion sort by triangle index
      const uint32_t ki = s_cidx[i];
      const float di = s_cd[i];
      int j = i - 1;
      while (j >= 0 && s_cidx[j] > ki) {
        s_cidx[j + 1] = s_cidx[j];
        s_cd[j + 1] = s_cd[j];
        --j;
      }
      s_cidx[j + 1] = ki;
      s_cd[j + 1] = di;
    }
    float best = F32_MAX;
    for (int i = 0; i < n; ++i)
      if (compare_distances(best, s_cd[i], nan) == 1) best = s_cd[i];
    *result = best;
  }
  __syncwarp();
  return true;
}

enum QueryMode { Q_BVH_RAYCAST = 0, Q_BVH_NORMAL = 1, Q_RTREE = 2, Q_VECTOR = 3 };

// A query whose single-thread search ran over its node budget, with its
// partial result (an upper bound) and its ray vote.
struct HardQuery {
  uint32_t i;
  float d2;
  uint32_t tri;
  uint32_t leaf_inside;  // leaf | inside << 31
};

// Result of a query from its nearest triangle (and ray vote), per method.
template <int MODE, bool STATS = false>
__device__ __forceinline__ void finish_query(const MeshView& m, uint64_t i, P3 p, Nearest nn, bool inside,
                                             float* out, float* vec, uint8_t* inside_out, bool* nan, bool* overflow,
                                             QCount* qc = nullptr) {
  if (nn.tri == 0xFFFFFFFFu) nn = {INFINITY, 0u, 0u};  // every distance NaN
  audit_region<STATS>(m, p, nn.tri, qc);
  if (MODE == Q_BVH_RAYCAST) {
    // bvh.rs:283-328 / rtree_bvh.rs:156-199: unsigned distance, 3-ray vote.
    float d = fminf(F32_MAX, fsqrt(nn.d2));
    out[i] = inside ? -d : d;
  } else if (MODE == Q_RTREE) {
    // rtree.rs:149-154: signed distance of the nearest triangle.
    TriRec r = load_tri(m.tris, nn.tri);
    out[i] = point_triangle_signed_distance(p, p3(r.a), p3(r.b), p3(r.c), __float_as_int(r.a.w));
  } else if (MODE == Q_BVH_NORMAL) {
    out[i] = normal_band_fold<STATS>(m, p, nn.d2, nan, overflow, qc);
  } else {
    TriRec r = load_tri(m.tris, nn.tri);
    P3 cp = closest_point_triangle(p, p3(r.a), p3(r.b), p3(r.c), __float_as_int(r.a.w));
    P3 v = vsub(cp, p);  // rtree_bvh.rs:273
    vec[3 * i] = v.x;
    vec[3 * i + 1] = v.y;
    vec[3 * i + 2] = v.z;
    inside_out[i] = inside ? 1 : 0;
  }
}

// Bvh(Normal) with the band fold's result already formed.
template <bool STATS = false>
__device__ __forceinline__ void finish_normal(const MeshView& m, uint64_t i, P3 p, Nearest nn, float band_result,
                                              float* out, QCount* qc) {
  if (nn.tri == 0xFFFFFFFFu) nn = {INFINITY, 0u, 0u};  // every distance NaN
  audit_region<STATS>(m, p, nn.tri, qc);
  out[i] = band_result;
}

// Pass 1: one thread per query.  Searches that exceed `budget` node visits
// are handed to pass 2 (k_query_hard) with their partial result; for
// Bvh(Normal) so are the tie-band folds that exceed it.
// Adds a thread's traversal counts to qstats[0..3] (one atomic per warp).
__device__ __forceinline__ void add_counts(const QCount& c, unsigned long long* qstats) {
  const unsigned mask = __activemask();  // lanes past the last query have left
  const unsigned v[kQueryCounters] = {
      __reduce_add_sync(mask, c.visits),          __reduce_add_sync(mask, c.tests),
      __reduce_add_sync(mask, c.sign_visits),     __reduce_add_sync(mask, c.sign_tests),
      __reduce_add_sync(mask, c.ray_tests),       __reduce_add_sync(mask, c.ray_ambiguous),
      __reduce_add_sync(mask, c.ray_disagree),    __reduce_add_sync(mask, c.vote_flip),
      __reduce_add_sync(mask, c.region),          __reduce_add_sync(mask, c.region_ambiguous),
      __reduce_add_sync(mask, c.region_disagree)};
  if ((threadIdx.x & 31) == (unsigned)(__ffs(mask) - 1))
    for (int f = 0; f < kQueryCounters; ++f)
      if (v[f]) atomicAdd(&qstats[f], (unsigned long long)v[f]);
}

template <int MODE, bool STATS = false>
__global__ void __launch_bounds__(128) k_query(MeshView m, const float* __restrict__ q,
                                               const uint32_t* __restrict__ order, uint64_t nq,
                                               float* __restrict__ out, float* __restrict__ vec,
                                               uint8_t* __restrict__ inside_out, uint32_t* status, uint32_t budget,
                                               HardQuery* hard, uint32_t* hard_count, bool packet,
                                               unsigned long long* qstats = nullptr) {
  uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (!packet && k >= nq) return;  // a packet search needs every lane of the warp
  const bool active = k < nq;
  uint64_t i = active ? (order ? order[k] : k) : 0;
  P3 p = active ? load_query(q, i) : P3{0.0f, 0.0f, 0.0f};
  bool overflow = false, nan = false;
  bool inside = false;
  QCount qc;
  bool finished = true;
  const uint32_t bud = !hard ? 0xFFFFFFFFu : budget;
  Nearest nn;
  if (packet) {
    nn = nearest_triangle_packet<STATS>(m, p, active, &overflow, bud, &finished, &qc);
    if (!active) return;
  } else {
    nn = nearest_triangle<STATS>(m, p, &overflow, Nearest{INFINITY, 0xFFFFFFFFu, 0}, bud, &finished, &qc);
  }
  if (MODE == Q_BVH_RAYCAST || MODE == Q_VECTOR) inside = vote_inside<STATS>(m, p, &overflow, &qc);
  float band_result = 0.0f;
  if (MODE == Q_BVH_NORMAL && hard && finished)
    band_result = normal_band_fold<STATS>(m, p, nn.d2, &nan, &overflow, &qc, budget, &finished);
  if (finished) {
    if (MODE == Q_BVH_NORMAL && hard) finish_normal<STATS>(m, i, p, nn, band_result, out, &qc);
    else finish_query<MODE, STATS>(m, i, p, nn, inside, out, vec, inside_out, &nan, &overflow, &qc);
  } else {
    uint32_t pos = atomicAdd(hard_count, 1u);
    hard[pos] = HardQuery{(uint32_t)i, nn.d2, nn.tri, nn.leaf | (inside ? 0x80000000u : 0u)};
  }
  if (overflow) atomicOr(status, bit(M2S_ERR_LIMIT));
  if (nan) atomicOr(status, bit(M2S_ERR_NAN_DISTANCE));
  if constexpr (STATS) add_counts(qc, qstats);
}

// Pass 2: one warp per hard query (see nearest_triangle_warp).
constexpr int kHardWarps = 2;  // warps per block; each owns a kWarpStack-entry stack

template <int MODE, bool STATS = false>
__global__ void __launch_bounds__(32 * kHardWarps) k_query_hard(MeshView m, const float* __restrict__ q,
                                                               const HardQuery* __restrict__ hard,
                                                               const uint32_t* hard_count, float* __restrict__ out,
                                                               float* __restrict__ vec, uint8_t* __restrict__ inside_out,
                                                               uint32_t* status, unsigned long long* qstats = nullptr) {
  QCount qc;  // every lane's node fetches and tests of the warp searches
  __shared__ uint32_t s_node[kHardWarps][kWarpStack];
  __shared__ float s_dist[kHardWarps][kWarpStack];
  __shared__ uint32_t s_cidx[MODE == Q_BVH_NORMAL ? kHardWarps : 1][kBandWarp];
  __shared__ float s_cd[MODE == Q_BVH_NORMAL ? kHardWarps : 1][kBandWarp];
  __shared__ uint32_t s_ccount[kHardWarps];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const uint32_t n = *hard_count;
  bool overflow = false, nan = false;
  for (uint32_t h = blockIdx.x * kHardWarps + w; h < n; h += gridDim.x * kHardWarps) {
    const HardQuery hq = hard[h];
    const P3 p = load_query(q, hq.i);
    Nearest nn{hq.d2, hq.tri, hq.leaf_inside & 0x7FFFFFFFu};
    const bool inside = (hq.leaf_inside >> 31) != 0;
    const bool ok = nearest_triangle_warp<STATS>(m, p, &nn, s_node[w], s_dist[w], &qc);
    if (MODE == Q_BVH_NORMAL) {
      if (lane == 0 && !ok) nn = nearest_triangle<STATS>(m, p, &overflow, nn, 0xFFFFFFFFu, nullptr, &qc);
      nn.d2 = __shfl_sync(0xFFFFFFFFu, nn.d2, 0);
      nn.tri = __shfl_sync(0xFFFFFFFFu, nn.tri, 0);
      nn.leaf = __shfl_sync(0xFFFFFFFFu, nn.leaf, 0);
      float r = 0.0f;
      const bool wok = normal_band_fold_warp<STATS>(m, p, nn.d2, s_node[w], s_cidx[MODE == Q_BVH_NORMAL ? w : 0],
                                                    s_cd[MODE == Q_BVH_NORMAL ? w : 0], &s_ccount[w], &r, &nan, &qc);
      if (lane == 0) {
        if (!wok) r = normal_band_fold<STATS>(m, p, nn.d2, &nan, &overflow, &qc);  // list or stack full: one lane
        finish_normal<STATS>(m, hq.i, p, nn, r, out, &qc);
      }
    } else if (lane == 0) {
      if (!ok) nn = nearest_triangle<STATS>(m, p, &overflow, nn, 0xFFFFFFFFu, nullptr, &qc);  // stack full: finish on one lane
      finish_query<MODE, STATS>(m, hq.i, p, nn, inside, out, vec, inside_out, &nan, &overflow, &qc);
    }
    __syncwarp();
  }
  if (overflow) atomicOr(status, bit(M2S_ERR_LIMIT));
  if (nan) atomicOr(status, bit(M2S_ERR_NAN_DISTANCE));
  if constexpr (STATS) add_counts(qc, qstats);
}

// Small batches: one warp per query from the start.  A batch of a few
// thousand queries leaves most of the GPU idle under one thread per query,
// and its time is its longest chain of dependent node fetches (the search,
// then three ray traversals, then the warp pass for long searches).  Here the
// warp searches (nearest_triangle_warp) and casts the three rays
// (vote_inside_warp) together, 32 nodes a step.  Results are the other
// passes' bit for bit: the exact minimum of (distance, triangle) and exact
// crossing counts.  kSmallStack entries of stack per warp; on overflow lane 0
// finishes alone.  512 entries (16 KB a block) fit 14 blocks per SM against 7
// with 1,024, so a batch of 8,192 queries runs in one wave (bit-identical;
// star s6 Rtree 0.68 -> 0.59 ms, the terrain strip's Rtree 0.27 -> 0.20 ms;
// batches up to 4,096 fit either way and are unchanged).
constexpr int kSmallWarps = 4;
constexpr int kSmallStack = 512;

template <int MODE, bool STATS = false>
__global__ void __launch_bounds__(32 * kSmallWarps) k_query_warpwise(MeshView m, const float* __restrict__ q,
                                                                    uint64_t nq, float* __restrict__ out,
                                                                    float* __restrict__ vec,
                                                                    uint8_t* __restrict__ inside_out, uint32_t* status,
                                                                    unsigned long long* qstats = nullptr) {
  QCount qc;
  __shared__ uint32_t s_node[kSmallWarps][kSmallStack];
  __shared__ float s_dist[kSmallWarps][kSmallStack];
  __shared__ uint32_t s_cidx[MODE == Q_BVH_NORMAL ? kSmallWarps : 1][kBandWarp];
  __shared__ float s_cd[MODE == Q_BVH_NORMAL ? kSmallWarps : 1][kBandWarp];
  __shared__ uint32_t s_ccount[kSmallWarps];
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  bool overflow = false, nan = false;
  for (uint64_t i = (uint64_t)blockIdx.x * kSmallWarps + w; i < nq; i += (uint64_t)gridDim.x * kSmallWarps) {
    const P3 p = load_query(q, i);
    Nearest nn{INFINITY, 0xFFFFFFFFu, 0};
    const bool ok = nearest_triangle_warp<STATS, kSmallStack>(m, p, &nn, s_node[w], s_dist[w], &qc);
    bool inside = false;
    if (MODE == Q_BVH_RAYCAST || MODE == Q_VECTOR) inside = vote_inside_warp<kSmallStack, STATS>(m, p, s_node[w], &overflow, &qc);
    if (MODE == Q_BVH_NORMAL) {
      if (lane == 0 && !ok) nn = nearest_triangle<STATS>(m, p, &overflow, nn, 0xFFFFFFFFu, nullptr, &qc);
      nn.d2 = __shfl_sync(0xFFFFFFFFu, nn.d2, 0);
      nn.tri = __shfl_sync(0xFFFFFFFFu, nn.tri, 0);
      nn.leaf = __shfl_sync(0xFFFFFFFFu, nn.leaf, 0);
      float r = 0.0f;
      const bool wok = normal_band_fold_warp<STATS, kSmallStack>(m, p, nn.d2, s_node[w],
                                                                 s_cidx[MODE == Q_BVH_NORMAL ? w : 0],
                                                                 s_cd[MODE == Q_BVH_NORMAL ? w : 0], &s_ccount[w], &r,
                                                                 &nan, &qc);
      if (lane == 0) {
        if (!wok) r = normal_band_fold<STATS>(m, p, nn.d2, &nan, &overflow, &qc);
        finish_normal<STATS>(m, i, p, nn, r, out, &qc);
      }
      __syncwarp();
      continue;
    }
    if (lane == 0) {
      if (!ok) nn = nearest_triangle<STATS>(m, p, &overflow, nn, 0xFFFFFFFFu, nullptr, &qc);  // stack full: finish alone
      finish_query<MODE, STATS>(m, i, p, nn, inside, out, vec, inside_out, &nan, &overflow, &qc);
    }
    __syncwarp();
  }
  if (overflow) atomicOr(status, bit(M2S_ERR_LIMIT));
  if (nan) atomicOr(status, bit(M2S_ERR_NAN_DISTANCE));
  if constexpr (STATS) add_counts(qc, qstats);
}

// Morton order of the queries (spatially coherent warps).
__global__ void k_query_keys(const float* __restrict__ q, uint64_t nq, MeshView m, uint32_t* keys, uint32_t* vals) {
  uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  float4 lo, hi;
  if (m.root & LEAF_BIT) {
    TriRec r = m.stris[0];
    lo = make_float4(fminf(r.a.x, fminf(r.b.x, r.c.x)), fminf(r.a.y, fminf(r.b.y, r.c.y)),
                     fminf(r.a.z, fminf(r.b.z, r.c.z)), 0);
    hi = make_float4(fmaxf(r.a.x, fmaxf(r.b.x, r.c.x)), fmaxf(r.a.y, fmaxf(r.b.y, r.c.y)),
                     fmaxf(r.a.z, fmaxf(r.b.z, r.c.z)), 0);
  } else {
    BvhNode nd = m.nodes[0];
    lo = make_float4(fminf(nd.l_lo.x, nd.r_lo.x), fminf(nd.l_lo.y, nd.r_lo.y), fminf(nd.l_lo.z, nd.r_lo.z), 0);
    hi = make_float4(fmaxf(nd.l_hi.x, nd.r_hi.x), fmaxf(nd.l_hi.y, nd.r_hi.y), fmaxf(nd.l_hi.z, nd.r_hi.z), 0);
  }
  P3 p = load_query(q, i);
  float c[3] = {p.x, p.y, p.z}, l[3] = {lo.x, lo.y, lo.z}, h[3] = {hi.x, hi.y, hi.z};
  uint32_t key = 0;
  for (int d = 0; d < 3; ++d) {
    float ext = h[d] - l[d];
    float u = ext > 0.0f ? (c[d] - l[d]) / ext : 0.0f;
    uint32_t v = (uint32_t)fminf(fmaxf(u * 1024.0f, 0.0f), 1023.0f);
    for (int b = 0; b < 10; ++b) key |= ((v >> b) & 1u) << (3 * b + (2 - d));
  }
  keys[i] = key;
  vals[i] = (uint32_t)i;
}

}  // namespace

// Node-visit budget of the single-thread search (0: single pass only).
std::atomic<uint32_t> g_query_budget{768};

// Batch size from which Raycast, Rtree and vector queries search a warp at a
// time (measured crossover: star s6 and the 512^2 terrain are even at 400k to
// 600k queries; 1M star points 8.0 -> 7.1 ms, 4M terrain points 15.2 -> 10.7 ms;
// 100k star points 2.4 -> 2.9 ms).
constexpr uint64_t kPacketMinQueries = 1u << 19;
// Batches up to this many queries run one warp per query (k_query_warpwise).
// Measured on B200, star s6, RtreeBvh / Rtree, against the two-pass path:
// 1,000 queries 0.39 / 0.37 ms against 0.57 / 0.45 ms, 4,000 0.43 / 0.39
// against 0.60 / 0.46 ms, but 16,000 1.24 / 1.13 against 0.98 / 0.74 ms
// (bit-identical results throughout).
constexpr uint64_t kWarpwiseMaxQueries = 8192;
constexpr uint64_t kMortonMinQueries = 1u << 17;  // batch size from which queries run in Morton order

namespace {
// Order-preserving int image of a float (for atomic min / max).
__device__ __forceinline__ int f2o(float f) {
  const int i = __float_as_int(f);
  return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__device__ __forceinline__ float o2f(int i) { return __int_as_float(i >= 0 ? i : i ^ 0x7FFFFFFF); }
__global__ void k_bf_bounds_init(int* b) {
  if (threadIdx.x < 3) b[threadIdx.x] = 0x7FFFFFFF;
  else if (threadIdx.x < 6) b[threadIdx.x] = (int)0x80000000;
}
__global__ void k_bf_bounds(const float* __restrict__ q, uint64_t nq, int* b) {
  int lo[3] = {0x7FFFFFFF, 0x7FFFFFFF, 0x7FFFFFFF}, hi[3] = {(int)0x80000000, (int)0x80000000, (int)0x80000000};
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nq; i += (uint64_t)gridDim.x * blockDim.x)
    for (int d = 0; d < 3; ++d) {
      const int v = f2o(q[3 * i + d]);
      lo[d] = min(lo[d], v);
      hi[d] = max(hi[d], v);
    }
  for (int d = 0; d < 3; ++d) {
    for (int o = 16; o; o >>= 1) {
      lo[d] = min(lo[d], __shfl_xor_sync(0xFFFFFFFFu, lo[d], o));
      hi[d] = max(hi[d], __shfl_xor_sync(0xFFFFFFFFu, hi[d], o));
    }
    if ((threadIdx.x & 31) == 0) {
      atomicMin(&b[d], lo[d]);
      atomicMax(&b[3 + d], hi[d]);
    }
  }
}
__global__ void k_bf_keys(const float* __restrict__ q, uint64_t nq, const int* __restrict__ b, uint32_t* keys,
                          uint32_t* vals) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= nq) return;
  uint32_t key = 0;
  for (int d = 0; d < 3; ++d) {
    const float l = o2f(b[d]), h = o2f(b[3 + d]);
    const float ext = h - l;
    const float u = ext > 0.0f ? (q[3 * i + d] - l) / ext : 0.0f;
    const uint32_t v = (uint32_t)fminf(fmaxf(u * 1024.0f, 0.0f), 1023.0f);  // NaN -> 0
    for (int bt = 0; bt < 10; ++bt) key |= ((v >> bt) & 1u) << (3 * bt + (2 - d));
  }
  keys[i] = key;
  vals[i] = (uint32_t)i;
}
}  // namespace

int brute_force_sdf(const MeshView& m, int sign, const float* d_q, uint64_t nq, float* d_out, uint32_t* d_status,
                    cudaStream_t s, bool allow_alloc) {
  if (nq == 0) return M2S_OK;
  unsigned blocks = (unsigned)((nq + kBfThreads - 1) / kBfThreads);
  // Thread-per-query kernels visit large batches (2^28 pairs or more: the
  // sort's ~20 launches take ~0.1 ms, the order saves ~13 % of the kernel)
  // in Morton order (of the
  // queries' own bounding box): the lanes of a warp then mostly fall in the
  // same Voronoi regions of a triangle and take the same branches (65,536
  // points x 81,920 triangles Raycast 24.3 -> 21.2 ms, 262,144 Normal 108.5
  // -> 88.9 ms).  Results are per query, so the order changes none.
  DevBuf<uint32_t> keys, order;
  DevBuf<int> bounds;
  const uint32_t* ord = nullptr;
  const bool thread_kernel = sign == M2S_SIGN_RAYCAST || nq >= kBruteWarpMaxQueries;
  if (allow_alloc && thread_kernel && nq >= 4096 && nq <= 0xFFFFFFFFull && nq * m.n_tris >= kBruteSortMinPairs) {
    int st;
    if ((st = keys.alloc(nq, s)) || (st = order.alloc(nq, s)) || (st = bounds.alloc(6, s))) return st;
    k_bf_bounds_init<<<1, 32, 0, s>>>(bounds.p);
    k_bf_bounds<<<(unsigned)std::min<uint64_t>((nq + 255) / 256, 148u * 8u), 256, 0, s>>>(d_q, nq, bounds.p);
    k_bf_keys<<<(unsigned)((nq + 255) / 256), 256, 0, s>>>(d_q, nq, bounds.p, keys.p, order.p);
    M2S_CUDA(cudaGetLastError());
    if ((st = radix_sort_pairs(keys.p, order.p, nq, 30, s))) return st;
    ord = order.p;
  }
  if (sign == M2S_SIGN_RAYCAST) {
    // Enough (query, triangle chunk) blocks to fill the GPU ~4 deep.
    const uint32_t tiles = (m.n_tris + kBfTile - 1) / kBfTile;
    uint32_t chunks = (uint32_t)std::max<uint64_t>(1, (148ull * 16ull + blocks - 1) / blocks);
    chunks = std::max(1u, std::min(chunks, std::min(tiles, 64u)));
    if (chunks == 1 || !allow_alloc) {
      k_brute<0><<<blocks, kBfThreads, 0, s>>>(m.tris, m.n_tris, d_q, nq, d_out, d_status, nullptr, ord);
    } else {
      DevBuf<uint2> part;
      int st = part.alloc(nq, s);
      if (st) return st;
      k_brute_init<<<(unsigned)std::min<uint64_t>((nq + 255) / 256, 148u * 16u), 256, 0, s>>>(part.p, nq);
      k_brute<0><<<dim3(blocks, chunks), kBfThreads, 0, s>>>(m.tris, m.n_tris, d_q, nq, d_out, d_status, part.p, ord);
      k_brute_finish<<<(unsigned)std::min<uint64_t>((nq + 255) / 256, 148u * 16u), 256, 0, s>>>(part.p, nq, d_out);
    }
  } else if (nq < kBruteWarpMaxQueries) {
    // Too few queries for one thread each to fill the GPU (the thread kernel
    // needs about 150k): a warp per query (8,192 queries x 81,920 triangles:
    // 26.7 -> 4.4 ms; 65,536: 37.6 -> 31.0 ms; at 262,144 the thread kernel
    // is ahead, 109 against 122 ms).
    const unsigned wblocks = (unsigned)((nq + kBwThreads / 32 - 1) / (kBwThreads / 32));
    k_brute_normal_warp<<<wblocks, kBwThreads, 0, s>>>(m.tris, m.n_tris, d_q, nq, d_out, d_status);
  } else {
    k_brute<1><<<blocks, kBfThreads, 0, s>>>(m.tris, m.n_tris, d_q, nq, d_out, d_status, nullptr, ord);
  }
  M2S_CUDA(cudaGetLastError());
  return M2S_OK;
}

namespace {
template <bool ST>
void launch_queries(int mode, const MeshView& m, const float* d_q, const uint32_t* ord, uint64_t nq, float* d_out,
                    float* d_vec, uint8_t* d_inside, uint32_t* d_status, uint32_t budget, HardQuery* hp, uint32_t* hc,
                    bool two_pass, bool packet, unsigned blocks, unsigned long long* qs, cudaStream_t s) {
  const unsigned hard_blocks = 148u * 32u;
  switch (mode) {
    case Q_BVH_RAYCAST:
      k_query<Q_BVH_RAYCAST, ST><<<blocks, 128, 0, s>>>(m, d_q, ord, nq, d_out, nullptr, nullptr, d_status, budget, hp,
                                                        hc, packet, qs);
      if (two_pass)
        k_query_hard<Q_BVH_RAYCAST, ST><<<hard_blocks, 32 * kHardWarps, 0, s>>>(m, d_q, hp, hc, d_out, nullptr,
                                                                                  nullptr, d_status, qs);
      break;
    case Q_BVH_NORMAL:
      k_query<Q_BVH_NORMAL, ST><<<blocks, 128, 0, s>>>(m, d_q, ord, nq, d_out, nullptr, nullptr, d_status, budget, hp,
                                                       hc, packet, qs);
      if (two_pass)
        k_query_hard<Q_BVH_NORMAL, ST><<<hard_blocks, 32 * kHardWarps, 0, s>>>(m, d_q, hp, hc, d_out, nullptr,
                                                                                 nullptr, d_status, qs);
      break;
    case Q_RTREE:
      k_query<Q_RTREE, ST><<<blocks, 128, 0, s>>>(m, d_q, ord, nq, d_out, nullptr, nullptr, d_status, budget, hp, hc,
                                                  packet, qs);
      if (two_pass)
        k_query_hard<Q_RTREE, ST><<<hard_blocks, 32 * kHardWarps, 0, s>>>(m, d_q, hp, hc, d_out, nullptr, nullptr,
                                                                            d_status, qs);
      break;
    default:
      k_query<Q_VECTOR, ST><<<blocks, 128, 0, s>>>(m, d_q, ord, nq, nullptr, d_vec, d_inside, d_status, budget, hp, hc,
                                                   packet, qs);
      if (two_pass)
        k_query_hard<Q_VECTOR, ST><<<hard_blocks, 32 * kHardWarps, 0, s>>>(m, d_q, hp, hc, nullptr, d_vec, d_inside,
                                                                             d_status, qs);
  }
}
}  // namespace

int query_points(const MeshView& m, int accel, int sign, const float* d_q, uint64_t nq, float* d_out, float* d_vec,
                 uint8_t* d_inside, uint32_t* d_status, cudaStream_t s, int64_t budget_override) {
  if (nq == 0) return M2S_OK;
  if (accel == M2S_ACCEL_NONE && !d_vec) return brute_force_sdf(m, sign, d_q, nq, d_out, d_status, s);
  if (m.n_tris == 0) return M2S_ERR_EMPTY_MESH;
  if (nq > 0xFFFFFFFFull) return M2S_ERR_INVALID_ARGUMENT;
  const int mode = d_vec ? Q_VECTOR
                         : (accel == M2S_ACCEL_RTREE
                                ? Q_RTREE
                                : ((accel == M2S_ACCEL_BVH && sign == M2S_SIGN_NORMAL) ? Q_BVH_NORMAL : Q_BVH_RAYCAST));
  // Small batches (a mesh of more than one triangle): one warp per query.
  if (nq <= kWarpwiseMaxQueries && !(m.root & LEAF_BIT)) {
    const bool counting = profiling_enabled() || grid_tuning().fp64_audit;
    DevBuf<unsigned long long> qs;
    int st;
    if (counting) {
      if ((st = qs.alloc(kQueryCounters, s))) return st;
      M2S_CUDA(cudaMemsetAsync(qs.p, 0, 8 * kQueryCounters, s));
    }
    const unsigned wb = (unsigned)std::min<uint64_t>((nq + kSmallWarps - 1) / kSmallWarps, 148ull * 64ull);
    auto go = [&](auto st_tag) {
      constexpr bool ST = decltype(st_tag)::value;
      unsigned long long* qp = ST ? qs.p : nullptr;
      if (mode == Q_BVH_RAYCAST)
        k_query_warpwise<Q_BVH_RAYCAST, ST><<<wb, 32 * kSmallWarps, 0, s>>>(m, d_q, nq, d_out, nullptr, nullptr,
                                                                            d_status, qp);
      else if (mode == Q_RTREE)
        k_query_warpwise<Q_RTREE, ST><<<wb, 32 * kSmallWarps, 0, s>>>(m, d_q, nq, d_out, nullptr, nullptr, d_status,
                                                                      qp);
      else if (mode == Q_BVH_NORMAL)
        k_query_warpwise<Q_BVH_NORMAL, ST><<<wb, 32 * kSmallWarps, 0, s>>>(m, d_q, nq, d_out, nullptr, nullptr,
                                                                           d_status, qp);
      else
        k_query_warpwise<Q_VECTOR, ST><<<wb, 32 * kSmallWarps, 0, s>>>(m, d_q, nq, nullptr, d_vec, d_inside, d_status,
                                                                       qp);
    };
    if (counting) go(std::true_type{});
    else go(std::false_type{});
    M2S_CUDA(cudaGetLastError());
    if (counting) {
      unsigned long long h[kQueryCounters];
      M2S_CUDA(cudaMemcpyAsync(h, qs.p, 8 * kQueryCounters, cudaMemcpyDeviceToHost, s));
      M2S_CUDA(cudaStreamSynchronize(s));
      const uint64_t rec[1 + kQueryCounters] = {nq, h[0], h[1], h[2], h[3], h[4], h[5], h[6], h[7], h[8], h[9], h[10]};
      record_query_stats(rec);
    }
    return M2S_OK;
  }
  // Morton-ordered launch for large batches: from 2^17 queries (below, the
  // sort's launches cost more than coherent warps save: 10k RtreeBvh points
  // on icosphere s3 0.33 -> 0.21 ms unsorted, star s6 50k 1.84 -> 1.65 ms; at
  // 200k sorting wins, 3.75 -> 3.20 ms), and from 4096 for Bvh(Normal), whose
  // packet search needs the order.
  DevBuf<uint32_t> keys, order;
  const uint32_t* ord = nullptr;
  int st;
  if (nq >= (mode == Q_BVH_NORMAL ? 4096u : kMortonMinQueries)) {
    if ((st = keys.alloc(nq, s)) || (st = order.alloc(nq, s))) return st;
    k_query_keys<<<(unsigned)((nq + 255) / 256), 256, 0, s>>>(d_q, nq, m, keys.p, order.p);
    M2S_CUDA(cudaGetLastError());
    if ((st = radix_sort_pairs(keys.p, order.p, nq, 30, s))) return st;
    ord = order.p;
  }
  unsigned blocks = (unsigned)((nq + 127) / 128);
  // Queries over the node budget continue one warp per query.
  DevBuf<HardQuery> hard;
  DevBuf<uint32_t> hard_count;
  const uint32_t base_budget =
      budget_override >= 0 ? (uint32_t)budget_override : g_query_budget.load(std::memory_order_relaxed);
  // Bvh(Normal) hands long searches and tie-band folds to the warp pass in
  // batches below 2^18 queries (where the budget is base / 16), whose
  // single-thread band traversals set the time (star s6: 1,000 points 6.17
  // -> 0.59 ms, 10,000 15.5 -> 1.4 ms, 131,072 21.9 -> 3.4 ms, 262,143 23.9
  // -> 5.2 ms; star s4 200,000 4.1 -> 1.9 ms; the terrain strip: 20,000 3.69
  // -> 1.39 ms, 131,072 2.85 -> 2.38 ms, though 262,143 3.36 -> 4.31 ms);
  // from there on the one-pass packet search keeps its coherence and wins on
  // the terrain (400,000 points 4.1 against 9.0 ms with the hand-off at the
  // default budget, 1M 6.7 against 20.0) and ties on the star (1M 30.2
  // against 30.7 ms).  A base budget of at most kNormalHandoffMaxBudget keeps
  // the hand-off at every size, which suits closed meshes whose deep-interior
  // points make long searches (star s6 at budget 64: 400,000 points 27.5 ->
  // 7.7 ms, 1M 29.8 -> 17.0 ms) but not open ones (the terrain: 4.1 -> 6.3
  // and 6.6 -> 14.7 ms); the autotuner tries it.
  const bool two_pass =
      base_budget > 0 && (mode != Q_BVH_NORMAL || nq < (1u << 18) || base_budget <= kNormalHandoffMaxBudget);
  if (two_pass) {
    if ((st = hard.alloc(nq, s)) || (st = hard_count.alloc(1, s))) return st;
    M2S_CUDA(cudaMemsetAsync(hard_count.p, 0, 4, s));
  }
  // Smaller batches hand long searches to the warp pass sooner: their time is
  // the longest single-thread search, not the throughput of many.
  const uint32_t budget = effective_query_budget(base_budget, nq);
  HardQuery* hp = two_pass ? hard.p : nullptr;
  uint32_t* hc = two_pass ? hard_count.p : nullptr;
  // With profiling on, the counting instantiations run and their totals are
  // read back (a synchronisation, as profiling's phase timings are).
  const bool counting = profiling_enabled() || grid_tuning().fp64_audit;
  DevBuf<unsigned long long> qs;
  if (counting) {
    if ((st = qs.alloc(kQueryCounters, s))) return st;
    M2S_CUDA(cudaMemsetAsync(qs.p, 0, 8 * kQueryCounters, s));
  }
  // Morton-ordered warps search together (nearest_triangle_packet): always
  // for Bvh(Normal), and for the others from kPacketMinQueries on, where
  // throughput rather than the longest warp sets the time.
  const bool packet = ord != nullptr && (mode == Q_BVH_NORMAL || nq >= kPacketMinQueries);
  if (counting)
    launch_queries<true>(mode, m, d_q, ord, nq, d_out, d_vec, d_inside, d_status, budget, hp, hc, two_pass, packet,
                         blocks, qs.p, s);
  else
    launch_queries<false>(mode, m, d_q, ord, nq, d_out, d_vec, d_inside, d_status, budget, hp, hc, two_pass, packet,
                          blocks, nullptr, s);
  M2S_CUDA(cudaGetLastError());
  if (counting) {
    unsigned long long h[kQueryCounters];
    M2S_CUDA(cudaMemcpyAsync(h, qs.p, 8 * kQueryCounters, cudaMemcpyDeviceToHost, s));
    M2S_CUDA(cudaStreamSynchronize(s));
    const uint64_t rec[1 + kQueryCounters] = {nq, h[0], h[1], h[2], h[3], h[4], h[5], h[6], h[7], h[8], h[9], h[10]};
    record_query_stats(rec);
  }
  return M2S_OK;
}

}  // namespace m2s
