// generate_grid_sdf on the device (generate/grid.rs:265-684), for one grid or
// for a batch of (mesh, grid) pairs in one set of launches.
//
// 1. Seeding (generate_preheap, grid.rs:383-457): one warp per triangle walks
//    the cells of its padded, snapped and widened box and keeps, per cell, the
//    best (distance, triangle) under compare_distances.  Cells hold one packed
//    64-bit key: high word = f32 bits of the distance, low word = triangle
//    shifted left by one over a dirty bit (8 bytes of state per cell).
// 2. Propagation (generate_heap + propagate_heap, grid.rs:464-558): the
//    reference pops (cell, triangle) states from heaps in distance order and
//    evaluates the popped triangle on the 27 cells of the 3x3x3 block, keeping
//    strict improvements.  Here the heap becomes delta-stepping in one
//    cooperative launch.  States are binned by distance: a quarter of the
//    smallest cell size per bucket for the first 8 cells, logarithmically
//    wider beyond.  Each round relaxes the lowest non-empty bucket, one thread
//    per (state, neighbour) proposal.  Proposals lower the cell's key in
//    place with atomics; the first to lower a clean key sets its dirty bit
//    and stages the cell, and the commit clears it and queues the round's
//    best proposal per cell for further propagation — the same winner as if
//    every proposal had competed with the value at the start of the round.  Sixteen consecutive buckets (the
//    window) have their own lists; states beyond the window wait in a far list
//    and are moved into the window, each to its exact bucket, when the window
//    runs empty.  So every state is relaxed in the round of its own bucket,
//    whatever else shares the launch, and the result does not depend on the
//    order of atomics.
// 3. Sign (compute_raycasts, grid.rs:568-684): every triangle is tested, with
//    the reference's aligned ray test, against the rays that start at the cell
//    centres of the three low faces and lie in its padded box.  A hit at t
//    toggles bit k = min(floor(t / size), n - 1) of that ray's column; a
//    suffix XOR turns toggles into per-cell crossing parities, and a cell is
//    inside when at least two of its three parities are odd (grid.rs:622-639).
//
// Batches.  The grids of a batch share one cell index space (grid k starts at
// a cell offset) and one triangle array (each triangle knows its grid).
// Buckets are measured in each grid's own cell size and a grid only ever
// touches its own cells, so a grid's states are relaxed in the same rounds, in
// the same buckets, as when it runs alone: batched results are bit-identical
// to single-grid results, and the batch takes as many rounds as its slowest
// grid instead of the sum.  Kernels are instantiated with MULTI = false (the
// grid travels in the kernel parameters) and MULTI = true (grid table).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

#include "m2s_audit.cuh"
#include "m2s_internal.cuh"

namespace m2s {
namespace {

// A cell's 64-bit key: the f32 distance bits (high word), the triangle
// (bits 1..31; a job holds fewer than 2^31 - 1 triangles) and bit 0, kDirty:
// set while the cell has been lowered in the current relax round and not yet
// committed.  Between rounds every key is clean.
constexpr uint32_t NO_TRI = 0x7FFFFFFFu;
constexpr unsigned long long kDirty = 1ull;
constexpr unsigned long long KEY_EMPTY = (0x7F7FFFFFull << 32) | ((unsigned long long)NO_TRI << 1);  // (f32::MAX, none)
constexpr int kRing = 16;           // buckets of the window
constexpr int kCur0 = kRing;        // list relaxed first (empty)
constexpr int kFar0 = kRing + 1;    // far lists kFar0 and kFar0 + 1 (ping-pong)
constexpr int kLists = kRing + 3;
constexpr uint32_t kNoBucket = 0xFFFFFFFFu;
constexpr uint32_t kMaxSteps = 1u << 22;  // bound on rounds + redistributions
constexpr int kAuditStats = 7;

// Unsigned 32-bit division by an invariant divisor with a multiply-high and
// two shifts (Granlund & Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994, Figure 4.1): exact for every 32-bit dividend.
struct FastDiv {
  uint32_t d, m, s1, s2;
};
FastDiv make_fastdiv(uint32_t d) {
  uint32_t l = 0;
  while (l < 32 && (1ull << l) < d) ++l;  // l = ceil(log2 d)
  unsigned __int128 num = ((unsigned __int128)1 << 32) * (((unsigned __int128)1 << l) - d);
  FastDiv f;
  f.d = d;
  f.m = (uint32_t)(num / d + 1);
  f.s1 = l < 1 ? l : 1;
  f.s2 = l > 0 ? l - 1 : 0;
  return f;
}
__device__ __forceinline__ uint32_t fdiv(const FastDiv& f, uint32_t n) {
  uint32_t t = __umulhi(f.m, n);
  return (t + ((n - t) >> f.s1)) >> f.s2;
}

// One grid of a job.
struct GridK {
  float f[3], s[3];
  int n[3];
  uint32_t ncell;     // cells of this grid
  uint32_t cell_off;  // its first cell in the job's cell index space
  float inv_delta;    // 1 / bucket width
  FastDiv div_z;      // by n[2]
  FastDiv div_y;      // by n[1]
  uint32_t words[3];  // 32-bit words per ray column, per axis
  unsigned long long bits_off[3];  // its first ray word, per axis
  unsigned long long col_off[3];   // its first ray column, per axis
  unsigned long long out_off;      // its first value in the caller's output
};

// Kernel view of a job.
struct GridSet {
  GridK g0;                               // single grid: the grid itself
  const GridK* table;                     // batch: every grid
  const uint32_t* tri_grid;               // batch: grid of each triangle
  const uint32_t* cell_off;               // batch: ngrids + 1 cell offsets
  const unsigned long long* col_off[3];   // batch: ngrids + 1 ray-column offsets per axis
  uint32_t ngrids;
  uint32_t ncell;                         // cells of the whole job
  unsigned long long ncols[3];            // ray columns of the whole job, per axis
};

// Index k with off[k] <= v < off[k + 1] (off has n + 1 entries, off[0] <= v < off[n]).
template <class T>
__device__ __forceinline__ uint32_t find_segment(const T* off, uint32_t n, T v) {
  uint32_t lo = 0, hi = n;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (off[mid] <= v) lo = mid;
    else hi = mid;
  }
  return lo;
}

// Segment lookups for a thread that walks increasing values: it searches only
// when the value leaves the segment of the previous one.
template <class T>
struct SegCursor {
  uint32_t k = 0;
  T lo = 1, hi = 0;
  __device__ __forceinline__ uint32_t at(const T* off, uint32_t n, T v) {
    if (v < lo || v >= hi) {
      k = find_segment(off, n, v);
      lo = off[k];
      hi = off[k + 1];
    }
    return k;
  }
};

template <bool MULTI>
__device__ __forceinline__ const GridK& grid_of_tri(const GridSet& gs, uint32_t t) {
  if constexpr (!MULTI) return gs.g0;
  else return gs.table[__ldg(gs.tri_grid + t)];
}

// (x, y, z) of a local cell index (grid.rs:127-132).
__device__ __forceinline__ void cell_coords(const GridK& g, uint32_t cell, int* x, int* y, int* z) {
  uint32_t q = fdiv(g.div_z, cell);
  *z = (int)(cell - q * (uint32_t)g.n[2]);
  uint32_t xx = fdiv(g.div_y, q);
  *y = (int)(q - xx * (uint32_t)g.n[1]);
  *x = (int)xx;
}

// The bucket schedule every block keeps in shared memory.
struct Sched {
  uint32_t b, B;
  uint32_t slot[kRing];
  uint32_t cur, fp, round, n;
  uint32_t prev_n;  // states of the relax round before this one
  uint32_t steps;   // rounds + redistributions so far
  int action;
};

struct PropState {
  Sched handoff;         // the schedule block 0 leaves after relaxing rounds alone
  uint32_t b;            // current bucket
  uint32_t B;            // window: buckets B .. B + kRing - 1
  uint32_t slot[kRing];  // list holding bucket b + k
  uint32_t cur;          // list relaxed in the current round
  uint32_t fp;           // far list receiving states beyond the window
  uint32_t count[kLists];
  uint32_t far_min[2];   // lowest bucket in each far list
  uint32_t touched2[2];  // touched cells per round parity
  uint32_t done;
  uint32_t overflow;      // a list push did not fit (collection, commit, redistribution)
  uint32_t overflow2[2];  // a spill did not fit, per round parity (propose)
  uint32_t round;
  uint32_t far_phases;
  uint32_t max_list;      // largest bucket list relaxed in one round
  uint32_t log_n;         // steps recorded in the round log
  uint32_t solo_rounds;   // rounds relaxed by block 0 alone
  unsigned long long entries, evals, seeds, ray_hits;
  unsigned long long filter_same;   // proposals dropped: the neighbour holds the proposing triangle
  unsigned long long filter_bound;  // proposals dropped by the distance bound
  // FP64 audit (GridTuning::fp64_audit): ray tests, ambiguous, FP64 decides
  // otherwise; cells whose 2-of-3 vote the FP64 decisions flip; cells whose
  // region was audited (proper triangles), ambiguous, FP64 picks another.
  unsigned long long audit[kAuditStats];
};

__device__ __forceinline__ P3 center(const GridK& g, int x, int y, int z) {
  // grid.rs:135-141: first + (i as f32) * size
  return {fa(g.f[0], fm(__int2float_rn(x), g.s[0])), fa(g.f[1], fm(__int2float_rn(y), g.s[1])),
          fa(g.f[2], fm(__int2float_rn(z), g.s[2]))};
}
__device__ __forceinline__ uint32_t local_index(const GridK& g, int x, int y, int z) {
  return (uint32_t)z + (uint32_t)y * (uint32_t)g.n[2] + (uint32_t)x * ((uint32_t)g.n[1] * (uint32_t)g.n[2]);
}

// Rust `f as isize` (saturating, NaN -> 0).
__device__ __forceinline__ long long sat_i64(float f) {
  if (isnan(f)) return 0;
  if (f >= 9.2233720368547758e18f) return LLONG_MAX;
  if (f <= -9.2233720368547758e18f) return LLONG_MIN;
  return (long long)f;
}
__device__ __forceinline__ unsigned long long sat_u64(float f) {
  if (isnan(f) || f <= 0.0f) return 0;
  if (f >= 1.8446744073709552e19f) return ULLONG_MAX;
  return (unsigned long long)f;
}

// Grid::snap_point_to_grid (grid.rs:145-170), the cell only.
__device__ __forceinline__ void snap(const GridK& g, P3 p, int cell[3]) {
  float pc[3] = {p.x, p.y, p.z};
  for (int d = 0; d < 3; ++d) {
    float bbmin = fs(g.f[d], fm(g.s[d], 0.5f));  // get_bounding_box().0, grid.rs:111
    long long c = sat_i64(floorf(fd(fs(pc[d], bbmin), g.s[d])));
    long long hi = (long long)g.n[d] - 1;
    cell[d] = (int)(c < 0 ? 0 : (c > hi ? hi : c));
  }
}

template <int SIGN>
__device__ __forceinline__ float cell_distance(P3 pos, P3 a, P3 b, P3 c, int kind) {
  if (SIGN == M2S_SIGN_RAYCAST) return fsqrt(point_triangle_distance2_sel(pos, a, b, c, kind));
  return point_triangle_signed_distance_sel(pos, a, b, c, kind);
}

__device__ __forceinline__ unsigned long long pack(float d, uint32_t tri) {
  return ((unsigned long long)__float_as_uint(d) << 32) | ((unsigned long long)tri << 1);
}
__device__ __forceinline__ float key_dist(unsigned long long k) { return __uint_as_float((uint32_t)(k >> 32)); }
__device__ __forceinline__ uint32_t key_tri(unsigned long long k) { return (uint32_t)k >> 1; }

// Does `cand` beat `cur`?  Raycast: plain order of non-negative distances,
// ties to the lower triangle (a proposal's dirty bit never beats the same
// distance and triangle).  Normal: compare_distances (lib.rs:315-332), exact
// ties to the lower triangle; the dirty bit is ignored.
template <int SIGN>
__device__ __forceinline__ bool beats(unsigned long long cand, unsigned long long cur, bool* nan) {
  if (SIGN == M2S_SIGN_RAYCAST) return cand < cur;
  float d = key_dist(cand), o = key_dist(cur);
  int c = compare_distances(d, o, nan);
  return c == -1 || (c == 0 && (uint32_t)(cand >> 32) == (uint32_t)(cur >> 32) && key_tri(cand) < key_tri(cur));
}

// Lowers *slot to cand (a proposal, dirty bit set) if cand beats it; returns
// true when this call lowered a clean key — the cell's first lowering of the
// round, which exactly one proposal per touched cell makes.  `seen` is the
// key as the proposal read it, the first guess of the exchange.
template <int SIGN>
__device__ __forceinline__ bool improve_first(unsigned long long* slot, unsigned long long cand, unsigned long long seen,
                                              bool* nan) {
  if (SIGN == M2S_SIGN_RAYCAST) {
    const unsigned long long old = atomicMin(slot, cand);
    return cand < old && !(old & kDirty);
  }
  unsigned long long old = seen;
  while (beats<SIGN>(cand, old, nan)) {
    unsigned long long prev = atomicCAS(slot, old, cand);
    if (prev == old) return !(old & kDirty);
    old = prev;
  }
  return false;
}

template <int SIGN>
__device__ __forceinline__ bool update_min(unsigned long long* slot, unsigned long long cand, bool* nan) {
  if (SIGN == M2S_SIGN_RAYCAST) return atomicMin(slot, cand) > cand;
  unsigned long long old = *(volatile unsigned long long*)slot;
  while (beats<SIGN>(cand, old, nan)) {
    unsigned long long prev = atomicCAS(slot, old, cand);
    if (prev == old) return true;
    old = prev;
  }
  return false;
}

// ---- the propagation's proposal filter -------------------------------------
// Most proposals cannot win (on the star s6 256^3 grid under 5 % beat the
// cell's key), and a proposal's closest-point evaluation is most of its cost.
// A triangle lies in its plane and, inside that plane, on the inner side of
// each of its three edge lines, so the distance from p to the triangle is at
// least sqrt(h^2 + o^2), where h is p's distance to the plane and o the
// largest distance of p's projection outside an edge line.  A proposal whose
// bound already exceeds the key's distance by a slack far above the
// rounding of both computations cannot beat the key (for Normal: not
// even enter compare_distances' tie band), so it is dropped unevaluated.
// Results are unchanged; the filter only skips work whose outcome is known.
//
// TriBound: n = unit normal, n.w = n . a; e0, e1, e2 = unit in-plane normals
// of the edges ab, bc, ca pointing into the triangle, .w = e . (the edge's
// first vertex).  Built in double from the exact f32 vertices.
struct __align__(16) TriBound {
  float4 n, e0, e1, e2;
};
// Slack of the test, relative to the key's distance and per unit of the
// largest coordinate magnitude involved (the point's and the triangle's: the
// f32 closest-point arithmetic errs by a few ulps of these; the slack is
// about a thousand times that).
constexpr float kBoundRel = 1.0f / 65536.0f;
constexpr double kBoundAbs = 1.0 / 16384.0;
// Triangles whose area is tiny against their longest edge (slivers: the
// reference's region tests lose accuracy there) and degenerate ones are never
// filtered: their record is zero and their slack infinite.
constexpr double kBoundMinShape = 1e-4;

__global__ void k_bounds(const TriRec* __restrict__ tris, uint32_t T, TriBound* __restrict__ out,
                         float* __restrict__ slack) {
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x) {
    const TriRec r = tris[t];
    const double ax = r.a.x, ay = r.a.y, az = r.a.z, bx = r.b.x, by = r.b.y, bz = r.b.z;
    const double cx = r.c.x, cy = r.c.y, cz = r.c.z;
    const double abx = bx - ax, aby = by - ay, abz = bz - az, acx = cx - ax, acy = cy - ay, acz = cz - az;
    const double bcx = cx - bx, bcy = cy - by, bcz = cz - bz;
    const double nx = aby * acz - abz * acy, ny = abz * acx - abx * acz, nz = abx * acy - aby * acx;
    const double nn = sqrt(nx * nx + ny * ny + nz * nz);
    const double lab = sqrt(abx * abx + aby * aby + abz * abz), lac = sqrt(acx * acx + acy * acy + acz * acz);
    const double lbc = sqrt(bcx * bcx + bcy * bcy + bcz * bcz);
    const double emax = fmax(lab, fmax(lac, lbc));
    const double vmax = fmax(fmax(fmax(fabs(ax), fabs(ay)), fmax(fabs(az), fabs(bx))),
                             fmax(fmax(fabs(by), fabs(bz)), fmax(fmax(fabs(cx), fabs(cy)), fabs(cz))));
    const double scale = vmax + emax;
    const bool ok = __float_as_int(r.a.w) == 0 && isfinite(scale) && scale < 1e18 && emax > 0.0 &&
                    nn > kBoundMinShape * emax * emax;
    if (!ok) {
      const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
      out[t] = TriBound{z, z, z, z};
      slack[t] = __int_as_float(0x7F800000);  // +inf: never filtered
      continue;
    }
    const double ux = nx / nn, uy = ny / nn, uz = nz / nn;
    // In-plane normal of edge (p, q) toward the third vertex: u x (q - p) / |q - p|
    // (u = ab x ac / |ab x ac|, so u x ab points from ab toward c, and so on).
    auto edge = [&](double px, double py, double pz, double dx, double dy, double dz, double len) {
      const double mx = (uy * dz - uz * dy) / len, my = (uz * dx - ux * dz) / len, mz = (ux * dy - uy * dx) / len;
      return make_float4((float)mx, (float)my, (float)mz, (float)(mx * px + my * py + mz * pz));
    };
    TriBound b;
    b.n = make_float4((float)ux, (float)uy, (float)uz, (float)(ux * ax + uy * ay + uz * az));
    b.e0 = edge(ax, ay, az, abx, aby, abz, lab);
    b.e1 = edge(bx, by, bz, bcx, bcy, bcz, lbc);
    b.e2 = edge(cx, cy, cz, -acx, -acy, -acz, lac);
    out[t] = b;
    slack[t] = (float)(kBoundAbs * scale);
  }
}

// True when triangle `tb` (slack `sl`) provably cannot beat the cell key
// `snap` at the cell centre p.
template <int SIGN>
__device__ __forceinline__ bool bound_rejects(const TriBound& tb, float sl, P3 p, unsigned long long snap) {
  const float h = fmaf(tb.n.x, p.x, fmaf(tb.n.y, p.y, fmaf(tb.n.z, p.z, -tb.n.w)));
  const float s0 = fmaf(tb.e0.x, p.x, fmaf(tb.e0.y, p.y, fmaf(tb.e0.z, p.z, -tb.e0.w)));
  const float s1 = fmaf(tb.e1.x, p.x, fmaf(tb.e1.y, p.y, fmaf(tb.e1.z, p.z, -tb.e1.w)));
  const float s2 = fmaf(tb.e2.x, p.x, fmaf(tb.e2.y, p.y, fmaf(tb.e2.z, p.z, -tb.e2.w)));
  const float o = fmaxf(0.0f, -fminf(s0, fminf(s1, s2)));
  const float lb2 = fmaf(h, h, o * o);
  const float pm = fmaxf(fabsf(p.x), fmaxf(fabsf(p.y), fabsf(p.z)));
  float thr = fmaf(fabsf(key_dist(snap)), 1.0f + kBoundRel, fmaf((float)kBoundAbs, pm, sl));
  if (SIGN == M2S_SIGN_NORMAL) thr += 1e-6f;  // compare_distances' absolute tie band (lib.rs:321)
  return lb2 > thr * thr;                     // false when thr is infinite or anything is NaN
}

__global__ void k_fill_u64(unsigned long long* p, unsigned long long n, unsigned long long v) {
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x)
    p[i] = v;
}

// Batch triangle array: triangle t of the job is triangle t - tri_off[k] of
// mesh k.  Keys store the job-wide index, which keeps each mesh's triangle
// order, so ties resolve exactly as for the mesh alone.
__global__ void k_gather_tris(const TriRec* const* __restrict__ src, const uint32_t* __restrict__ tri_off,
                              uint32_t ngrids, uint32_t T, TriRec* __restrict__ out, uint32_t* __restrict__ tri_grid) {
  SegCursor<uint32_t> sc;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x) {
    const uint32_t k = sc.at(tri_off, ngrids, t);
    out[t] = src[k][t - tri_off[k]];
    tri_grid[t] = k;
  }
}

// ---- 1. seeding -------------------------------------------------------------
template <int SIGN, bool MULTI>
__global__ void k_seed(const __grid_constant__ GridSet gs, const TriRec* __restrict__ tris, uint32_t T,
                       unsigned long long* keys, uint32_t* status, PropState* st) {
  const uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (t >= T) return;
  const GridK& g = grid_of_tri<MULTI>(gs, t);
  TriRec r = tris[t];
  P3 a = p3(r.a), b = p3(r.b), c = p3(r.c);
  int kind = __float_as_int(r.a.w);
  P3 lo, hi;
  padded_box(a, b, c, &lo, &hi);  // grid.rs:400
  int mn[3], mx[3];
  snap(g, lo, mn);
  snap(g, hi, mx);
  // grid.rs:410-426: widen by one cell where the box pokes past a centre.
  P3 mnf = center(g, mn[0], mn[1], mn[2]);
  P3 mxf = center(g, mx[0], mx[1], mx[2]);
  for (int d = 0; d < 3; ++d) {
    if (mn[d] > 0 && vget(mnf, d) > vget(lo, d)) mn[d] -= 1;
    if (mx[d] < g.n[d] - 1 && vget(mxf, d) < vget(hi, d)) mx[d] += 1;
  }
  long long ex = mx[0] - mn[0] + 1, ey = mx[1] - mn[1] + 1, ez = mx[2] - mn[2] + 1;
  if (ex <= 0 || ey <= 0 || ez <= 0) return;
  long long total = ex * ey * ez;
  bool nan = false;
  uint32_t updates = 0;
  auto visit = [&](int x, int y, int z) {
    float d = cell_distance<SIGN>(center(g, x, y, z), a, b, c, kind);
    if (isnan(d)) nan = true;
    if (update_min<SIGN>(&keys[g.cell_off + local_index(g, x, y, z)], pack(d, t), &nan)) ++updates;
  };
  if (total <= 0x7FFFFFFFll) {  // 32-bit division (64-bit costs ~4x the instructions)
    const uint32_t uez = (uint32_t)ez, uey = (uint32_t)ey, utotal = (uint32_t)total;
    for (uint32_t k = lane; k < utotal; k += 32) {
      const uint32_t q = k / uez, xq = q / uey;
      visit(mn[0] + (int)xq, mn[1] + (int)(q - xq * uey), mn[2] + (int)(k - q * uez));
    }
  } else {
    for (long long k = lane; k < total; k += 32)
      visit(mn[0] + (int)(k / (ez * ey)), mn[1] + (int)((k / ez) % ey), mn[2] + (int)(k % ez));
  }
  if (nan) atomicOr(status, bit(M2S_ERR_NAN_DISTANCE));
  for (int o = 16; o; o >>= 1) updates += __shfl_xor_sync(0xFFFFFFFFu, updates, o);
  if (lane == 0 && updates) atomicAdd(&st->seeds, (unsigned long long)updates);
}

// Distance bucket of a state, in its own grid's cell units: u = |d| / (a
// quarter of the smallest cell size).  Buckets are one unit wide up to u = 32
// (8 cells) and beyond grow with the distance — kLogBuckets per doubling of u,
// from the piecewise-linear log2 that the f32 bit pattern gives (exponent,
// then mantissa) — so the far field, where many triangles are nearly
// equidistant, takes few rounds.  Everything after the one rounded product is
// integer arithmetic, so every kernel files a state under the same bucket.
constexpr float kLinearBuckets = 32.0f;
constexpr uint64_t kLogBuckets = 22;
__device__ __forceinline__ uint32_t bucket_of(float inv_delta, float d) {
  const float u = __fmul_rn(fabsf(d), inv_delta);
  if (isnan(u)) return 0;  // a NaN distance is already an error
  if (u <= kLinearBuckets) return (uint32_t)u;  // floor, u >= 0
  const uint32_t b = __float_as_uint(u);   // u > 32: exponent >= 5; +inf has exponent 128
  const uint64_t lin = ((uint64_t)((b >> 23) - 127 - 5) << 23) | (b & 0x7FFFFFu);
  return 32u + (uint32_t)((kLogBuckets * lin) >> 23);
}

__global__ void k_state_init(PropState* st) {
  st->b = 0;
  st->B = 0;
  for (int k = 0; k < kRing; ++k) st->slot[k] = k;
  st->cur = kCur0;
  st->fp = 0;
  st->far_min[0] = st->far_min[1] = kNoBucket;
}

// Appends (cell, triangle) of bucket nb: inside the window to its bucket's list
// (buckets at or below the current one to the list relaxed next), beyond it to
// the far list fp.  Lanes of a warp that target the same list share one
// atomicAdd.  Must be called by all 32 lanes; `act` says whether this lane pushes.
// Where the list counts, far-list minima and the push-overflow flag live: in
// PropState (global), or in block 0's shared memory during a solo run.
struct Counters {
  uint32_t* count;     // kLists
  uint32_t* far_min;   // 2
  uint32_t* overflow;  // push overflow
};
__device__ __forceinline__ Counters global_counters(PropState* st) { return {st->count, st->far_min, &st->overflow}; }

__device__ __forceinline__ void push_entry_warp(const Counters& ct, uint32_t b, uint32_t B, const uint32_t* slots,
                                                uint32_t fp, uint2* lists, uint32_t cap, bool act, uint32_t cell,
                                                uint32_t tri, uint32_t nb) {
  const int lane = threadIdx.x & 31;
  const bool far = act && nb >= B + kRing;
  uint32_t slot = 0xFFFFFFFFu;
  if (act) slot = far ? (uint32_t)kFar0 + fp : slots[nb > b ? nb - b : 0];
  const uint32_t farmask = __ballot_sync(0xFFFFFFFFu, far);
  if (farmask) {
    const uint32_t m = __reduce_min_sync(0xFFFFFFFFu, far ? nb : kNoBucket);
    if (lane == __ffs(farmask) - 1) atomicMin(&ct.far_min[fp], m);
  }
  const uint32_t group = __match_any_sync(0xFFFFFFFFu, slot);
  if (!act) return;
  const int leader = __ffs(group) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(&ct.count[slot], (uint32_t)__popc(group));
  base = __shfl_sync(group, base, leader);
  const uint32_t pos = base + __popc(group & ((1u << lane) - 1u));
  if (pos < cap)
    lists[(unsigned long long)slot * cap + pos] = make_uint2(cell, tri);
  else
    atomicOr(ct.overflow, 1u);  // the job is rerun with larger lists
}

// Initial states: every seeded cell with its seed triangle (window 0..15).
template <bool MULTI>
__global__ void k_collect(const __grid_constant__ GridSet gs, const unsigned long long* keys, PropState* st,
                          uint2* lists, uint32_t cap) {
  SegCursor<uint32_t> sc;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long base = (unsigned long long)blockIdx.x * blockDim.x; base < gs.ncell; base += stride) {
    const unsigned long long i = base + threadIdx.x;  // warp-uniform loop, lanes mask out past the end
    const unsigned long long k = i < gs.ncell ? keys[i] : KEY_EMPTY;
    const bool act = key_tri(k) != NO_TRI;
    uint32_t nb = 0;
    if (act) {
      const float inv = MULTI ? gs.table[sc.at(gs.cell_off, gs.ngrids, (uint32_t)i)].inv_delta : gs.g0.inv_delta;
      nb = bucket_of(inv, key_dist(k));
    }
    push_entry_warp(global_counters(st), 0, 0, st->slot, 0, lists, cap, act, (uint32_t)i, key_tri(k), nb);
  }
}

// ---- 2. relaxation (one persistent cooperative launch) -------------------------
// Every block keeps an identical copy of the bucket schedule in shared memory
// and advances it from the global list counts after each grid barrier, so no
// block waits for a scheduler.
//
// One arrival counter for every barrier of a launch: a block adds 1 when it
// arrives at its g-th barrier and passes once the counter has reached
// g x blocks.  The counter is never reset, so nothing but the last arrival
// stands between the blocks and the release (arrival and wait are a
// fire-and-forget add and polls of one word), and comparisons are by signed
// difference, which stays right when the counter wraps: while a block waits
// at barrier g, barrier g - 1 is complete and no block is past g + 1, so
// its difference stays inside (-blocks, blocks).
constexpr unsigned int kMaxBarrierBlocks = 2048;
struct GridBarrier {
  unsigned int arrivals;
  unsigned int abort;
  unsigned int pad0[30];
};

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Barrier over the co-resident blocks of a cooperative launch.  Every block
// passes the same sequence of barriers, so each keeps its barrier count g in
// shared memory and waits for the arrivals to reach g x blocks.  A wait spins
// briefly, then backs off with __nanosleep so waiting blocks leave the memory
// system to the ones working (block 0 alone during a solo run).  It is bounded
// in time: after kBarrierTimeoutNs it gives up, and every block leaves the
// kernel at its next barrier (kAbortOffset below).
constexpr uint64_t kBarrierTimeoutNs = 2000000000ull;  // two seconds
constexpr uint32_t kBarrierSpins = 64;

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void red_add_release(unsigned int* p, unsigned int v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
// The first block to give up adds kAbortOffset to the counter once (the
// abort word picks that block): every later wait, in any barrier of the
// launch, then sees a difference of about 2^30 and leaves as well.
constexpr unsigned int kAbortOffset = 1u << 30;
__device__ __forceinline__ bool grid_barrier(GridBarrier* bar, unsigned int nblocks, unsigned int* gen) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int target = (*gen + 1u) * nblocks;
    red_add_release(&bar->arrivals, 1u);
    uint32_t polls = 0;
    uint64_t t0 = 0;
    int pass = 1;
    for (;;) {
      const int diff = (int)(ld_acquire(&bar->arrivals) - target);
      if (diff >= (int)(kAbortOffset >> 2)) {
        pass = 0;
        break;
      }
      if (diff >= 0) break;
      if (++polls < kBarrierSpins) continue;
      if (polls == kBarrierSpins) t0 = global_ns();
      __nanosleep(256);
      if (global_ns() - t0 > kBarrierTimeoutNs) {
        if (atomicExch(&bar->abort, 1u) == 0u) atomicAdd(&bar->arrivals, kAbortOffset);
        pass = 0;
        break;
      }
    }
    *gen = *gen + 1u;
    ok = pass;
  }
  __syncthreads();
  return ok != 0;
}

// Diagnostics of the barrier's bound: the launched blocks wait at one grid
// barrier that expects `expected` blocks.  With fewer launched, no block is
// the last to arrive, every wait gives up after kBarrierTimeoutNs and the
// abort flag is raised; result[0] counts blocks that passed, result[1] blocks
// that gave up.
__global__ void k_barrier_probe(GridBarrier* bar, unsigned int expected, unsigned int* result) {
  __shared__ unsigned int gen;
  if (threadIdx.x == 0) gen = 0;
  const bool ok = grid_barrier(bar, expected, &gen);
  if (threadIdx.x == 0) atomicAdd(&result[ok ? 0 : 1], 1u);
}

// Touched cells staged per block and round in shared memory; a block commits
// the cells it touched itself, so only a block whose stage fills up writes to
// the global spill list.
constexpr int kTouchStage = 6144;
constexpr int kUnroll = 2;  // proposals per thread in flight


enum { kRelax = 0, kRedistribute = 1, kDone = 2, kLimit = 3 };

// Next step of the schedule, computed by warp 0 of every block from the
// global list counts (final at this point: the last grid barrier ordered every
// push before it): lane k reads the count of the list of bucket b + k, all in
// one round trip, and the lanes rotate the ring by shuffles.  Block 0 also
// empties the list relaxed last round, which no block reads here and which
// receives pushes only after the next barrier.  Every lane returns the action.
__device__ __forceinline__ int next_step(Sched& sh, const Counters& ct, uint32_t spill_overflow, bool leader) {
  const int lane = threadIdx.x & 31;
  const uint32_t my_slot = lane < kRing ? sh.slot[lane] : 0u;
  const uint32_t c = lane < kRing ? *(volatile uint32_t*)&ct.count[my_slot] : 0u;
  // Bit k: the list of bucket b + k holds states (bits past the window's end cleared).
  uint32_t nonempty = __ballot_sync(0xFFFFFFFFu, lane < kRing && c != 0u);
  const uint32_t b = sh.b, B = sh.B, fp = sh.fp, cur = sh.cur;
  const uint32_t left = B + kRing - b;  // buckets b .. B + kRing - 1 lie in the window
  if (left < kRing) nonempty &= (1u << left) - 1u;
  // Only values no block can change before every block has passed this step:
  // list counts (pushes come after the next barrier), the push overflow flag
  // and the spill overflow flag of the round just finished (the next propose
  // phase writes the other parity).
  const uint32_t overflow = *(volatile uint32_t*)ct.overflow | spill_overflow;
  const uint32_t far_n = *(volatile uint32_t*)&ct.count[kFar0 + fp];
  const uint32_t far_b = *(volatile uint32_t*)&ct.far_min[fp];
  __syncwarp();  // every lane has read the schedule before it changes
  if (overflow) return kDone;
  if (nonempty) {
    // slot[k] holds bucket b + k; advance b to the first non-empty bucket q.
    const int q = __ffs(nonempty) - 1;
    const uint32_t nq = __shfl_sync(0xFFFFFFFFu, c, q);
    const uint32_t moved = __shfl_sync(0xFFFFFFFFu, my_slot, (lane + q) & (kRing - 1));
    if (lane < kRing) sh.slot[lane] = lane == 0 ? cur : moved;  // slot 0: the consumed list, re-queued at b
    if (lane == 0) {
      sh.cur = moved;
      sh.b = b + q;
      sh.prev_n = sh.n;
      sh.n = nq;
      sh.round += 1;
      if (leader) ct.count[cur] = 0;
    }
    __syncwarp();
    return kRelax;
  }
  // Every window list is empty.  Far states all lie at or beyond B + kRing, so
  // the new window starts at the lowest of them.
  if (far_n == 0) return kDone;
  if (lane == 0) sh.B = sh.b = far_b;
  __syncwarp();
  return kRedistribute;
}

// Rounds of at most solo_max states are relaxed by block 0 alone, with block
// barriers only, while the other blocks wait at one grid barrier: a grid-wide
// round costs two grid barriers and the slowest block, far more than relaxing
// a few states.  Far-field tails and lateral spreading along a surface make
// long chains of such rounds.  A solo run lasts at most kSoloRounds rounds so
// the waiting blocks' bounded wait always ends.  The work of a round does not
// depend on which threads do it: results are the same either way.
constexpr uint32_t kSoloRounds = 1024;  // the threshold (default 64 states) is GridTuning::solo_max
constexpr uint32_t kSoloCap = 64;  // largest solo_max
// A run starts at the second small round in a row: an isolated small round
// (a lull between large ones) costs more as a run of one, which adds a
// barrier's wait for the other blocks and the schedule handoff, than on every
// block (star s6 256^3: 10.12 -> 9.94 ms; star s4 96^3: 1.72 -> 1.57 ms),
// while chains of small rounds still run alone (terrain 384x384x128 Normal:
// 23.7 -> 23.3 ms).  Every block decides from the same schedule.
__device__ __forceinline__ bool solo_round(const Sched& sh, uint32_t solo_max) {
  return sh.n <= solo_max && sh.prev_n <= solo_max;
}

// Queue of one warp's proposals that need a distance evaluation (Normal sign).
constexpr uint32_t kQueue = 64;
struct WarpQueue {
  uint32_t tri[kQueue], j[kQueue];
  float px[kQueue], py[kQueue], pz[kQueue];  // the neighbour's cell centre
  unsigned long long snap[kQueue];
};
constexpr int kWarps = 8;  // k_propagate runs 256 threads per block

// Stages cell j, whose first lowering of the round this proposal made, for the
// block's commit (spilling to the round's global list when the stage is full).
__device__ __forceinline__ void stage_touch(uint32_t j, uint32_t* s_touch, uint32_t* s_ntouch, PropState* st,
                                            uint32_t parity, uint32_t* spill, uint32_t cap) {
  const uint32_t q = atomicAdd(s_ntouch, 1u);
  if (q < kTouchStage) {
    s_touch[q] = j;
  } else {
    const uint32_t pos = atomicAdd(&st->touched2[parity], 1u);
    if (pos < cap) spill[pos] = j;
    else atomicOr(&st->overflow2[parity], 1u);
  }
}

// Neighbour kk (0..25, the cell itself skipped) of the state with entry ent:
// its coordinates and index j; false when it lies off the grid.
template <bool MULTI>
__device__ __forceinline__ bool neighbour_cell(const GridSet& gs, uint2 ent, uint32_t kk, uint32_t& j, int& X, int& Y,
                                               int& Z) {
  const GridK& g = grid_of_tri<MULTI>(gs, ent.y);
  int x, y, z;
  cell_coords(g, ent.x - g.cell_off, &x, &y, &z);
  // iproduct!(-1..=1, -1..=1, -1..=1) order (grid.rs:512): x outermost; 13 is the cell itself.
  const uint32_t ku = kk + (kk >= 13u);
  X = x + (int)(ku / 9u) - 1;
  Y = y + (int)((ku / 3u) % 3u) - 1;
  Z = z + (int)(ku % 3u) - 1;
  if ((unsigned)X >= (unsigned)g.n[0] || (unsigned)Y >= (unsigned)g.n[1] || (unsigned)Z >= (unsigned)g.n[2])
    return false;
  j = g.cell_off + local_index(g, X, Y, Z);
  return true;
}

// Distance of triangle tri (record r) at cell j, centre pos, against the
// cell's key as read (`seen`); true when this proposal made the cell's first
// lowering of the round (it is then the cell's one staging proposal).
template <int SIGN>
__device__ __forceinline__ bool propose_dist(float d, uint32_t tri, uint32_t j, unsigned long long seen,
                                             unsigned long long* keys, bool& nan) {
  if (isnan(d)) nan = true;
  const unsigned long long cand = pack(d, tri) | kDirty;
  return beats<SIGN>(cand, seen, &nan) && improve_first<SIGN>(&keys[j], cand, seen, &nan);
}
template <int SIGN>
__device__ __forceinline__ bool propose_at(const TriRec& r, uint32_t tri, uint32_t j, P3 pos, unsigned long long seen,
                                           unsigned long long* keys, bool& nan) {
  return propose_dist<SIGN>(cell_distance<SIGN>(pos, p3(r.a), p3(r.b), p3(r.c), __float_as_int(r.a.w)), tri, j, seen,
                            keys, nan);
}

// A solo round (block 0 alone, n <= kSoloCap states) forms the round's minima
// in a table in shared memory instead of in the keys: a proposal that beats
// its cell's key meets the cell's other proposals in the cell's slot (open
// addressing, linear probing; at most 26 * kSoloCap cells ever take a slot,
// fewer than kHash), and the commit writes each slot's winner to the key.
// The round saves the key atomic and the commit's read of it: two dependent
// trips to L2 of the few a solo round waits for.  The table occupies the
// block's touch stage, free in a solo run.
constexpr uint32_t kHash = 2048;
constexpr uint32_t kNoCell = 0xFFFFFFFFu;
static_assert(26 * kSoloCap < kHash, "a solo round could fill the table");
static_assert(kHash * 3 <= (uint32_t)kTouchStage, "the table exceeds the touch stage");

__device__ __forceinline__ uint32_t hash_slot(uint32_t j) { return (j * 2654435761u) >> 21; }  // 11 bits

// Lowers cell j's slot to cand (which beats the cell's key) if it beats the
// slot's value; a slot taken here is listed for the commit.  Slots start as
// (kNoCell, KEY_EMPTY); every candidate that beats a key beats KEY_EMPTY too,
// the order being a total one.  Solo candidates are clean keys.
template <int SIGN>
__device__ __forceinline__ void table_improve(uint32_t* HJ, unsigned long long* HK, uint16_t* taken,
                                              uint32_t* ntaken, uint32_t j, unsigned long long cand, bool& nan) {
  uint32_t h = hash_slot(j);
  for (uint32_t probe = 0; probe < kHash; ++probe) {  // ends at a free slot: fewer cells than slots
    const uint32_t cur = atomicCAS(&HJ[h], kNoCell, j);
    if (cur == kNoCell) taken[atomicAdd(ntaken, 1u)] = (uint16_t)h;
    if (cur == kNoCell || cur == j) {
      if (SIGN == M2S_SIGN_RAYCAST) {
        atomicMin(&HK[h], cand);
      } else {
        unsigned long long old = *(volatile unsigned long long*)&HK[h];
        while (beats<SIGN>(cand, old, &nan)) {
          const unsigned long long prev = atomicCAS(&HK[h], old, cand);
          if (prev == old) break;
          old = prev;
        }
      }
      return;
    }
    h = (h + 1) & (kHash - 1);
  }
}

// Propose phase of a solo round: one thread per (state, neighbour) proposal.
// A neighbour that holds the state's triangle already cannot gain.
template <int SIGN, bool MULTI>
__device__ __forceinline__ void relax_propose_solo(const GridSet& gs, const TriRec* __restrict__ tris,
                                                   const unsigned long long* keys, const uint2* list, uint32_t n,
                                                   uint32_t* HJ, unsigned long long* HK, uint16_t* taken,
                                                   uint32_t* ntaken, bool& nan, unsigned long long& evals,
                                                   uint32_t& dropped_same) {
  const uint32_t P = 26u * n;
  for (uint32_t p = threadIdx.x; p < P; p += blockDim.x) {
    const uint2 ent = __ldcg(&list[p / 26u]);  // written by other blocks in earlier rounds
    uint32_t j;
    int X, Y, Z;
    if (!neighbour_cell<MULTI>(gs, ent, p % 26u, j, X, Y, Z)) continue;
    ++evals;
    const unsigned long long snap = __ldcg(&keys[j]);
    const TriRec r = tris[ent.y];
    if (key_tri(snap) == ent.y) {
      ++dropped_same;
      continue;
    }
    const GridK& g = grid_of_tri<MULTI>(gs, ent.y);
    const float d = cell_distance<SIGN>(center(g, X, Y, Z), p3(r.a), p3(r.b), p3(r.c), __float_as_int(r.a.w));
    if (isnan(d)) nan = true;
    const unsigned long long cand = pack(d, ent.y);
    if (beats<SIGN>(cand, snap, &nan)) table_improve<SIGN>(HJ, HK, taken, ntaken, j, cand, nan);
  }
}

// Commit phase of a solo round: every taken slot's winner becomes the cell's
// key and is queued under its bucket; the slot is freed.
template <bool MULTI>
__device__ __forceinline__ void relax_commit_solo(const GridSet& gs, unsigned long long* keys, uint32_t* HJ,
                                                  unsigned long long* HK, const uint16_t* taken, uint32_t ntaken,
                                                  const Counters& ct, const Sched& sh, uint2* lists, uint32_t cap) {
  for (uint32_t base = 0; base < ntaken; base += blockDim.x) {  // warp-uniform trip count
    const uint32_t i = base + threadIdx.x;
    const bool act = i < ntaken;
    uint32_t j = 0, nb = 0;
    unsigned long long w = KEY_EMPTY;
    if (act) {
      const uint32_t h = taken[i];
      j = HJ[h];
      w = HK[h];
      keys[j] = w;
      nb = bucket_of(grid_of_tri<MULTI>(gs, key_tri(w)).inv_delta, key_dist(w));
      HJ[h] = kNoCell;
      HK[h] = KEY_EMPTY;
    }
    push_entry_warp(ct, sh.b, sh.B, sh.slot, sh.fp, lists, cap, act, j, key_tri(w), nb);
  }
}

// Propose phase of a relax round over list[0..n): every state offers its
// triangle to the 26 cells around it (its own cell holds that triangle's
// distance or a better one, so it never gains).  Results do not depend on
// how proposals are shared out or ordered, nor on the filter below.
//
// With the filter (the default), a proposal is dropped unevaluated when the
// neighbour already holds the same triangle (the distance of a (cell,
// triangle) pair is one deterministic value, so it cannot gain) or when the
// triangle's distance bound proves that it cannot beat the cell's key; each
// warp queues the rest in shared memory and evaluates them 32 at a time with
// every lane busy.  The work unit is a row: state e and a (dx, dy) offset, the
// three neighbours at z - 1, z, z + 1 (nine rows per state; the state's own
// cell is left out of its row).  A row's three keys are adjacent, so
// a thread issues their loads together and they share a memory sector; the
// bound's plane values are formed once at the row's middle cell and moved
// along z by one addition each (the slack covers that rounding); only a
// survivor's exact cell centre is computed.  Units t0, t0 + T, ... advance as
// (state, row) pairs without division: T = 9 * dE + dR.
//
// Without the filter, Raycast proposals are evaluated where they arise.  In a
// round of at least two row units per thread (9 n >= 2 T) the unit is a row as
// above: one entry load, one coordinate decode and one triangle record serve
// its three proposals, and the three keys are loaded together.  Smaller rounds
// keep single (state, neighbour) pairs, T = 26 * dE + dK, kUnroll per thread at
// a time, so that more threads share the round's few states.  Normal
// proposals are single pairs that pass the same-triangle test and the queue.
template <int SIGN, bool MULTI, bool FILTER>
__device__ __forceinline__ void relax_propose(const GridSet& gs, const TriRec* __restrict__ tris,
                                              const TriBound* __restrict__ bounds, const float* __restrict__ slack,
                                              unsigned long long* keys, const uint2* list, uint32_t n,
                                              uint32_t T, uint32_t t0, uint32_t* s_touch, uint32_t* s_ntouch,
                                              PropState* st, uint32_t parity, uint32_t* spill, uint32_t cap,
                                              bool& nan, unsigned long long& evals, uint32_t& dropped_same,
                                              uint32_t& dropped_bound, WarpQueue* q) {
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t qn = 0;  // warp-uniform queue length, < 32 between pushes
  auto run = [&](uint32_t i) {
    const uint32_t tri = q->tri[i], j = q->j[i];
    if (propose_at<SIGN>(tris[tri], tri, j, P3{q->px[i], q->py[i], q->pz[i]}, q->snap[i], keys, nan))
      stage_touch(j, s_touch, s_ntouch, st, parity, spill, cap);
  };
  // Called by all 32 lanes: queues this lane's proposal if `keep`, and
  // evaluates 32 queued proposals once there are that many.
  auto queue_push = [&](bool keep, uint32_t tri, uint32_t j, P3 pos, unsigned long long snap) {
    const unsigned m = __ballot_sync(0xFFFFFFFFu, keep);
    if (keep) {
      const uint32_t w = qn + __popc(m & ((1u << lane) - 1u));  // qn + 31 at most
      q->tri[w] = tri;
      q->j[w] = j;
      q->px[w] = pos.x;
      q->py[w] = pos.y;
      q->pz[w] = pos.z;
      q->snap[w] = snap;
    }
    qn += __popc(m);
    if (qn >= 32u) {
      __syncwarp();
      run(qn - 32u + lane);
      __syncwarp();  // the slots are written again by the next push
      qn -= 32u;
    }
  };
  if constexpr (FILTER) {
    const uint32_t dE = T / 9u, dR = T % 9u;
    uint32_t e = t0 / 9u, r = t0 % 9u;
    // The entry of a thread's next unit is loaded while it works on the
    // current one (entries were written by other blocks in earlier rounds).
    uint2 ent_next = e < n ? __ldcg(&list[e]) : make_uint2(0u, 0u);
    while (__any_sync(0xFFFFFFFFu, e < n)) {
      const uint32_t eu = e, ru = r;
      const uint2 ent = ent_next;
      r += dR;
      e += dE;
      if (r >= 9u) {
        r -= 9u;
        ++e;
      }
      if (e < n) ent_next = __ldcg(&list[e]);
      bool on[3] = {false, false, false};
      uint32_t tri = 0, j0 = 0;
      int X = 0, Y = 0, z = 0;
      unsigned long long snap[3] = {0ull, 0ull, 0ull};
      const GridK* gp = nullptr;
      if (eu < n) {
        tri = ent.y;
        const GridK& g = grid_of_tri<MULTI>(gs, tri);
        gp = &g;
        int x, y;
        cell_coords(g, ent.x - g.cell_off, &x, &y, &z);
        X = x + (int)(ru / 3u) - 1;  // iproduct order (grid.rs:512): x outermost
        Y = y + (int)(ru % 3u) - 1;
        if ((unsigned)X < (unsigned)g.n[0] && (unsigned)Y < (unsigned)g.n[1]) {
          j0 = g.cell_off + local_index(g, X, Y, z);
          on[0] = z > 0;
          on[1] = ru != 4u;  // the state's own cell
          on[2] = z + 1 < g.n[2];
#pragma unroll
          for (int d = 0; d < 3; ++d)
            if (on[d]) snap[d] = __ldcg(&keys[j0 + d - 1]);
        }
      }
      bool keep[3] = {false, false, false};
      if (on[0] || on[1] || on[2]) {
        const GridK& g = *gp;
        const TriBound tb = bounds[tri];
        const float sl = slack[tri];
        // the bound's plane values at the row's middle cell, and their step along z
        const P3 pc = center(g, X, Y, z);
        const float fh = fmaf(tb.n.x, pc.x, fmaf(tb.n.y, pc.y, fmaf(tb.n.z, pc.z, -tb.n.w)));
        const float f0 = fmaf(tb.e0.x, pc.x, fmaf(tb.e0.y, pc.y, fmaf(tb.e0.z, pc.z, -tb.e0.w)));
        const float f1 = fmaf(tb.e1.x, pc.x, fmaf(tb.e1.y, pc.y, fmaf(tb.e1.z, pc.z, -tb.e1.w)));
        const float f2 = fmaf(tb.e2.x, pc.x, fmaf(tb.e2.y, pc.y, fmaf(tb.e2.z, pc.z, -tb.e2.w)));
        const float sz = g.s[2];
        const float ph = tb.n.z * sz, p0 = tb.e0.z * sz, p1 = tb.e1.z * sz, p2 = tb.e2.z * sz;
        const float pm = fmaxf(fmaxf(fabsf(pc.x), fabsf(pc.y)), fabsf(pc.z)) + fabsf(sz);
        const float base = fmaf((float)kBoundAbs, pm, sl) + (SIGN == M2S_SIGN_NORMAL ? 1e-6f : 0.0f);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          if (!on[d]) continue;
          ++evals;
          if (key_tri(snap[d]) == tri) {
            ++dropped_same;
            continue;
          }
          const float sd = (float)(d - 1);
          const float h = fmaf(sd, ph, fh);
          const float o = fmaxf(0.0f, -fminf(fmaf(sd, p0, f0), fminf(fmaf(sd, p1, f1), fmaf(sd, p2, f2))));
          const float thr = fmaf(fabsf(key_dist(snap[d])), 1.0f + kBoundRel, base);
          if (fmaf(h, h, o * o) > thr * thr) {  // false when thr is infinite or anything is NaN
            ++dropped_bound;
            continue;
          }
          keep[d] = true;
        }
      }
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        P3 pos{0.f, 0.f, 0.f};
        if (keep[d]) pos = center(*gp, X, Y, z + d - 1);
        queue_push(keep[d], tri, j0 + d - 1, pos, snap[d]);
      }
    }
  } else {
    const uint32_t dE = T / 26u, dK = T % 26u;
    uint32_t e = t0 / 26u, k = t0 % 26u;
    // The neighbour of state e for proposal k: false when it lies off the grid.
    auto neighbour = [&](uint32_t eu, uint32_t kk, uint32_t& tri, uint32_t& j, int& X, int& Y, int& Z) {
      const uint2 ent = __ldcg(&list[eu]);  // written by other blocks in earlier rounds
      tri = ent.y;
      return neighbour_cell<MULTI>(gs, ent, kk, j, X, Y, Z);
    };
    auto step = [&]() {
      k += dK;
      e += dE;
      if (k >= 26u) {
        k -= 26u;
        ++e;
      }
    };
    if (SIGN == M2S_SIGN_RAYCAST && 9u * n >= 2u * T) {
      const uint32_t dR = T / 9u, dRr = T % 9u;
      uint32_t er = t0 / 9u, rr = t0 % 9u;
      while (er < n) {
        const uint32_t eu = er, row = rr;
        rr += dRr;
        er += dR;
        if (rr >= 9u) {
          rr -= 9u;
          ++er;
        }
        const uint2 ent = __ldcg(&list[eu]);
        const uint32_t tri = ent.y;
        const GridK& g = grid_of_tri<MULTI>(gs, tri);
        int x, y, z;
        cell_coords(g, ent.x - g.cell_off, &x, &y, &z);
        const int X = x + (int)(row / 3u) - 1, Y = y + (int)(row % 3u) - 1;  // iproduct order, x outermost
        if ((unsigned)X >= (unsigned)g.n[0] || (unsigned)Y >= (unsigned)g.n[1]) continue;
        const TriRec r = tris[tri];
        const bool lo = z > 0, hi = z + 1 < g.n[2], mid = row != 4u;  // row 4's middle: the state's own cell
        const uint32_t j0 = g.cell_off + local_index(g, X, Y, z) - 1u;   // the cell at z - 1
        const unsigned long long k0 = lo ? __ldcg(&keys[j0]) : 0ull;
        const unsigned long long k1 = mid ? __ldcg(&keys[j0 + 1]) : 0ull;
        const unsigned long long k2 = hi ? __ldcg(&keys[j0 + 2]) : 0ull;
        // the row's cells share x and y, and so the x and y parts of the
        // closest-point dot products of a proper triangle
        const P3 a = p3(r.a), b = p3(r.b), c = p3(r.c);
        const int kind = __float_as_int(r.a.w);
        const bool proper = kind == TRI_PROPER;
        const P3 pm = center(g, X, Y, z);
        const RowXY rxy = row_xy(pm.x, pm.y, a, b, c);
        auto dist = [&](int dz) {
          const P3 pos{pm.x, pm.y, fa(g.f[2], fm(__int2float_rn(z + dz), g.s[2]))};  // center(g, X, Y, z + dz)
          return fsqrt(proper ? row_distance2(rxy, pos, a, b, c) : point_triangle_distance2_sel(pos, a, b, c, kind));
        };
        if (lo) {
          ++evals;
          if (propose_dist<SIGN>(dist(-1), tri, j0, k0, keys, nan))
            stage_touch(j0, s_touch, s_ntouch, st, parity, spill, cap);
        }
        if (mid) {
          ++evals;
          if (propose_dist<SIGN>(dist(0), tri, j0 + 1, k1, keys, nan))
            stage_touch(j0 + 1, s_touch, s_ntouch, st, parity, spill, cap);
        }
        if (hi) {
          ++evals;
          if (propose_dist<SIGN>(dist(1), tri, j0 + 2, k2, keys, nan))
            stage_touch(j0 + 2, s_touch, s_ntouch, st, parity, spill, cap);
        }
      }
      return;
    }
    if (SIGN == M2S_SIGN_RAYCAST) {
      while (e < n) {
        bool first[kUnroll];
        uint32_t jj[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; ++u) {
          first[u] = false;
          jj[u] = 0;
          const uint32_t eu = e, ku = k;
          step();
          uint32_t tri, j;
          int X, Y, Z;
          if (eu >= n || !neighbour(eu, ku, tri, j, X, Y, Z)) continue;
          ++evals;
          const P3 pos = center(grid_of_tri<MULTI>(gs, tri), X, Y, Z);
          first[u] = propose_at<SIGN>(tris[tri], tri, j, pos, __ldcg(&keys[j]), keys, nan);
          jj[u] = j;
        }
#pragma unroll
        for (int u = 0; u < kUnroll; ++u)
          if (first[u]) stage_touch(jj[u], s_touch, s_ntouch, st, parity, spill, cap);
      }
      return;
    }
    while (__any_sync(0xFFFFFFFFu, e < n)) {
      const uint32_t eu = e, ku = k;
      step();
      uint32_t tri = 0, j = 0;
      int X = 0, Y = 0, Z = 0;
      P3 pos{0.f, 0.f, 0.f};
      unsigned long long snap = 0;
      bool keep = false;
      if (eu < n && neighbour(eu, ku, tri, j, X, Y, Z)) {
        ++evals;
        snap = __ldcg(&keys[j]);
        pos = center(grid_of_tri<MULTI>(gs, tri), X, Y, Z);
        if (key_tri(snap) == tri) ++dropped_same;
        else keep = true;
      }
      queue_push(keep, tri, j, pos, snap);
    }
  }
  __syncwarp();
  if (lane < qn) run(lane);
  __syncwarp();
}

// Commit phase: clear each touched cell's dirty bit (its key holds the
// round's winner) and queue (cell, winner) under the winner's bucket.  A block
// commits the cells it staged; the spill list is shared out as
// spill_t0 + k * spill_T.
template <bool MULTI>
__device__ __forceinline__ void relax_commit(const GridSet& gs, unsigned long long* keys, const uint32_t* s_touch,
                                             uint32_t nloc, const uint32_t* spill, uint32_t nspill, uint32_t spill_t0,
                                             uint32_t spill_T, const Counters& ct, const Sched& sh, uint2* lists,
                                             uint32_t cap) {
  for (uint32_t base = 0; base < nloc; base += blockDim.x) {
    const uint32_t i = base + threadIdx.x;
    const bool act = i < nloc;
    uint32_t j = 0, nb = 0;
    unsigned long long w = KEY_EMPTY;
    if (act) {
      j = s_touch[i];
      w = __ldcg(&keys[j]) & ~kDirty;
      keys[j] = w;
      nb = bucket_of(grid_of_tri<MULTI>(gs, key_tri(w)).inv_delta, key_dist(w));
    }
    push_entry_warp(ct, sh.b, sh.B, sh.slot, sh.fp, lists, cap, act, j, key_tri(w), nb);
  }
  for (uint32_t base = spill_t0 - threadIdx.x; base < nspill; base += spill_T) {
    const uint32_t i = base + threadIdx.x;
    const bool act = i < nspill;
    uint32_t j = 0, nb = 0;
    unsigned long long w = KEY_EMPTY;
    if (act) {
      j = __ldcg(&spill[i]);
      w = __ldcg(&keys[j]) & ~kDirty;
      keys[j] = w;
      nb = bucket_of(grid_of_tri<MULTI>(gs, key_tri(w)).inv_delta, key_dist(w));
    }
    push_entry_warp(ct, sh.b, sh.B, sh.slot, sh.fp, lists, cap, act, j, key_tri(w), nb);
  }
}

// The kernel exists without and with the proposal filter (FILTER): without,
// 4 blocks of 256 threads fit per SM (64 registers a thread); the filtered
// propose loop needs about 80 registers, so that variant runs 3 per SM.
template <int SIGN, bool MULTI, bool FILTER>
__global__ void __launch_bounds__(256, FILTER ? 3 : 4) k_propagate(const __grid_constant__ GridSet gs, const TriRec* __restrict__ tris,
                                                   unsigned long long* keys,
                                                   uint2* lists, uint32_t cap, uint32_t* spill_lists,
                                                   PropState* st, GridBarrier* bar, uint32_t max_steps,
                                                   uint32_t* status, uint32_t* round_log, uint32_t log_cap,
                                                   uint32_t solo_max, const TriBound* __restrict__ bounds,
                                                   const float* __restrict__ slack) {
  __shared__ Sched sh;
  __shared__ __align__(16) uint32_t s_touch[kTouchStage];  // also a solo run's min table
  __shared__ uint16_t s_taken[26 * kSoloCap];              // a solo round's taken table slots
  constexpr bool kQueued = SIGN == M2S_SIGN_NORMAL || FILTER;  // the plain Raycast loop needs no queue
  __shared__ WarpQueue s_queue[kQueued ? kWarps : 1];
  __shared__ uint32_t s_ntouch, s_gen, s_pending, s_more, s_runs, s_solo_run;
  __shared__ uint32_t s_count[kLists], s_far_min[2], s_overflow;  // block 0's counters during a solo run
  // (built where used, so no pointer stays live across the propose loop)
  auto counters = [&](bool shared_ones) {
    return shared_ones ? Counters{s_count, s_far_min, &s_overflow} : global_counters(st);
  };
  const unsigned int nblocks = gridDim.x;
  const int lane = threadIdx.x & 31;
  const bool lead_block = blockIdx.x == 0;
  if (threadIdx.x == 0) {
    s_ntouch = 0;
    s_gen = 0;
    s_pending = 0;
    s_runs = 0;
    s_solo_run = 0;
    sh.b = st->b;
    sh.B = st->B;
    for (int k = 0; k < kRing; ++k) sh.slot[k] = st->slot[k];
    sh.cur = st->cur;
    sh.fp = st->fp;
    sh.round = 0;
    sh.steps = 0;
    sh.n = 0xFFFFFFFFu;  // no relax round yet: the first is never solo
  }
  bool nan = false;
  unsigned long long evals = 0;
  uint32_t dropped_same = 0, dropped_bound = 0;
  uint32_t far_phases = 0, logged = 0, max_list = 0, solo_rounds = 0;
  const uint64_t t_start = (lead_block && threadIdx.x == 0 && round_log) ? global_ns() : 0;
  bool aborted = false;
  // Warp 0: the next step (unless a solo run already chose it), logged by
  // block 0 when profiling: the relaxed list's size, or (top bit) the far list's.
  auto step = [&]() {
    const bool in_run = lead_block && s_solo_run;
    const uint32_t spill_ov = in_run ? 0u : *(volatile uint32_t*)&st->overflow2[sh.round & 1u];
    const bool limit = sh.steps >= max_steps;
    const int action = limit ? kLimit : next_step(sh, counters(in_run), spill_ov, lead_block);
    if (threadIdx.x != 0) {
      __syncwarp();
      return;
    }
    s_ntouch = 0;  // every thread read it in the last commit, before the last barrier
    sh.action = action;
    ++sh.steps;
    if (sh.action == kRelax) max_list = max(max_list, sh.n);
    // Profiling: block 0 records each step — the relaxed list's size (bit 30:
    // a solo round) or the far list's size (bit 31) — and when it was chosen.
    if (lead_block && round_log && logged < log_cap) {
      uint32_t v = 0;
      if (sh.action == kRelax) v = sh.n | (solo_round(sh, solo_max) ? 0x40000000u : 0u);
      else if (sh.action == kRedistribute) v = 0x80000000u | counters(in_run).count[kFar0 + sh.fp];
      else v = 0xC0000000u;  // the end
      round_log[2 * logged] = v;
      round_log[2 * logged + 1] = (uint32_t)(global_ns() - t_start);
      ++logged;
    }
    __syncwarp();
  };
  bool chosen = false;  // a solo round's tail chose this step already (block-uniform)
  for (;;) {
    if (!chosen) {
      if (threadIdx.x < 32) {
        const bool pending = s_pending;
        __syncwarp();
        if (!pending) step();
        else if (threadIdx.x == 0) s_pending = 0;
      }
      __syncthreads();
    }
    chosen = false;
    const int action = sh.action;
    if (action == kDone) break;
    if (action == kLimit) {
      if (lead_block && threadIdx.x == 0) atomicOr(status, bit(M2S_ERR_LIMIT));
      break;
    }
    if (action == kRedistribute) {
      // ---- move every far state to its bucket's list, or to the other far
      // list when it lies beyond the new window.  The bucket is recomputed
      // from the state's cell and triangle, the same arithmetic that produced
      // it, so it is exactly the bucket the state was filed under.  The
      // barrier first lets every block finish the step that chose this phase:
      // that step reads the list counts these pushes change.
      if (!grid_barrier(bar, nblocks, &s_gen)) {
        aborted = true;
        break;
      }
      const uint32_t F = kFar0 + sh.fp;
      const uint32_t nf = min(*(volatile uint32_t*)&st->count[F], cap);
      const uint2* far = lists + (unsigned long long)F * cap;
      for (uint32_t base = blockIdx.x * blockDim.x; base < nf; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + threadIdx.x;
        const bool act = i < nf;
        uint2 ent = make_uint2(0, 0);
        uint32_t nb = 0;
        if (act) {
          ent = __ldcg(&far[i]);
          const GridK& g = grid_of_tri<MULTI>(gs, ent.y);
          int x, y, z;
          cell_coords(g, ent.x - g.cell_off, &x, &y, &z);
          const TriRec r = tris[ent.y];
          const float d = cell_distance<SIGN>(center(g, x, y, z), p3(r.a), p3(r.b), p3(r.c), __float_as_int(r.a.w));
          nb = bucket_of(g.inv_delta, d);
        }
        push_entry_warp(global_counters(st), sh.b, sh.B, sh.slot, sh.fp ^ 1u, lists, cap, act, ent.x, ent.y, nb);
      }
      if (!grid_barrier(bar, nblocks, &s_gen)) {
        aborted = true;
        break;
      }
      if (threadIdx.x == 0) {
        if (lead_block) {  // the drained list is next written by the next redistribution
          st->count[F] = 0;
          st->far_min[sh.fp] = kNoBucket;
        }
        sh.fp ^= 1u;
        ++far_phases;
      }
      continue;
    }
    // ---- a relax round: by every block, or by block 0 alone when it is small
    const bool solo = solo_round(sh, solo_max);
    if (solo && !s_solo_run) {
      // A solo run starts.  Block 0 will change list counts at once (pushes,
      // and emptying the list it relaxes at its next step), so every block
      // first finishes reading this step's counts.
      if (!grid_barrier(bar, nblocks, &s_gen)) {
        aborted = true;
        break;
      }
      if (!lead_block) {  // wait for the run to end, then take block 0's schedule
        if (!grid_barrier(bar, nblocks, &s_gen)) {
          aborted = true;
          break;
        }
        if (threadIdx.x == 0) {
          const volatile uint32_t* src = (const volatile uint32_t*)&st->handoff;
          uint32_t* dst = (uint32_t*)&sh;
          for (uint32_t w = 0; w < sizeof(Sched) / 4; ++w) dst[w] = src[w];
          s_pending = 1;
        }
        continue;
      }
      if (threadIdx.x == 0) {
        // Block 0 alone pushes during the run: it keeps the counters in shared
        // memory and writes them back when it hands the schedule over.
        s_solo_run = 1;  // read again only after later block barriers
        for (int k = 0; k < kLists; ++k) s_count[k] = *(volatile uint32_t*)&st->count[k];
        s_far_min[0] = *(volatile uint32_t*)&st->far_min[0];
        s_far_min[1] = *(volatile uint32_t*)&st->far_min[1];
        s_overflow = *(volatile uint32_t*)&st->overflow | *(volatile uint32_t*)&st->overflow2[0] |
                     *(volatile uint32_t*)&st->overflow2[1];
      }
      for (uint32_t h = threadIdx.x; h < kHash; h += blockDim.x) {  // the run's min table, kept empty between rounds
        s_touch[h] = kNoCell;
        reinterpret_cast<unsigned long long*>(s_touch + kHash)[h] = KEY_EMPTY;
      }
      __syncthreads();
    }
    const uint32_t parity = sh.round & 1u;
    uint32_t* spill = spill_lists + (unsigned long long)parity * cap;
    const uint32_t n = min(sh.n, cap);
    const uint32_t T = solo ? blockDim.x : gridDim.x * blockDim.x;
    const uint32_t t0 = solo ? threadIdx.x : blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t* HJ = s_touch;
    unsigned long long* HK = reinterpret_cast<unsigned long long*>(s_touch + kHash);
    if (solo)
      relax_propose_solo<SIGN, MULTI>(gs, tris, keys, lists + (unsigned long long)sh.cur * cap, n, HJ, HK,
                                      s_taken, &s_ntouch, nan, evals, dropped_same);
    else
      relax_propose<SIGN, MULTI, FILTER>(gs, tris, bounds, slack, keys,
                                 lists + (unsigned long long)sh.cur * cap, n, T, t0, s_touch, &s_ntouch, st, parity,
                                 spill, cap, nan, evals, dropped_same, dropped_bound,
                                         &s_queue[kQueued ? threadIdx.x >> 5 : 0]);
    if (lead_block && threadIdx.x == 0) atomicAdd(&st->entries, (unsigned long long)n);
    if (solo) {
      __syncthreads();
    } else if (!grid_barrier(bar, nblocks, &s_gen)) {
      aborted = true;
      break;
    }
    if (solo) {
      relax_commit_solo<MULTI>(gs, keys, HJ, HK, s_taken, min(s_ntouch, 26u * kSoloCap),
                               counters(true), sh, lists, cap);
    } else {
      if (lead_block && threadIdx.x == 0) st->touched2[parity ^ 1u] = 0;
      const uint32_t nspill = min(*(volatile uint32_t*)&st->touched2[parity], cap);
      relax_commit<MULTI>(gs, keys, s_touch, min(s_ntouch, (uint32_t)kTouchStage), spill, nspill, t0,
                          T, global_counters(st), sh, lists, cap);
    }
    if (!solo) {
      if (!grid_barrier(bar, nblocks, &s_gen)) {
        aborted = true;
        break;
      }
      continue;
    }
    // Solo: block 0 chooses the next step at once; it goes on alone while the
    // rounds stay small, else hands the schedule (next action included) to the
    // other blocks at the barrier they wait at.
    __syncthreads();
    if (threadIdx.x < 32) step();
    if (threadIdx.x == 0) {
      ++s_runs;
      ++solo_rounds;
      s_more = sh.action == kRelax && solo_round(sh, solo_max) && s_runs < kSoloRounds;
      if (!s_more) {
        for (int k = 0; k < kLists; ++k) st->count[k] = s_count[k];
        st->far_min[0] = s_far_min[0];
        st->far_min[1] = s_far_min[1];
        if (s_overflow) st->overflow = 1u;
        volatile uint32_t* dst = (volatile uint32_t*)&st->handoff;
        const uint32_t* src = (const uint32_t*)&sh;
        for (uint32_t w = 0; w < sizeof(Sched) / 4; ++w) dst[w] = src[w];
        s_runs = 0;
        s_solo_run = 0;
        s_pending = 1;
      }
    }
    __syncthreads();
    if (s_more) {
      chosen = true;
      continue;
    }
    if (!grid_barrier(bar, nblocks, &s_gen)) {
      aborted = true;
      break;
    }
  }
  if (nan) atomicOr(status, bit(M2S_ERR_NAN_DISTANCE));
  for (int o = 16; o; o >>= 1) evals += __shfl_xor_sync(0xFFFFFFFFu, evals, o);
  if (lane == 0 && evals) atomicAdd(&st->evals, evals);
  unsigned long long ds = dropped_same, db = dropped_bound;
  for (int o = 16; o; o >>= 1) {
    ds += __shfl_xor_sync(0xFFFFFFFFu, ds, o);
    db += __shfl_xor_sync(0xFFFFFFFFu, db, o);
  }
  if (lane == 0 && ds) atomicAdd(&st->filter_same, ds);
  if (lane == 0 && db) atomicAdd(&st->filter_bound, db);
  if (aborted && lead_block && threadIdx.x == 0) atomicOr(status, bit(M2S_ERR_LIMIT));
  if (lead_block && threadIdx.x == 0) {
    st->round = sh.round;
    st->far_phases = far_phases;
    st->log_n = logged;
    st->max_list = max_list;
    st->solo_rounds = solo_rounds;
    st->done = 1;
  }
}

// ---- 3. rays -------------------------------------------------------------------
__device__ __forceinline__ unsigned long long column_of(const GridK& g, int axis, int x, int y, int z) {
  if (axis == 0) return (unsigned long long)y * g.n[2] + z;
  if (axis == 1) return (unsigned long long)x * g.n[2] + z;
  return (unsigned long long)x * g.n[1] + y;
}

// Range of lattice indices along `d` whose ray origin can lie in [lo, hi];
// one extra index on each side keeps it conservative.
__device__ __forceinline__ void lattice_range(const GridK& g, int d, float lo, float hi, int* a, int* b) {
  float u1 = (lo - g.f[d]) / g.s[d], u2 = (hi - g.f[d]) / g.s[d];
  float umin = fminf(u1, u2), umax = fmaxf(u1, u2);
  if (!(isfinite(umin) && isfinite(umax))) {
    *a = 0;
    *b = g.n[d] - 1;
    return;
  }
  float fa_ = floorf(umin) - 1.0f, fb_ = ceilf(umax) + 1.0f;
  *a = fa_ <= 0.0f ? 0 : (fa_ >= (float)(g.n[d] - 1) ? g.n[d] - 1 : (int)fa_);
  *b = fb_ <= 0.0f ? 0 : (fb_ >= (float)(g.n[d] - 1) ? g.n[d] - 1 : (int)fb_);
  if (fb_ < 0.0f || fa_ > (float)(g.n[d] - 1)) *b = *a - 1;  // no lattice point in range
}

// With AUDIT, each ray test is also audited (m2s_audit.cuh): the f32
// decision toggles `bits` exactly as without, the FP64 one toggles `bits64`.
template <int AXIS, bool MULTI, bool AUDIT = false>
__global__ void k_rays(const __grid_constant__ GridSet gs, const TriRec* __restrict__ tris, uint32_t T, uint32_t* bits,
                       PropState* st, uint32_t* bits64 = nullptr) {
  constexpr int IY = (AXIS + 1) % 3, IZ = (AXIS + 2) % 3;
  const uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (t >= T) return;
  const GridK& g = grid_of_tri<MULTI>(gs, t);
  TriRec r = tris[t];
  P3 a = p3(r.a), b = p3(r.b), c = p3(r.c);
  P3 lo, hi;
  padded_box(a, b, c, &lo, &hi);
  int j0, j1, k0, k1;
  lattice_range(g, IY, vget(lo, IY), vget(hi, IY), &j0, &j1);
  lattice_range(g, IZ, vget(lo, IZ), vget(hi, IZ), &k0, &k1);
  if (j1 < j0 || k1 < k0) return;
  const int nj = j1 - j0 + 1, nk = k1 - k0 + 1;
  const long long total = (long long)nj * nk;
  uint32_t* bitsA = bits + g.bits_off[AXIS];
  const uint32_t W = g.words[AXIS];
  uint32_t hits = 0, tests = 0, ambiguous = 0, disagree = 0;
  const bool small = total <= 0x7FFFFFFFll;  // 32-bit division (64-bit costs ~4x the instructions)
  for (long long q = lane; q < total; q += 32) {
    int c3[3];
    c3[AXIS] = 0;
    if (small) {
      const uint32_t uq = (uint32_t)q, row = uq / (uint32_t)nk;
      c3[IY] = j0 + (int)row;
      c3[IZ] = k0 + (int)(uq - row * (uint32_t)nk);
    } else {
      c3[IY] = j0 + (int)(q / nk);
      c3[IZ] = k0 + (int)(q % nk);
    }
    P3 o = center(g, c3[0], c3[1], c3[2]);  // ray origin: a low-face cell centre (grid.rs:580)
    float tt;
    const unsigned long long last = (unsigned long long)g.n[AXIS] - 1;
    const unsigned long long col = column_of(g, AXIS, c3[0], c3[1], c3[2]);
    if constexpr (AUDIT) {
      const RayAudit ra = ray_audit<AXIS>(o, a, b, c);
      ++tests;
      ambiguous += ra.ambiguous;
      disagree += ra.hit64 != ra.hit32;
      if (ra.hit64) {  // the FP64 decision's crossing, in the FP64 parity bits
        unsigned long long kk;
        if (ra.hit32) {
          kk = sat_u64(floorf(fd(ra.t32, g.s[AXIS])));
        } else {
          const double u = floor(ra.t64 / (double)g.s[AXIS]);
          kk = u <= 0.0 ? 0ull : (u >= 1.8e19 ? ULLONG_MAX : (unsigned long long)u);
        }
        const uint32_t k = (uint32_t)(kk < last ? kk : last);
        atomicXor(&bits64[g.bits_off[AXIS] + col * W + (k >> 5)], 1u << (k & 31));
      }
      if (!ra.hit32) continue;
      tt = ra.t32;
    } else {
      if (!ray_hit_aligned<AXIS>(o, a, b, c, &tt)) continue;
    }
    ++hits;
    // grid.rs:604-607
    unsigned long long kk = sat_u64(floorf(fd(tt, g.s[AXIS])));
    uint32_t k = (uint32_t)(kk < last ? kk : last);
    atomicXor(&bitsA[col * W + (k >> 5)], 1u << (k & 31));
  }
  for (int o = 16; o; o >>= 1) hits += __shfl_xor_sync(0xFFFFFFFFu, hits, o);
  if (lane == 0 && hits) atomicAdd(&st->ray_hits, (unsigned long long)hits);
  if constexpr (AUDIT) {
    for (int o = 16; o; o >>= 1) {
      tests += __shfl_xor_sync(0xFFFFFFFFu, tests, o);
      ambiguous += __shfl_xor_sync(0xFFFFFFFFu, ambiguous, o);
      disagree += __shfl_xor_sync(0xFFFFFFFFu, disagree, o);
    }
    if (lane == 0) {
      atomicAdd(&st->audit[0], (unsigned long long)tests);
      atomicAdd(&st->audit[1], (unsigned long long)ambiguous);
      atomicAdd(&st->audit[2], (unsigned long long)disagree);
    }
  }
}

// FP64 audit of every cell (reports only): the Voronoi region of its final
// (cell, triangle) pair, and, for Raycast, whether the 2-of-3 vote of the
// FP64-decided parities differs from the f32 one.
template <int SIGN, bool MULTI>
__global__ void k_audit_cells(const __grid_constant__ GridSet gs, const TriRec* __restrict__ tris,
                              const unsigned long long* __restrict__ keys, const uint32_t* __restrict__ bits,
                              const uint32_t* __restrict__ bits64, PropState* st) {
  SegCursor<uint32_t> sc;
  uint32_t flips = 0, audited = 0, ambiguous = 0, disagree = 0;
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < gs.ncell;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    const GridK& g = MULTI ? gs.table[sc.at(gs.cell_off, gs.ngrids, (uint32_t)i)] : gs.g0;
    int x, y, z;
    cell_coords(g, (uint32_t)i - g.cell_off, &x, &y, &z);
    if (SIGN == M2S_SIGN_RAYCAST) {
      uint32_t v32 = 0, v64 = 0;
      const uint32_t c3[3] = {(uint32_t)x, (uint32_t)y, (uint32_t)z};
      for (int a = 0; a < 3; ++a) {
        const unsigned long long w = g.bits_off[a] + column_of(g, a, x, y, z) * g.words[a] + (c3[a] >> 5);
        v32 += (bits[w] >> (c3[a] & 31)) & 1u;
        v64 += (bits64[w] >> (c3[a] & 31)) & 1u;
      }
      flips += (v32 >= 2) != (v64 >= 2);
    }
    const uint32_t t = key_tri(keys[i]);
    if (t == NO_TRI) continue;
    const TriRec r = tris[t];
    if (__float_as_int(r.a.w) != TRI_PROPER) continue;
    const RegionAudit ra = region_audit(center(g, x, y, z), p3(r.a), p3(r.b), p3(r.c));
    ++audited;
    ambiguous += ra.ambiguous;
    disagree += ra.region64 != ra.region32;
  }
  const int lane = threadIdx.x & 31;
  for (int o = 16; o; o >>= 1) {
    flips += __shfl_xor_sync(0xFFFFFFFFu, flips, o);
    audited += __shfl_xor_sync(0xFFFFFFFFu, audited, o);
    ambiguous += __shfl_xor_sync(0xFFFFFFFFu, ambiguous, o);
    disagree += __shfl_xor_sync(0xFFFFFFFFu, disagree, o);
  }
  if (lane == 0) {
    atomicAdd(&st->audit[3], (unsigned long long)flips);
    atomicAdd(&st->audit[4], (unsigned long long)audited);
    atomicAdd(&st->audit[5], (unsigned long long)ambiguous);
    atomicAdd(&st->audit[6], (unsigned long long)disagree);
  }
}

// Toggle bits -> suffix parity: bit i becomes the XOR of toggles i..n-1, i.e.
// the parity of the hits whose cell range 0..=k covers cell i.
template <bool MULTI>
__global__ void k_suffix(const __grid_constant__ GridSet gs, int axis, uint32_t* bits) {
  SegCursor<unsigned long long> sc;
  const unsigned long long ncols = gs.ncols[axis];
  for (unsigned long long col = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; col < ncols;
       col += (unsigned long long)gridDim.x * blockDim.x) {
    const GridK& g = MULTI ? gs.table[sc.at(gs.col_off[axis], gs.ngrids, col)] : gs.g0;
    const uint32_t W = g.words[axis];
    uint32_t* w = bits + g.bits_off[axis] + (col - g.col_off[axis]) * W;
    uint32_t carry = 0;
    for (int i = (int)W - 1; i >= 0; --i) {
      uint32_t s = w[i];
      s ^= s >> 1;
      s ^= s >> 2;
      s ^= s >> 4;
      s ^= s >> 8;
      s ^= s >> 16;
      if (carry) s = ~s;
      carry = s & 1u;
      w[i] = s;
    }
  }
}

template <int SIGN, bool MULTI>
__global__ void k_finalize(const __grid_constant__ GridSet gs, const unsigned long long* __restrict__ keys,
                           const uint32_t* __restrict__ bits, float* __restrict__ out) {
  SegCursor<uint32_t> sc;
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < gs.ncell;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    float d = key_dist(keys[i]);
    if (SIGN == M2S_SIGN_RAYCAST) {
      const GridK& g = MULTI ? gs.table[sc.at(gs.cell_off, gs.ngrids, (uint32_t)i)] : gs.g0;
      int x, y, z;
      cell_coords(g, (uint32_t)i - g.cell_off, &x, &y, &z);
      uint32_t px = (bits[g.bits_off[0] + column_of(g, 0, x, y, z) * g.words[0] + (x >> 5)] >> (x & 31)) & 1u;
      uint32_t py = (bits[g.bits_off[1] + column_of(g, 1, x, y, z) * g.words[1] + (y >> 5)] >> (y & 31)) & 1u;
      uint32_t pz = (bits[g.bits_off[2] + column_of(g, 2, x, y, z) * g.words[2] + (z >> 5)] >> (z & 31)) & 1u;
      if (px + py + pz >= 2) d = -d;
      out[g.out_off + ((uint32_t)i - g.cell_off)] = d;
    } else {
      const GridK& g = MULTI ? gs.table[sc.at(gs.cell_off, gs.ngrids, (uint32_t)i)] : gs.g0;
      out[g.out_off + ((uint32_t)i - g.cell_off)] = d;
    }
  }
}

unsigned blocks_for(unsigned long long n, int threads, unsigned cap = 148u * 16u) {
  unsigned long long b = (n + threads - 1) / threads;
  return (unsigned)std::max<unsigned long long>(1, std::min<unsigned long long>(b, cap));
}

// Pinned host copy of the propagation state, one per host thread.
struct HostState {
  PropState* p = nullptr;
  ~HostState() {
    if (p) cudaFreeHost(p);
  }
};
PropState* host_state() {
  thread_local HostState h;
  if (!h.p && cudaHostAlloc((void**)&h.p, sizeof(PropState), cudaHostAllocPortable) != cudaSuccess) {
    cudaGetLastError();
    h.p = nullptr;
  }
  return h.p;
}

template <int SIGN>
const void* propagate_kernel(bool multi, bool filter) {
  if (filter) return multi ? (const void*)k_propagate<SIGN, true, true> : (const void*)k_propagate<SIGN, false, true>;
  return multi ? (const void*)k_propagate<SIGN, true, false> : (const void*)k_propagate<SIGN, false, false>;
}

}  // namespace

struct GridJob::Impl {
  std::vector<GridK> grids;
  GridSet gs{};
  bool multi = false;
  int sign = 0;
  uint32_t T = 0;
  const TriRec* tris = nullptr;
  float* d_out = nullptr;
  uint32_t* d_status = nullptr;
  uint32_t cap = 0;
  unsigned coop_blocks = 0;
  unsigned coop_max = 0;
  uint32_t solo_max = 64;
  unsigned long long ray_words = 0;
  uint64_t launches = 0;
  DevBuf<TriRec> comb_tris;
  DevBuf<const TriRec*> src_tris;
  DevBuf<uint32_t> tri_grid, tri_off, cell_off;
  DevBuf<unsigned long long> col_off[3];
  DevBuf<GridK> table;
  DevBuf<unsigned long long> keys;  // one per cell
  DevBuf<PropState> state;
  DevBuf<GridBarrier> bar;
  DevBuf<uint32_t> bits;
  DevBuf<uint2> lists;
  DevBuf<uint32_t> touched;
  DevBuf<uint32_t> round_log;  // profiling only
  DevBuf<TriBound> bounds;     // the proposal filter's per-triangle records
  DevBuf<float> slack;
  bool filter = false;
  bool audit = false;          // FP64 audit (reports only)
  DevBuf<uint32_t> bits64;     // the audit's FP64-decided ray parities
};

GridJob::GridJob() : p(new Impl) {}
GridJob::~GridJob() { delete p; }
uint32_t GridJob::capacity() const { return p->cap; }
int GridJob::enable_round_log(uint32_t cap, cudaStream_t s) { return p->round_log.alloc(2ull * cap, s); }
int GridJob::read_round_log(std::vector<uint32_t>* out, uint32_t n, cudaStream_t s) {
  n = std::min<uint32_t>(n, (uint32_t)(p->round_log.n / 2));
  out->resize(2ull * n);
  if (n) M2S_CUDA(cudaMemcpyAsync(out->data(), p->round_log.p, 8ull * n, cudaMemcpyDeviceToHost, s));
  M2S_CUDA(cudaStreamSynchronize(s));
  return M2S_OK;
}
void GridJob::set_capacity(uint32_t cap) { p->cap = cap; }
uint64_t GridJob::cells() const { return p->gs.ncell; }
unsigned GridJob::cooperative_blocks() const { return p->coop_blocks; }
unsigned GridJob::max_cooperative_blocks() const { return p->coop_max; }
void GridJob::set_cooperative_blocks(unsigned blocks) { p->coop_blocks = std::max(1u, std::min(blocks, p->coop_max)); }
int GridJob::sign() const { return p->sign; }
uint32_t GridJob::grids() const { return p->gs.ngrids; }
uint64_t GridJob::device_bytes() const {
  const Impl& J = *p;
  return J.comb_tris.n * sizeof(TriRec) + J.tri_grid.n * 4 + J.keys.n * 8 + J.bits.n * 4 +
         J.bounds.n * sizeof(TriBound) + J.slack.n * 4 +
         (uint64_t)kLists * J.cap * 8 + 2ull * J.cap * 4 + J.table.n * sizeof(GridK);
}

int propagate_blocks_per_sm(int sign) {
  const bool filter = grid_tuning().bound_filter;
  const void* kern = sign == M2S_SIGN_RAYCAST ? propagate_kernel<M2S_SIGN_RAYCAST>(true, filter)
                                              : propagate_kernel<M2S_SIGN_NORMAL>(true, filter);
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0) != cudaSuccess) return 1;
  return std::max(per_sm, 1);
}

uint32_t default_list_capacity(uint64_t cells) {
  return (uint32_t)std::min<uint64_t>(std::max<uint64_t>(cells / 2, std::min<uint64_t>(cells + 1024, 1ull << 20)),
                                      0x40000000ull);
}

uint64_t grid_job_bytes(uint64_t cells) {
  const uint64_t cap = default_list_capacity(cells);
  const uint64_t ray_words = 3 * (cells / 32 + 3 * std::cbrt((double)cells) * std::cbrt((double)cells));
  return 8 * cells + (uint64_t)kLists * 8 * cap + 8 * cap + 4 * ray_words + (1u << 20);  // + 68 B per triangle
}

int check_grid(const GridDesc& g) {
  for (int d = 0; d < 3; ++d)
    if (g.n[d] == 0 || g.n[d] > 0x7FFFFFFFull) return M2S_ERR_INVALID_ARGUMENT;
  if (g.cells() >= 0xFFFFFFFFull) return M2S_ERR_INVALID_ARGUMENT;  // cells are addressed with 32-bit indices
  return M2S_OK;
}

int GridJob::prepare(const MeshView* meshes, uint32_t n, const GridDesc* gds, int sign, float* d_out,
                     uint32_t* d_status, cudaStream_t s, const GridTuning& tune, const uint64_t* out_offsets) {
  Impl& J = *p;
  if (n == 0) return M2S_ERR_INVALID_ARGUMENT;
  J.sign = sign;
  J.d_out = d_out;
  J.d_status = d_status;
  J.multi = n > 1;
  J.grids.assign(n, GridK{});
  unsigned long long cells = 0, tris = 0, cols[3] = {0, 0, 0}, words[3] = {0, 0, 0};
  std::vector<uint32_t> h_cell_off(n + 1), h_tri_off(n + 1);
  std::vector<unsigned long long> h_col_off[3];
  std::vector<const TriRec*> h_src(n);
  for (int a = 0; a < 3; ++a) h_col_off[a].assign(n + 1, 0);
  int st;
  for (uint32_t k = 0; k < n; ++k) {
    const GridDesc& gd = gds[k];
    if ((st = check_grid(gd))) return st;
    GridK& g = J.grids[k];
    for (int d = 0; d < 3; ++d) {
      g.f[d] = gd.first[d];
      g.s[d] = gd.size[d];
      g.n[d] = (int)gd.n[d];
    }
    const unsigned long long nk = gd.cells();
    if (cells + nk >= 0xFFFFFFFFull) return M2S_ERR_INVALID_ARGUMENT;  // 32-bit cell indices across the job
    g.ncell = (uint32_t)nk;
    g.cell_off = (uint32_t)cells;
    g.out_off = out_offsets ? out_offsets[k] : cells;
    h_cell_off[k] = (uint32_t)cells;
    cells += nk;
    g.div_z = make_fastdiv((uint32_t)g.n[2]);
    g.div_y = make_fastdiv((uint32_t)g.n[1]);
    const float minsize = std::min(std::fabs(g.s[0]), std::min(std::fabs(g.s[1]), std::fabs(g.s[2])));
    const float delta = 0.25f * minsize;
    g.inv_delta = (delta > 0.0f && std::isfinite(delta)) ? 1.0f / delta : 1.0f;
    for (int a = 0; a < 3; ++a) {
      const unsigned long long nc = nk / gd.n[a];
      g.words[a] = (uint32_t)((gd.n[a] + 31) / 32);
      g.col_off[a] = cols[a];
      h_col_off[a][k] = cols[a];
      g.bits_off[a] = words[a];
      cols[a] += nc;
      words[a] += nc * g.words[a];
    }
    h_tri_off[k] = (uint32_t)tris;
    h_src[k] = meshes[k].tris;
    tris += meshes[k].n_tris;
    if (tris > 0x7FFFFFFFull) return M2S_ERR_INVALID_ARGUMENT;
  }
  h_cell_off[n] = (uint32_t)cells;
  h_tri_off[n] = (uint32_t)tris;
  // The three axes share one bit array, axis after axis.
  unsigned long long woff = 0;
  for (int a = 0; a < 3; ++a) {
    h_col_off[a][n] = cols[a];
    for (auto& g : J.grids) g.bits_off[a] += woff;
    woff += words[a];
    J.gs.ncols[a] = cols[a];
  }
  J.ray_words = woff;
  J.T = (uint32_t)tris;
  J.gs.g0 = J.grids[0];
  J.gs.ngrids = n;
  J.gs.ncell = (uint32_t)cells;
  if (J.multi) {
    if ((st = J.table.alloc(n, s)) || (st = J.cell_off.alloc(n + 1, s)) || (st = J.tri_off.alloc(n + 1, s)) ||
        (st = J.src_tris.alloc(n, s)) || (st = J.comb_tris.alloc(tris, s)) || (st = J.tri_grid.alloc(tris, s)))
      return st;
    for (int a = 0; a < 3; ++a)
      if ((st = J.col_off[a].alloc(n + 1, s))) return st;
    // Pageable sources: each copy has read its source when the call returns.
    M2S_CUDA(cudaMemcpyAsync(J.table.p, J.grids.data(), n * sizeof(GridK), cudaMemcpyHostToDevice, s));
    M2S_CUDA(cudaMemcpyAsync(J.cell_off.p, h_cell_off.data(), (n + 1) * 4ull, cudaMemcpyHostToDevice, s));
    M2S_CUDA(cudaMemcpyAsync(J.tri_off.p, h_tri_off.data(), (n + 1) * 4ull, cudaMemcpyHostToDevice, s));
    M2S_CUDA(cudaMemcpyAsync(J.src_tris.p, h_src.data(), n * sizeof(TriRec*), cudaMemcpyHostToDevice, s));
    for (int a = 0; a < 3; ++a)
      M2S_CUDA(cudaMemcpyAsync(J.col_off[a].p, h_col_off[a].data(), (n + 1) * 8ull, cudaMemcpyHostToDevice, s));
    if (tris) {
      k_gather_tris<<<blocks_for(tris, 256), 256, 0, s>>>(J.src_tris.p, J.tri_off.p, n, (uint32_t)tris, J.comb_tris.p,
                                                          J.tri_grid.p);
      M2S_CUDA(cudaGetLastError());
    }
    J.tris = J.comb_tris.p;
    J.gs.table = J.table.p;
    J.gs.tri_grid = J.tri_grid.p;
    J.gs.cell_off = J.cell_off.p;
    for (int a = 0; a < 3; ++a) J.gs.col_off[a] = J.col_off[a].p;
  } else {
    J.tris = meshes[0].tris;
  }
  const unsigned long long N = cells;
  if ((st = J.keys.alloc(N, s)) || (st = J.state.alloc(1, s)) ||
      (st = J.bar.alloc(1, s)))
    return st;
  J.filter = tune.bound_filter;
  J.audit = tune.fp64_audit;
  if (tris && ((st = J.bounds.alloc(tris, s)) || (st = J.slack.alloc(tris, s)))) return st;
  if (sign == M2S_SIGN_RAYCAST && (st = J.bits.alloc(woff, s))) return st;
  if (sign == M2S_SIGN_RAYCAST && J.audit && (st = J.bits64.alloc(woff, s))) return st;
  J.cap = tune.list_capacity ? tune.list_capacity : default_list_capacity(N);
  J.solo_max = std::min<uint32_t>(tune.solo_max, kSoloCap);  // a solo round never spills
  // Cooperative grid: co-resident blocks, fewer for small jobs (a barrier
  // over fewer blocks is faster and a small bucket does not fill many).
  const void* kern = sign == M2S_SIGN_RAYCAST ? propagate_kernel<M2S_SIGN_RAYCAST>(J.multi, J.filter)
                                              : propagate_kernel<M2S_SIGN_NORMAL>(J.multi, J.filter);
  int dev = 0, sms = 0, per_sm = 0;
  M2S_CUDA(cudaGetDevice(&dev));
  M2S_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  M2S_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0));
  if (per_sm < 1) {
    set_error("grid propagation kernel cannot be resident");
    return M2S_ERR_CUDA;
  }
  J.coop_max = (unsigned)std::min<unsigned long long>((unsigned long long)sms * per_sm,
                                                     (unsigned long long)kMaxBarrierBlocks);
  if (tune.blocks_per_sm > 0) per_sm = std::min(per_sm, tune.blocks_per_sm);
  const unsigned long long cpb = std::max<uint32_t>(tune.cells_per_block, 1);
  // At least one block per SM: a round's proposals are chains of dependent
  // L2 trips, so a small grid's rounds finish sooner spread over every SM
  // (measured on 32^3 and 64^3 grids; from 128^3 on the occupancy limit is reached).
  const unsigned long long want = std::max<unsigned long long>((unsigned long long)sms, (N + cpb - 1) / cpb);
  J.coop_blocks = (unsigned)std::min<unsigned long long>(
      want, std::min<unsigned long long>((unsigned long long)sms * per_sm, J.coop_max));
  return M2S_OK;
}

int GridJob::alloc_lists(cudaStream_t s) {
  Impl& J = *p;
  int st;
  if ((st = J.lists.alloc((unsigned long long)kLists * J.cap, s)) || (st = J.touched.alloc(2ull * J.cap, s))) return st;
  return M2S_OK;
}

int GridJob::enqueue(cudaStream_t s, cudaEvent_t* ev) {
  Impl& J = *p;
  const unsigned long long N = J.gs.ncell;
  const bool raycast = J.sign == M2S_SIGN_RAYCAST;
  const bool multi = J.multi;
  J.launches = 0;
  auto mark = [&](int i) -> int {
    if (ev) M2S_CUDA(cudaEventRecord(ev[i], s));
    return M2S_OK;
  };
  int st;
  if ((st = mark(0))) return st;
  M2S_CUDA(cudaMemsetAsync(J.state.p, 0, sizeof(PropState), s));
  k_state_init<<<1, 1, 0, s>>>(J.state.p);
  k_fill_u64<<<blocks_for(N, 256), 256, 0, s>>>(J.keys.p, N, KEY_EMPTY);
  J.launches += 2;
  if (J.T > 0) {
    const unsigned sb = (unsigned)((J.T * 32ull + 255) / 256);
    if (raycast) {
      if (multi) k_seed<M2S_SIGN_RAYCAST, true><<<sb, 256, 0, s>>>(J.gs, J.tris, J.T, J.keys.p, J.d_status, J.state.p);
      else k_seed<M2S_SIGN_RAYCAST, false><<<sb, 256, 0, s>>>(J.gs, J.tris, J.T, J.keys.p, J.d_status, J.state.p);
    } else {
      if (multi) k_seed<M2S_SIGN_NORMAL, true><<<sb, 256, 0, s>>>(J.gs, J.tris, J.T, J.keys.p, J.d_status, J.state.p);
      else k_seed<M2S_SIGN_NORMAL, false><<<sb, 256, 0, s>>>(J.gs, J.tris, J.T, J.keys.p, J.d_status, J.state.p);
    }
    ++J.launches;
  }
  M2S_CUDA(cudaGetLastError());
  if ((st = mark(1))) return st;
  if (J.T > 0) {
    M2S_CUDA(cudaMemsetAsync(J.bar.p, 0, sizeof(GridBarrier), s));
    if (J.filter) {
      k_bounds<<<blocks_for(J.T, 256), 256, 0, s>>>(J.tris, J.T, J.bounds.p, J.slack.p);
      ++J.launches;
    }
    if (multi) k_collect<true><<<blocks_for(N, 256), 256, 0, s>>>(J.gs, J.keys.p, J.state.p, J.lists.p, J.cap);
    else k_collect<false><<<blocks_for(N, 256), 256, 0, s>>>(J.gs, J.keys.p, J.state.p, J.lists.p, J.cap);
    M2S_CUDA(cudaGetLastError());
    const void* kern = raycast ? propagate_kernel<M2S_SIGN_RAYCAST>(multi, J.filter)
                               : propagate_kernel<M2S_SIGN_NORMAL>(multi, J.filter);
    uint32_t max_steps = kMaxSteps;
    const TriRec* tris = J.tris;
    uint32_t* log = J.round_log.p;
    uint32_t log_cap = (uint32_t)(J.round_log.n / 2);
    void* args[] = {&J.gs,     &tris,   &J.keys.p,  &J.lists.p, &J.cap,     &J.touched.p,
                    &J.state.p, &J.bar.p, &max_steps, &J.d_status, &log,       &log_cap, &J.solo_max,
                    &J.bounds.p, &J.slack.p};
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(J.coop_blocks);
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    M2S_CUDA(cudaLaunchKernelExC(&cfg, kern, args));
    J.launches += 2;
  }
  if ((st = mark(2))) return st;
  const unsigned fb = blocks_for(N, 256, 148u * 32u);
  if (raycast) {
    M2S_CUDA(cudaMemsetAsync(J.bits.p, 0, J.ray_words * 4, s));
    if (J.audit) M2S_CUDA(cudaMemsetAsync(J.bits64.p, 0, J.ray_words * 4, s));
    if (J.T > 0) {
      const unsigned rb = (unsigned)((J.T * 32ull + 255) / 256);
      uint32_t* b64 = J.bits64.p;
      if (J.audit) {
        if (multi) {
          k_rays<0, true, true><<<rb, 256, 0, s>>>(J.gs, J.tris, J.T, J.bits.p, J.state.p, b64);
          k_rays<1, true, true><<<rb, 256, 0, s>>>(J.gs, J.tris, J.T, J.bits.p, J.state.p, b64);
          k_rays<2, true, true><<<rb, 256, 0, s>>>(J.gs, J.tris, J.T, J.bits.p, J.state.p, b64);
        } else {
          k_rays<0, false, true><<<rb, 256, 0, s>>>(J.gs, J.tris, J.T, J.bits.p, J.state.p, b64);
          k_rays<1, false, true><<<rb, 256, 0, s>>>(J.gs, J.tris, J.T, J.bits.p, J.state.p, b64);
          k_rays<2, false, true><<<rb, 256, 0, s>>>(J.gs, J.tris, J.T, J.bits.p, J.state.p, b64);
        }
      } else if (multi) {
        k_rays<0, true><<<rb, 256, 0, s>>>(J.gs, J.tris, J.T, J.bits.p, J.state.p);
        k_rays<1, true><<<rb, 256, 0, s>>>(J.gs, J.tris, J.T, J.bits.p, J.state.p);
        k_rays<2, true><<<rb, 256, 0, s>>>(J.gs, J.tris, J.T, J.bits.p, J.state.p);
      } else {
        k_rays<0, false><<<rb, 256, 0, s>>>(J.gs, J.tris, J.T, J.bits.p, J.state.p);
        k_rays<1, false><<<rb, 256, 0, s>>>(J.gs, J.tris, J.T, J.bits.p, J.state.p);
        k_rays<2, false><<<rb, 256, 0, s>>>(J.gs, J.tris, J.T, J.bits.p, J.state.p);
      }
      J.launches += 3;
    }
    for (int a = 0; a < 3; ++a) {
      if (multi) k_suffix<true><<<blocks_for(J.gs.ncols[a], 256), 256, 0, s>>>(J.gs, a, J.bits.p);
      else k_suffix<false><<<blocks_for(J.gs.ncols[a], 256), 256, 0, s>>>(J.gs, a, J.bits.p);
      if (J.audit) {
        if (multi) k_suffix<true><<<blocks_for(J.gs.ncols[a], 256), 256, 0, s>>>(J.gs, a, J.bits64.p);
        else k_suffix<false><<<blocks_for(J.gs.ncols[a], 256), 256, 0, s>>>(J.gs, a, J.bits64.p);
      }
    }
    J.launches += J.audit ? 6 : 3;
    M2S_CUDA(cudaGetLastError());
    if ((st = mark(3))) return st;
    if (multi) k_finalize<M2S_SIGN_RAYCAST, true><<<fb, 256, 0, s>>>(J.gs, J.keys.p, J.bits.p, J.d_out);
    else k_finalize<M2S_SIGN_RAYCAST, false><<<fb, 256, 0, s>>>(J.gs, J.keys.p, J.bits.p, J.d_out);
  } else {
    if ((st = mark(3))) return st;
    if (multi) k_finalize<M2S_SIGN_NORMAL, true><<<fb, 256, 0, s>>>(J.gs, J.keys.p, nullptr, J.d_out);
    else k_finalize<M2S_SIGN_NORMAL, false><<<fb, 256, 0, s>>>(J.gs, J.keys.p, nullptr, J.d_out);
  }
  M2S_CUDA(cudaGetLastError());
  ++J.launches;
  if (J.audit) {  // reports only: the output is written already
    if (raycast) {
      if (multi) k_audit_cells<M2S_SIGN_RAYCAST, true><<<fb, 256, 0, s>>>(J.gs, J.tris, J.keys.p, J.bits.p, J.bits64.p, J.state.p);
      else k_audit_cells<M2S_SIGN_RAYCAST, false><<<fb, 256, 0, s>>>(J.gs, J.tris, J.keys.p, J.bits.p, J.bits64.p, J.state.p);
    } else {
      if (multi) k_audit_cells<M2S_SIGN_NORMAL, true><<<fb, 256, 0, s>>>(J.gs, J.tris, J.keys.p, nullptr, nullptr, J.state.p);
      else k_audit_cells<M2S_SIGN_NORMAL, false><<<fb, 256, 0, s>>>(J.gs, J.tris, J.keys.p, nullptr, nullptr, J.state.p);
    }
    M2S_CUDA(cudaGetLastError());
    ++J.launches;
  }
  return mark(4);
}

int GridJob::read_state(cudaStream_t s, GridRunInfo* info) {
  Impl& J = *p;
  PropState* h = host_state();
  if (!h) return M2S_ERR_OUT_OF_MEMORY;
  M2S_CUDA(cudaMemcpyAsync(h, J.state.p, sizeof(PropState), cudaMemcpyDeviceToHost, s));
  M2S_CUDA(cudaStreamSynchronize(s));
  info->overflow = (h->overflow | h->overflow2[0] | h->overflow2[1]) != 0;
  info->seeds = h->seeds;
  info->rounds = h->round;
  info->entries = h->entries;
  info->evals = h->evals;
  info->ray_hits = h->ray_hits;
  info->far_phases = h->far_phases;
  info->solo_rounds = h->solo_rounds;
  info->max_list = h->max_list;
  info->log_n = h->log_n;
  info->filter_same = h->filter_same;
  info->filter_bound = h->filter_bound;
  for (int k = 0; k < kAuditStats; ++k) info->audit[k] = h->audit[k];
  info->launches = J.launches;
  return M2S_OK;
}

int run_grid_job(GridJob& job, cudaStream_t s, uint64_t stats[kGridStats], float phase_ms[4]) {
  cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  struct EvFree {
    cudaEvent_t* e;
    ~EvFree() {
      for (int i = 0; i < 5; ++i)
        if (e[i]) cudaEventDestroy(e[i]);
    }
  } evf{ev};
  if (phase_ms)
    for (auto& e : ev) M2S_CUDA(cudaEventCreate(&e));
  GridRunInfo info;
  uint32_t restarts = 0;
  int st;
  if (phase_ms && (st = job.enable_round_log(1u << 16, s))) return st;
  for (;; ++restarts) {
    if ((st = job.alloc_lists(s))) return st;
    if ((st = job.enqueue(s, phase_ms ? ev : nullptr))) return st;
    if ((st = job.read_state(s, &info))) return st;
    if (!info.overflow) break;
    if (restarts >= 6 || job.capacity() >= 0x40000000u) {
      set_error("grid propagation lists overflowed at the largest capacity");
      return M2S_ERR_LIMIT;
    }
    job.set_capacity(job.capacity() * 2);  // the rerun starts over from an empty grid
  }
  if (stats) {
    stats[0] = info.seeds;
    stats[1] = info.rounds;
    stats[2] = info.entries;
    stats[3] = info.evals;
    stats[4] = info.ray_hits;
    stats[5] = restarts;
    stats[6] = info.launches;
    stats[7] = info.far_phases;
    stats[8] = info.solo_rounds;
    stats[9] = info.max_list;
    stats[10] = info.filter_same;
    stats[11] = info.filter_bound;
    for (int k = 0; k < kAuditStats; ++k) stats[12 + k] = info.audit[k];
  }
  if (phase_ms) {
    for (int i = 0; i < 4; ++i) M2S_CUDA(cudaEventElapsedTime(&phase_ms[i], ev[i], ev[i + 1]));
    std::vector<uint32_t> log;
    if ((st = job.read_round_log(&log, (uint32_t)info.log_n, s))) return st;
    record_round_log(log);
  }
  return M2S_OK;
}

std::vector<std::vector<uint32_t>> plan_waves(const GridDesc* gds, uint32_t n, uint64_t wave_cells) {
  std::vector<uint32_t> order(n);
  for (uint32_t k = 0; k < n; ++k) order[k] = k;
  std::stable_sort(order.begin(), order.end(),
                   [&](uint32_t a, uint32_t b) { return gds[a].cells() > gds[b].cells(); });
  std::vector<std::vector<uint32_t>> waves;
  std::vector<uint64_t> fill;
  for (uint32_t k : order) {  // first fit, largest grids first
    const uint64_t c = gds[k].cells();
    size_t w = 0;
    while (w < waves.size() && fill[w] + c > wave_cells) ++w;
    if (w == waves.size()) {
      waves.emplace_back();
      fill.push_back(0);
    }
    waves[w].push_back(k);
    fill[w] += c;
  }
  for (auto& w : waves) std::sort(w.begin(), w.end());  // keep triangle/grid order inside a wave
  return waves;
}

int prepare_waves(const MeshView* meshes, uint32_t n, const GridDesc* gds, int sign, float* d_out, uint32_t* d_status,
                  cudaStream_t s, const GridTuning& tune, std::vector<std::unique_ptr<GridJob>>* jobs) {
  std::vector<uint64_t> out_off(n);
  uint64_t acc = 0;
  for (uint32_t k = 0; k < n; ++k) {
    out_off[k] = acc;
    acc += gds[k].cells();
  }
  const uint64_t wave = tune.wave_cells ? tune.wave_cells : ~0ull;
  for (const auto& w : plan_waves(gds, n, wave)) {
    std::vector<MeshView> m;
    std::vector<GridDesc> g;
    std::vector<uint64_t> o;
    for (uint32_t k : w) {
      m.push_back(meshes[k]);
      g.push_back(gds[k]);
      o.push_back(out_off[k]);
    }
    jobs->emplace_back(new GridJob());
    int st = jobs->back()->prepare(m.data(), (uint32_t)w.size(), g.data(), sign, d_out, d_status, s, tune, o.data());
    if (st) return st;
  }
  return M2S_OK;
}

int grid_sdf_batch(const MeshView* meshes, uint32_t n, const GridDesc* gds, int sign, float* d_out, uint32_t* d_status,
                   cudaStream_t s, uint64_t stats[kGridStats], float phase_ms[4], const GridTuning& tune) {
  if (n == 0) return M2S_OK;
  for (uint32_t k = 0; k < n; ++k) {
    int st = check_grid(gds[k]);
    if (st) return st;
  }
  std::vector<uint64_t> out_off(n);
  uint64_t acc = 0;
  for (uint32_t k = 0; k < n; ++k) {
    out_off[k] = acc;
    acc += gds[k].cells();
  }
  uint64_t total[kGridStats] = {};
  float ms[4] = {0, 0, 0, 0};
  // One job at a time, so only one workspace is alive.
  for (const auto& w : plan_waves(gds, n, tune.wave_cells ? tune.wave_cells : ~0ull)) {
    std::vector<MeshView> m;
    std::vector<GridDesc> g;
    std::vector<uint64_t> o;
    for (uint32_t k : w) {
      m.push_back(meshes[k]);
      g.push_back(gds[k]);
      o.push_back(out_off[k]);
    }
    GridJob job;
    int st = job.prepare(m.data(), (uint32_t)w.size(), g.data(), sign, d_out, d_status, s, tune, o.data());
    if (st) return st;
    uint64_t one[kGridStats] = {};
    float pm[4] = {0, 0, 0, 0};
    if ((st = run_grid_job(job, s, one, phase_ms ? pm : nullptr))) return st;
    for (int i = 0; i < kGridStats; ++i) total[i] = i == 9 ? std::max(total[i], one[i]) : total[i] + one[i];
    for (int i = 0; i < 4; ++i) ms[i] += pm[i];
  }
  if (stats)
    for (int i = 0; i < kGridStats; ++i) stats[i] = total[i];
  if (phase_ms)
    for (int i = 0; i < 4; ++i) phase_ms[i] = ms[i];
  return M2S_OK;
}

namespace {
std::mutex g_grid_tuning_mu;
GridTuning g_grid_tuning;
}  // namespace

GridTuning grid_tuning() {
  std::lock_guard<std::mutex> lk(g_grid_tuning_mu);
  return g_grid_tuning;
}

void set_grid_tuning(const GridTuning& t) {
  std::lock_guard<std::mutex> lk(g_grid_tuning_mu);
  g_grid_tuning = t;
}

int grid_sdf(const MeshView& m, const GridDesc& gd, int sign, float* d_out, uint32_t* d_status, cudaStream_t s,
             uint64_t stats[kGridStats], float phase_ms[4]) {
  if (gd.cells() == 0) return M2S_OK;
  return grid_sdf_batch(&m, 1, &gd, sign, d_out, d_status, s, stats, phase_ms, grid_tuning());
}

}  // namespace m2s

using namespace m2s;

extern "C" int m2s_test_grid_barrier(uint32_t blocks, uint32_t expected, uint32_t out[2]) {
  if (!out || blocks == 0 || blocks > 64 || expected == 0 || expected > 64) return M2S_ERR_INVALID_ARGUMENT;
  int st;
  if ((st = require_device())) return st;
  cudaStream_t s = nullptr;
  DevBuf<GridBarrier> bar;
  DevBuf<unsigned int> res;
  if ((st = bar.alloc(1, s)) || (st = res.alloc(2, s))) return st;
  M2S_CUDA(cudaMemsetAsync(bar.p, 0, sizeof(GridBarrier), s));
  M2S_CUDA(cudaMemsetAsync(res.p, 0, 8, s));
  k_barrier_probe<<<blocks, 64, 0, s>>>(bar.p, expected, res.p);
  M2S_CUDA(cudaGetLastError());
  M2S_CUDA(cudaMemcpyAsync(out, res.p, 8, cudaMemcpyDeviceToHost, s));
  M2S_CUDA(cudaStreamSynchronize(s));
  return M2S_OK;
}
