// generate_grid_sdf on the device (generate/grid.rs:265-684).
//
// 1. Seeding (generate_preheap, grid.rs:383-457): one warp per triangle walks
//    the cells of its padded, snapped and widened box and keeps, per cell, the
//    best (distance, triangle) under compare_distances.  Cells hold a packed
//    64-bit key: high word = f32 bits of the distance, low word = triangle.
// 2. Propagation (generate_heap + propagate_heap, grid.rs:464-558): the
//    reference pops (cell, triangle) states from heaps in distance order and
//    evaluates the popped triangle on the 27 cells of the 3x3x3 block, keeping
//    strict improvements.  Here the heap becomes delta-stepping: states are
//    binned by distance (bucket width a quarter of the smallest cell size) and
//    each round relaxes the lowest non-empty bucket, one warp per state and one
//    lane per neighbour.  A proposal competes with the cell's value at the
//    start of the round; the round's best proposal per cell wins and is queued
//    for further propagation.  The result does not depend on the order of
//    atomics, and on the reference's own test meshes it stays closer to the
//    single-heap reference than the reference's multi-threaded heaps do.
// 3. Sign (compute_raycasts, grid.rs:568-684): every triangle is tested, with
//    the reference's aligned ray test, against the rays that start at the cell
//    centres of the three low faces and lie in its padded box.  A hit at t
//    toggles bit k = min(floor(t / size), n - 1) of that ray's column; a
//    suffix XOR turns toggles into per-cell crossing parities, and a cell is
//    inside when at least two of its three parities are odd (grid.rs:622-639).
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>

#include "m2s_internal.cuh"

namespace m2s {
namespace {

constexpr uint32_t NO_TRI = 0xFFFFFFFFu;
constexpr unsigned long long KEY_EMPTY = (0x7F7FFFFFull << 32) | 0xFFFFFFFFull;  // (f32::MAX, none)
constexpr int kRing = 16;            // pending distance buckets
constexpr uint32_t kMaxRounds = 1u << 22;  // bound on propagation rounds

// Unsigned 32-bit division by an invariant divisor with a multiply-high and
// two shifts (Granlund & Montgomery, "Division by invariant integers using
// multiplication", PLDI 1994, Figure 4.1): exact for every 32-bit dividend.
struct FastDiv {
  uint32_t d, m, s1, s2;
};
inline FastDiv make_fastdiv(uint32_t d) {
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

struct GridK {
  float f[3], s[3];
  int n[3];
  unsigned long long ncell;
  float inv_delta;  // 1 / bucket width
  FastDiv div_z;    // by n[2]
  FastDiv div_y;    // by n[1]
};

// (x, y, z) of a cell index (grid.rs:127-132), 32-bit indices.
__device__ __forceinline__ void cell_coords(const GridK& g, uint32_t cell, int* x, int* y, int* z) {
  uint32_t q = fdiv(g.div_z, cell);
  *z = (int)(cell - q * (uint32_t)g.n[2]);
  uint32_t xx = fdiv(g.div_y, q);
  *y = (int)(q - xx * (uint32_t)g.n[1]);
  *x = (int)xx;
}

struct PropState {
  unsigned long long b;  // current bucket
  uint32_t slot[kRing];  // list holding bucket b + k
  uint32_t cur;          // list relaxed this round
  uint32_t count[kRing + 1];
  uint32_t touched;
  uint32_t touched2[2];  // persistent kernel: touched count per round parity
  uint32_t done;
  uint32_t overflow;
  uint32_t round;
  unsigned long long entries, evals, seeds, ray_hits;
  unsigned long long min_bucket;
};

__device__ __forceinline__ P3 center(const GridK& g, int x, int y, int z) {
  // grid.rs:135-141: first + (i as f32) * size
  return {fa(g.f[0], fm(__int2float_rn(x), g.s[0])), fa(g.f[1], fm(__int2float_rn(y), g.s[1])),
          fa(g.f[2], fm(__int2float_rn(z), g.s[2]))};
}
__device__ __forceinline__ unsigned long long cell_index(const GridK& g, int x, int y, int z) {
  return (unsigned long long)z + (unsigned long long)y * g.n[2] + (unsigned long long)x * g.n[1] * g.n[2];
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
  if (SIGN == M2S_SIGN_RAYCAST) return fsqrt(point_triangle_distance2(pos, a, b, c, kind));
  return point_triangle_signed_distance(pos, a, b, c, kind);
}

__device__ __forceinline__ unsigned long long pack(float d, uint32_t tri) {
  return ((unsigned long long)__float_as_uint(d) << 32) | tri;
}
__device__ __forceinline__ float key_dist(unsigned long long k) { return __uint_as_float((uint32_t)(k >> 32)); }
__device__ __forceinline__ uint32_t key_tri(unsigned long long k) { return (uint32_t)k; }

// Does `cand` beat `cur`?  Raycast: plain order of non-negative distances,
// ties to the lower triangle.  Normal: compare_distances (lib.rs:315-332),
// exact ties to the lower triangle.
template <int SIGN>
__device__ __forceinline__ bool beats(unsigned long long cand, unsigned long long cur, bool* nan) {
  if (SIGN == M2S_SIGN_RAYCAST) return cand < cur;
  float d = key_dist(cand), o = key_dist(cur);
  int c = compare_distances(d, o, nan);
  return c == -1 || (c == 0 && (uint32_t)(cand >> 32) == (uint32_t)(cur >> 32) && key_tri(cand) < key_tri(cur));
}

// Lowers *slot to cand if cand beats it; returns true when this call moved the
// cell off `snap`, its value at the start of the round — exactly one proposal
// per touched cell and round sees that.
template <int SIGN>
__device__ __forceinline__ bool improve_first(unsigned long long* slot, unsigned long long cand, unsigned long long snap,
                                              bool* nan) {
  if (SIGN == M2S_SIGN_RAYCAST) return atomicMin(slot, cand) == snap;
  unsigned long long old = *(volatile unsigned long long*)slot;
  while (beats<SIGN>(cand, old, nan)) {
    unsigned long long prev = atomicCAS(slot, old, cand);
    if (prev == old) return old == snap;
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

__global__ void k_fill_u64(unsigned long long* p, unsigned long long n, unsigned long long v) {
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (unsigned long long)gridDim.x * blockDim.x)
    p[i] = v;
}

// ---- 1. seeding -------------------------------------------------------------
template <int SIGN>
__global__ void k_seed(GridK g, const TriRec* __restrict__ tris, uint32_t T, unsigned long long* keys,
                       uint32_t* status, PropState* st) {
  const uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (t >= T) return;
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
  for (long long k = lane; k < total; k += 32) {
    int z = mn[2] + (int)(k % ez);
    int y = mn[1] + (int)((k / ez) % ey);
    int x = mn[0] + (int)(k / (ez * ey));
    float d = cell_distance<SIGN>(center(g, x, y, z), a, b, c, kind);
    if (isnan(d)) nan = true;
    if (update_min<SIGN>(&keys[cell_index(g, x, y, z)], pack(d, t), &nan)) ++updates;
  }
  if (nan) atomicOr(status, bit(M2S_ERR_NAN_DISTANCE));
  for (int o = 16; o; o >>= 1) updates += __shfl_xor_sync(0xFFFFFFFFu, updates, o);
  if (lane == 0 && updates) atomicAdd(&st->seeds, (unsigned long long)updates);
}

// Distance bucket of a state.  Buckets are a quarter cell wide for the first
// kLinearBuckets (8 cells) and widen in proportion to the distance beyond, so
// the far field, where many triangles are nearly equidistant, takes few rounds.
constexpr float kLinearBuckets = 32.0f;
__device__ __forceinline__ unsigned long long bucket_of(const GridK& g, float d) {
  float u = fabsf(d) * g.inv_delta;
  if (u > kLinearBuckets) u = kLinearBuckets * (1.0f + logf(u / kLinearBuckets));
  return sat_u64(floorf(u));
}

// Lowest bucket among the seeded cells.
__global__ void k_min_bucket(GridK g, const unsigned long long* keys, PropState* st) {
  unsigned long long best = ULLONG_MAX;
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.ncell;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    unsigned long long k = keys[i];
    if (k != KEY_EMPTY && key_tri(k) != NO_TRI) best = min(best, bucket_of(g, key_dist(k)));
  }
  for (int o = 16; o; o >>= 1) best = min(best, __shfl_xor_sync(0xFFFFFFFFu, best, o));
  if ((threadIdx.x & 31) == 0 && best != ULLONG_MAX) atomicMin(&st->min_bucket, best);
}

__global__ void k_state_init(PropState* st) {
  // Lists 0..kRing-1 hold buckets b..b+kRing-1, list kRing is the relax list.
  st->b = st->min_bucket == ULLONG_MAX ? 0 : st->min_bucket;
  for (int k = 0; k < kRing; ++k) st->slot[k] = k;
  st->cur = kRing;
  for (int k = 0; k <= kRing; ++k) st->count[k] = 0;
  st->touched = 0;
  st->done = 0;
  st->overflow = 0;
}

// Appends (cell, triangle) to the list of its distance bucket.  Lanes of a warp
// that target the same list share one atomicAdd.  Must be called by all 32
// lanes; `act` says whether this lane pushes.
__device__ __forceinline__ void push_entry_warp(const GridK& g, PropState* st, unsigned long long b,
                                                const uint32_t* slots, uint2* lists, uint32_t cap, bool act,
                                                unsigned long long cell, uint32_t tri, float d) {
  const int lane = threadIdx.x & 31;
  uint32_t slot = 0xFFFFFFFFu;
  if (act) {
    unsigned long long nb = bucket_of(g, d);
    unsigned long long rel = nb > b ? nb - b : 0;
    slot = slots[rel >= kRing ? kRing - 1 : rel];
  }
  const uint32_t group = __match_any_sync(0xFFFFFFFFu, slot);
  if (!act) return;
  const int leader = __ffs(group) - 1;
  uint32_t base = 0;
  if (lane == leader) base = atomicAdd(&st->count[slot], (uint32_t)__popc(group));
  base = __shfl_sync(group, base, leader);
  const uint32_t pos = base + __popc(group & ((1u << lane) - 1u));
  if (pos < cap)
    lists[(unsigned long long)slot * cap + pos] = make_uint2((uint32_t)cell, tri);
  else
    atomicOr(&st->overflow, 1u);  // the propagation is redone with larger lists
}

__global__ void k_collect(GridK g, const unsigned long long* keys, PropState* st, uint2* lists, uint32_t cap) {
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long base = (unsigned long long)blockIdx.x * blockDim.x; base < g.ncell; base += stride) {
    const unsigned long long i = base + threadIdx.x;  // warp-uniform loop, lanes mask out past the end
    unsigned long long k = i < g.ncell ? keys[i] : KEY_EMPTY;
    bool act = k != KEY_EMPTY && key_tri(k) != NO_TRI;
    push_entry_warp(g, st, st->b, st->slot, lists, cap, act, i, key_tri(k), key_dist(k));
  }
}

// Picks the next list to relax: the lowest non-empty bucket.
__global__ void k_advance(PropState* st, uint32_t cap) {
  if (st->done) return;
  if (st->overflow) {  // this attempt is void; the host restarts it with larger lists
    st->done = 1;
    return;
  }
  st->count[st->cur] = 0;
  st->touched = 0;
  for (int it = 0; it <= kRing; ++it) {
    uint32_t s0 = st->slot[0];
    if (st->count[s0] > 0) {
      st->slot[0] = st->cur;
      st->cur = s0;
      st->round += 1;
      return;
    }
    st->b += 1;
    for (int k = 0; k + 1 < kRing; ++k) st->slot[k] = st->slot[k + 1];
    st->slot[kRing - 1] = s0;
  }
  st->done = 1;
}

// ---- 2. relaxation rounds (persistent) -------------------------------------
// ---- persistent propagation ---------------------------------------------------
// All rounds in one cooperative launch.  Every block keeps an identical copy of
// the bucket schedule in shared memory and advances it from the global list
// counts after the round's second barrier, so no block waits for a scheduler.
// Two-level arrival counters (groups of kBarrierFan blocks, then the group
// leaders) keep the atomics of a barrier from queueing on one address.  Each
// counter lives in its own 128-byte line.
constexpr int kBarrierFan = 16;
constexpr int kBarrierGroups = 128;  // supports up to 2048 co-resident blocks
struct GridBarrier {
  unsigned int gen;
  unsigned int abort;
  unsigned int pad0[30];
  unsigned int top[32];
  unsigned int group[kBarrierGroups][32];
};

__device__ __forceinline__ unsigned int atom_add_acq_rel(unsigned int* p, unsigned int v) {
  unsigned int old;
  asm volatile("atom.add.acq_rel.gpu.global.u32 %0, [%1], %2;" : "=r"(old) : "l"(p), "r"(v) : "memory");
  return old;
}
__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
  unsigned int v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned int* p, unsigned int v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Sense-reversing barrier over the co-resident blocks of a cooperative launch.
// The wait is bounded: after kBarrierPolls polls it raises `abort`, which makes
// every block leave the kernel at its next barrier.
constexpr uint32_t kBarrierPolls = 1u << 22;  // about a second of polling

__device__ __forceinline__ bool grid_barrier(GridBarrier* bar, unsigned int nblocks) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int g0 = ld_acquire(&bar->gen);
    const unsigned int grp = blockIdx.x / kBarrierFan;
    const unsigned int ngroups = (nblocks + kBarrierFan - 1) / kBarrierFan;
    const unsigned int in_grp = min((unsigned)kBarrierFan, nblocks - grp * kBarrierFan);
    bool last = false;
    if (atom_add_acq_rel(&bar->group[grp][0], 1u) == in_grp - 1) {
      bar->group[grp][0] = 0;  // nobody touches this counter again before the release below
      last = atom_add_acq_rel(&bar->top[0], 1u) == ngroups - 1;
    }
    if (last) {
      bar->top[0] = 0;
      st_release(&bar->gen, g0 + 1);
    } else {
      uint32_t polls = 0;
      while (ld_acquire(&bar->gen) == g0) {
        if (ld_acquire(&bar->abort)) break;
        if (++polls > kBarrierPolls) {
          atomicExch(&bar->abort, 1u);
          break;
        }
      }
    }
    ok = ld_acquire(&bar->abort) ? 0 : 1;
  }
  __syncthreads();
  return ok != 0;
}

constexpr int kTouchStage = 2048;  // touched cells staged per block and round

struct Sched {
  unsigned long long b;
  uint32_t slot[kRing];
  uint32_t cur;
  uint32_t round;
  uint32_t done;
};

template <int SIGN>
__global__ void __launch_bounds__(256) k_propagate(GridK g, const TriRec* __restrict__ tris,
                                                   unsigned long long* snap_keys, unsigned long long* work_keys,
                                                   uint2* lists, uint32_t cap, uint32_t* touched_lists,
                                                   PropState* st, GridBarrier* bar, uint32_t max_rounds,
                                                   uint32_t* status) {
  __shared__ Sched sh;
  __shared__ uint32_t s_touch[kTouchStage];
  __shared__ uint32_t s_ntouch, s_touch_base;
  const unsigned int nblocks = gridDim.x;
  const int lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    s_ntouch = 0;
    sh.b = st->b;
    for (int k = 0; k < kRing; ++k) sh.slot[k] = st->slot[k];
    sh.cur = st->cur;
    sh.round = st->round;
    sh.done = st->done;
  }
  __syncthreads();
  bool nan = false;
  unsigned long long evals = 0;
  uint32_t prev_cur = 0xFFFFFFFFu;
  bool aborted = false;
  for (uint32_t it = 0; !sh.done; ++it) {
    if (it >= max_rounds) {
      if (blockIdx.x == 0 && threadIdx.x == 0) atomicOr(status, bit(M2S_ERR_LIMIT));
      break;
    }
    const uint32_t parity = sh.round & 1u;
    uint32_t* touched_list = touched_lists + (unsigned long long)parity * cap;
    // ---- propose: every state of the bucket evaluates its triangle at the 27
    // cells of its 3x3x3 block (one lane per cell); a proposal that beats the
    // cell's value at the start of the round enters the working value (atomic
    // minimum) and the first such proposal lists the cell as touched.
    if (blockIdx.x == 0 && threadIdx.x == 0 && prev_cur != 0xFFFFFFFFu) st->count[prev_cur] = 0;
    const uint32_t n = min(*(volatile uint32_t*)&st->count[sh.cur], cap);
    const uint2* list = lists + (unsigned long long)sh.cur * cap;
    // One thread per (state, neighbour) proposal; consecutive threads share a
    // state, so its entry and triangle loads are warp broadcasts.  Two
    // independent proposals per iteration keep two load chains in flight.
    // Thread t takes proposals t, t + T, t + 2T, ... as (state e, neighbour k)
    // pairs advanced without division: T = 27 * dE + dK.
    const uint32_t T = gridDim.x * blockDim.x;
    const uint32_t dE = T / 27u, dK = T % 27u;
    const uint32_t t0 = blockIdx.x * blockDim.x + threadIdx.x;
    uint32_t e = t0 / 27u, k = t0 % 27u;
    while (e < n) {
      bool first[2] = {false, false};
      unsigned long long jj[2] = {0, 0};
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const uint32_t eu = e, ku = k;
        k += dK;
        e += dE;
        if (k >= 27u) {
          k -= 27u;
          ++e;
        }
        if (eu >= n) continue;
        const uint2 ent = __ldcg(&list[eu]);  // written by other blocks last round
        const uint32_t tri = ent.y;
        int x, y, z;
        cell_coords(g, ent.x, &x, &y, &z);
        // iproduct!(-1..=1, -1..=1, -1..=1) order (grid.rs:512): x outermost.
        const int X = x + (int)(ku / 9u) - 1, Y = y + (int)((ku / 3u) % 3u) - 1, Z = z + (int)(ku % 3u) - 1;
        if (X < 0 || Y < 0 || Z < 0 || X >= g.n[0] || Y >= g.n[1] || Z >= g.n[2]) continue;
        const uint32_t j = (uint32_t)Z + (uint32_t)Y * (uint32_t)g.n[2] + (uint32_t)X * ((uint32_t)g.n[1] * (uint32_t)g.n[2]);
        const unsigned long long snap = __ldcg(&snap_keys[j]);
        const TriRec r = tris[tri];
        const float d = cell_distance<SIGN>(center(g, X, Y, Z), p3(r.a), p3(r.b), p3(r.c), __float_as_int(r.a.w));
        ++evals;
        if (isnan(d)) nan = true;
        const unsigned long long cand = pack(d, tri);
        if (beats<SIGN>(cand, snap, &nan)) {
          first[u] = improve_first<SIGN>(&work_keys[j], cand, snap, &nan);
          jj[u] = j;
        }
      }
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const unsigned long long j = jj[u];
        if (first[u]) {
          const uint32_t q = atomicAdd(&s_ntouch, 1u);
          if (q < kTouchStage) {
            s_touch[q] = (uint32_t)j;
          } else {
            const uint32_t pos = atomicAdd(&st->touched2[parity], 1u);
            if (pos < cap) touched_list[pos] = (uint32_t)j;
            else atomicOr(&st->overflow, 1u);
          }
        }
      }
    }
    // flush this block's staged touched cells with one global atomic
    __syncthreads();
    {
      const uint32_t nloc = min(s_ntouch, (uint32_t)kTouchStage);
      if (threadIdx.x == 0) {
        s_touch_base = nloc ? atomicAdd(&st->touched2[parity], nloc) : 0;
        s_ntouch = 0;
      }
      __syncthreads();
      for (uint32_t i = threadIdx.x; i < nloc; i += blockDim.x) {
        const uint32_t pos = s_touch_base + i;
        if (pos < cap) touched_list[pos] = s_touch[i];
        else atomicOr(&st->overflow, 1u);
      }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) atomicAdd(&st->entries, (unsigned long long)n);
    if (!grid_barrier(bar, nblocks)) {
      aborted = true;
      break;
    }
    // ---- commit: each touched cell publishes its round winner to the snapshot
    // and queues (cell, winning triangle) in the winner's distance bucket.
    if (blockIdx.x == 0 && threadIdx.x == 0) st->touched2[parity ^ 1u] = 0;
    const uint32_t nt = min(*(volatile uint32_t*)&st->touched2[parity], cap);
    for (uint32_t base = blockIdx.x * blockDim.x; base < nt; base += gridDim.x * blockDim.x) {
      const uint32_t i = base + threadIdx.x;
      const bool act = i < nt;
      unsigned long long j = 0, w = KEY_EMPTY;
      if (act) {
        j = __ldcg(&touched_list[i]);
        w = __ldcg(&work_keys[j]);
        snap_keys[j] = w;
      }
      push_entry_warp(g, st, sh.b, sh.slot, lists, cap, act, j, key_tri(w), key_dist(w));
    }
    if (!grid_barrier(bar, nblocks)) {
      aborted = true;
      break;
    }
    // ---- advance (every block, identically)
    if (threadIdx.x == 0) {
      const uint32_t consumed = sh.cur;
      if (*(volatile uint32_t*)&st->overflow) {
        sh.done = 1;
      } else {
        bool found = false;
        for (int k = 0; k <= kRing && !found; ++k) {
          uint32_t s0 = sh.slot[0];
          if (*(volatile uint32_t*)&st->count[s0] > 0) {
            sh.slot[0] = consumed;
            sh.cur = s0;
            sh.round += 1;
            found = true;
          } else {
            sh.b += 1;
            for (int q = 0; q + 1 < kRing; ++q) sh.slot[q] = sh.slot[q + 1];
            sh.slot[kRing - 1] = s0;
          }
        }
        if (!found) sh.done = 1;
      }
    }
    __syncthreads();
    prev_cur = sh.slot[0];  // the consumed list now sits in slot 0 (or the schedule is done)
  }
  if (nan) atomicOr(status, bit(M2S_ERR_NAN_DISTANCE));
  for (int o = 16; o; o >>= 1) evals += __shfl_xor_sync(0xFFFFFFFFu, evals, o);
  if (lane == 0 && evals) atomicAdd(&st->evals, evals);
  if (aborted && blockIdx.x == 0 && threadIdx.x == 0) atomicOr(status, bit(M2S_ERR_LIMIT));
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->round = sh.round;
    st->done = 1;
  }
}

// ---- 3. rays -------------------------------------------------------------------
struct RayK {
  uint32_t* bits[3];  // per axis: column-major toggles, words[col * W + w]
  uint32_t words[3];  // W per axis
};

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

template <int AXIS>
__global__ void k_rays(GridK g, const TriRec* __restrict__ tris, uint32_t T, RayK rk, PropState* st) {
  constexpr int IY = (AXIS + 1) % 3, IZ = (AXIS + 2) % 3;
  const uint32_t t = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (t >= T) return;
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
  uint32_t* bitsA = rk.bits[AXIS];
  const uint32_t W = rk.words[AXIS];
  uint32_t hits = 0;
  for (long long q = lane; q < total; q += 32) {
    int c3[3];
    c3[AXIS] = 0;
    c3[IY] = j0 + (int)(q / nk);
    c3[IZ] = k0 + (int)(q % nk);
    P3 o = center(g, c3[0], c3[1], c3[2]);  // ray origin: a low-face cell centre (grid.rs:580)
    float tt;
    if (!ray_hit_aligned<AXIS>(o, a, b, c, &tt)) continue;
    ++hits;
    // grid.rs:604-607
    unsigned long long kk = sat_u64(floorf(fd(tt, g.s[AXIS])));
    unsigned long long last = (unsigned long long)g.n[AXIS] - 1;
    uint32_t k = (uint32_t)(kk < last ? kk : last);
    unsigned long long col = column_of(g, AXIS, c3[0], c3[1], c3[2]);
    atomicXor(&bitsA[col * W + (k >> 5)], 1u << (k & 31));
  }
  for (int o = 16; o; o >>= 1) hits += __shfl_xor_sync(0xFFFFFFFFu, hits, o);
  if (lane == 0 && hits) atomicAdd(&st->ray_hits, (unsigned long long)hits);
}

// Toggle bits -> suffix parity: bit i becomes the XOR of toggles i..n-1, i.e.
// the parity of the hits whose cell range 0..=k covers cell i.
__global__ void k_suffix(uint32_t* bits, unsigned long long ncols, uint32_t W) {
  for (unsigned long long col = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; col < ncols;
       col += (unsigned long long)gridDim.x * blockDim.x) {
    uint32_t carry = 0;
    uint32_t* w = bits + col * W;
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

template <int SIGN>
__global__ void k_finalize(GridK g, const unsigned long long* __restrict__ keys, RayK rk, float* __restrict__ out) {
  for (unsigned long long i = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; i < g.ncell;
       i += (unsigned long long)gridDim.x * blockDim.x) {
    float d = key_dist(keys[i]);
    if (SIGN == M2S_SIGN_RAYCAST) {
      int z = (int)(i % g.n[2]);
      int y = (int)((i / g.n[2]) % g.n[1]);
      int x = (int)(i / ((unsigned long long)g.n[1] * g.n[2]));
      uint32_t px = (rk.bits[0][column_of(g, 0, x, y, z) * rk.words[0] + (x >> 5)] >> (x & 31)) & 1u;
      uint32_t py = (rk.bits[1][column_of(g, 1, x, y, z) * rk.words[1] + (y >> 5)] >> (y & 31)) & 1u;
      uint32_t pz = (rk.bits[2][column_of(g, 2, x, y, z) * rk.words[2] + (z >> 5)] >> (z & 31)) & 1u;
      if (px + py + pz >= 2) d = -d;
    }
    out[i] = d;
  }
}

unsigned blocks_for(unsigned long long n, int threads, unsigned cap = 148u * 16u) {
  unsigned long long b = (n + threads - 1) / threads;
  return (unsigned)std::max<unsigned long long>(1, std::min<unsigned long long>(b, cap));
}

}  // namespace

int grid_sdf(const MeshView& m, const GridDesc& gd, int sign, float* d_out, uint32_t* d_status, cudaStream_t s,
             uint64_t stats[kGridStats], float phase_ms[4]) {
  const unsigned long long N = gd.cells();
  if (N == 0) return M2S_OK;
  for (int d = 0; d < 3; ++d)
    if (gd.n[d] > 0x7FFFFFFFull) return M2S_ERR_INVALID_ARGUMENT;
  if (N > 0xFFFFFFFFull) return M2S_ERR_INVALID_ARGUMENT;  // cells are addressed with 32-bit entries
  GridK g;
  for (int d = 0; d < 3; ++d) {
    g.f[d] = gd.first[d];
    g.s[d] = gd.size[d];
    g.n[d] = (int)gd.n[d];
  }
  g.ncell = N;
  g.div_z = make_fastdiv((uint32_t)g.n[2]);
  g.div_y = make_fastdiv((uint32_t)g.n[1]);
  float minsize = std::min(std::fabs(g.s[0]), std::min(std::fabs(g.s[1]), std::fabs(g.s[2])));
  float delta = 0.25f * minsize;
  g.inv_delta = (delta > 0.0f && std::isfinite(delta)) ? 1.0f / delta : 1.0f;

  const uint32_t T = m.n_tris;
  uint64_t launches = 0;
  // Phase events (seeding, propagation, rays, finalize) when asked for.
  cudaEvent_t ev[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
  if (phase_ms)
    for (auto& e : ev) M2S_CUDA(cudaEventCreate(&e));
  struct EvFree {
    cudaEvent_t* e;
    ~EvFree() {
      for (int i = 0; i < 5; ++i)
        if (e[i]) cudaEventDestroy(e[i]);
    }
  } evf{ev};
  auto mark = [&](int i) {
    if (phase_ms) cudaEventRecord(ev[i], s);
  };
  mark(0);
  DevBuf<unsigned long long> snap_keys, work_keys;
  DevBuf<PropState> state;
  int st;
  if ((st = snap_keys.alloc(N, s)) || (st = state.alloc(1, s))) return st;
  M2S_CUDA(cudaMemsetAsync(state.p, 0, sizeof(PropState), s));
  k_fill_u64<<<blocks_for(N, 256), 256, 0, s>>>(snap_keys.p, N, KEY_EMPTY);
  M2S_CUDA(cudaGetLastError());
  ++launches;

  if (T > 0) {
    unsigned sb = (unsigned)((T * 32ull + 255) / 256);
    uint32_t cap = (uint32_t)std::min<unsigned long long>(std::max<unsigned long long>(N / 2, 1ull << 20),
                                                          0x7FFFFFFFull);
    PropState* hst = nullptr;
    M2S_CUDA(cudaMallocHost(&hst, sizeof(PropState)));
    struct HostFree {
      PropState* p;
      ~HostFree() { cudaFreeHost(p); }
    } hf{hst};
    if ((st = work_keys.alloc(N, s))) return st;
    uint32_t rounds_launched = 0, attempts = 0;
    for (;; ++attempts) {
      // ---- seeding (redone on a restart so every attempt starts from the same state)
      if (attempts > 0) {
        k_fill_u64<<<blocks_for(N, 256), 256, 0, s>>>(snap_keys.p, N, KEY_EMPTY);
        M2S_CUDA(cudaMemsetAsync(state.p, 0, sizeof(PropState), s));
        ++launches;
      }
      if (sign == M2S_SIGN_RAYCAST)
        k_seed<M2S_SIGN_RAYCAST><<<sb, 256, 0, s>>>(g, m.tris, T, snap_keys.p, d_status, state.p);
      else
        k_seed<M2S_SIGN_NORMAL><<<sb, 256, 0, s>>>(g, m.tris, T, snap_keys.p, d_status, state.p);
      M2S_CUDA(cudaGetLastError());
      ++launches;
      if (attempts == 0) mark(1);

      // ---- propagation: one cooperative launch runs every round
      DevBuf<uint2> lists;
      DevBuf<uint32_t> touched;
      DevBuf<GridBarrier> bar;
      if ((st = lists.alloc((kRing + 1ull) * cap, s)) || (st = touched.alloc(2ull * cap, s)) ||
          (st = bar.alloc(1, s)))
        return st;
      M2S_CUDA(cudaMemsetAsync(bar.p, 0, sizeof(GridBarrier), s));
      M2S_CUDA(cudaMemcpyAsync(work_keys.p, snap_keys.p, N * 8, cudaMemcpyDeviceToDevice, s));
      unsigned long long ull_max = ULLONG_MAX;
      M2S_CUDA(cudaMemcpyAsync(&state.p->min_bucket, &ull_max, 8, cudaMemcpyHostToDevice, s));
      k_min_bucket<<<blocks_for(N, 256), 256, 0, s>>>(g, snap_keys.p, state.p);
      k_state_init<<<1, 1, 0, s>>>(state.p);
      k_collect<<<blocks_for(N, 256), 256, 0, s>>>(g, snap_keys.p, state.p, lists.p, cap);
      k_advance<<<1, 1, 0, s>>>(state.p, cap);
      M2S_CUDA(cudaGetLastError());
      launches += 4;
      {
        void* kern = sign == M2S_SIGN_RAYCAST ? (void*)k_propagate<M2S_SIGN_RAYCAST> : (void*)k_propagate<M2S_SIGN_NORMAL>;
        int dev = 0, sms = 0, per_sm = 0;
        M2S_CUDA(cudaGetDevice(&dev));
        M2S_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        M2S_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, 256, 0));
        if (per_sm < 1) return M2S_ERR_CUDA;
        if (sms * per_sm > kBarrierFan * kBarrierGroups) per_sm = (kBarrierFan * kBarrierGroups) / sms;
        dim3 grid_dim((unsigned)(sms * per_sm)), block_dim(256);
        const TriRec* tris_p = m.tris;
        unsigned long long* snap_p = snap_keys.p;
        unsigned long long* work_p = work_keys.p;
        uint2* lists_p = lists.p;
        uint32_t* touched_p = touched.p;
        PropState* st_p = state.p;
        GridBarrier* bar_p = bar.p;
        uint32_t max_rounds = kMaxRounds;
        void* args[] = {&g, &tris_p, &snap_p, &work_p, &lists_p, &cap, &touched_p, &st_p, &bar_p, &max_rounds,
                        &d_status};
        M2S_CUDA(cudaLaunchCooperativeKernel(kern, grid_dim, block_dim, args, 0, s));
        ++launches;
      }
      M2S_CUDA(cudaMemcpyAsync(hst, state.p, sizeof(PropState), cudaMemcpyDeviceToHost, s));
      M2S_CUDA(cudaStreamSynchronize(s));
      rounds_launched += hst->round;
      if (!hst->overflow) break;
      if (attempts >= 6 || cap >= 0x40000000u) return M2S_ERR_LIMIT;
      cap *= 2;
    }
    if (stats) {
      stats[0] = hst->seeds;
      stats[1] = hst->round;
      stats[2] = hst->entries;
      stats[3] = hst->evals;
      stats[5] = attempts;
      stats[7] = rounds_launched;
    }
  } else {
    mark(1);
  }
  mark(2);

  // ---- sign: rays + finalize
  RayK rk{};
  DevBuf<uint32_t> rbits[3];
  if (sign == M2S_SIGN_RAYCAST) {
    for (int a = 0; a < 3; ++a) {
      unsigned long long ncols = N / gd.n[a];
      rk.words[a] = (uint32_t)((gd.n[a] + 31) / 32);
      if ((st = rbits[a].alloc(ncols * rk.words[a], s))) return st;
      M2S_CUDA(cudaMemsetAsync(rbits[a].p, 0, ncols * rk.words[a] * 4, s));
      rk.bits[a] = rbits[a].p;
    }
    if (T > 0) {
      unsigned rb = (unsigned)((T * 32ull + 255) / 256);
      k_rays<0><<<rb, 256, 0, s>>>(g, m.tris, T, rk, state.p);
      k_rays<1><<<rb, 256, 0, s>>>(g, m.tris, T, rk, state.p);
      k_rays<2><<<rb, 256, 0, s>>>(g, m.tris, T, rk, state.p);
      M2S_CUDA(cudaGetLastError());
      launches += 3;
    }
    for (int a = 0; a < 3; ++a) {
      unsigned long long ncols = N / gd.n[a];
      k_suffix<<<blocks_for(ncols, 256), 256, 0, s>>>(rk.bits[a], ncols, rk.words[a]);
    }
    launches += 3;
    mark(3);
    k_finalize<M2S_SIGN_RAYCAST><<<blocks_for(N, 256, 148u * 32u), 256, 0, s>>>(g, snap_keys.p, rk, d_out);
    if (stats) {
      unsigned long long h = 0;
      M2S_CUDA(cudaMemcpyAsync(&h, &state.p->ray_hits, 8, cudaMemcpyDeviceToHost, s));
      M2S_CUDA(cudaStreamSynchronize(s));
      stats[4] = h;
    }
  } else {
    mark(3);
    k_finalize<M2S_SIGN_NORMAL><<<blocks_for(N, 256, 148u * 32u), 256, 0, s>>>(g, snap_keys.p, rk, d_out);
  }
  M2S_CUDA(cudaGetLastError());
  ++launches;
  mark(4);
  if (stats) stats[6] = launches;
  if (phase_ms) {
    M2S_CUDA(cudaEventSynchronize(ev[4]));
    for (int i = 0; i < 4; ++i) cudaEventElapsedTime(&phase_ms[i], ev[i], ev[i + 1]);
  }
  return M2S_OK;
}

}  // namespace m2s
