// LBVH build on the device: triangle records, Morton codes, a stable LSD
// radix sort, Karras (2012) binary radix tree emission and a bottom-up refit.
//
// The tree replaces the bvh 0.10 / rstar 0.12 trees of the Rust crate
// (generate/generic/bvh.rs:230-254, rtree.rs:279-304, rtree_bvh.rs:100-141,
// generate/grid.rs:95-114).  Those trees only pre-filter candidates; every
// result is decided by the exact f32 tests of m2s_geo.cuh, so any tree over
// the same padded boxes (geo.rs:4-22) yields the same answers.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "m2s_internal.cuh"

namespace m2s {
namespace {

constexpr int kThreads = 256;

__device__ __forceinline__ uint32_t load_index(const void* idx, int bits, uint64_t k) {
  if (bits == 16) return ((const uint16_t*)idx)[k];
  if (bits == 32) return ((const uint32_t*)idx)[k];
  return (uint32_t)k;
}

// Topology::get_triangles (lib.rs:193-215): a list takes indices 3t..3t+2, a
// strip the window t..t+2 with no winding flip.  Indices >= n_vertices raise
// M2S_ERR_INDEX_RANGE (the crate panics through slice indexing).
__global__ void k_setup(MeshInput in, TriRec* __restrict__ tris, float4* __restrict__ boxes, uint32_t* status) {
  uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= in.n_tris) return;
  uint64_t base = in.topology == 0 ? 3 * t : t;
  uint64_t i0 = in.index_bits ? load_index(in.d_indices, in.index_bits, base) : base;
  uint64_t i1 = in.index_bits ? load_index(in.d_indices, in.index_bits, base + 1) : base + 1;
  uint64_t i2 = in.index_bits ? load_index(in.d_indices, in.index_bits, base + 2) : base + 2;
  if (i0 >= in.n_vertices || i1 >= in.n_vertices || i2 >= in.n_vertices) {
    atomicOr(status, bit(M2S_ERR_INDEX_RANGE));
    i0 = i1 = i2 = 0;
    if (in.n_vertices == 0) return;
  }
  const float* v = in.d_vertices;
  P3 a = {v[3 * i0], v[3 * i0 + 1], v[3 * i0 + 2]};
  P3 b = {v[3 * i1], v[3 * i1 + 1], v[3 * i1 + 2]};
  P3 c = {v[3 * i2], v[3 * i2 + 1], v[3 * i2 + 2]};
  int kind = degenerate_kind(a.x, a.y, a.z, b.x, b.y, b.z, c.x, c.y, c.z);
  TriRec r;
  r.a = make_float4(a.x, a.y, a.z, __int_as_float(kind));
  r.b = make_float4(b.x, b.y, b.z, __uint_as_float((uint32_t)t));
  r.c = make_float4(c.x, c.y, c.z, 0.0f);
  tris[t] = r;
  P3 lo, hi;
  padded_box(a, b, c, &lo, &hi);
  boxes[2 * t] = make_float4(lo.x, lo.y, lo.z, 0.0f);
  boxes[2 * t + 1] = make_float4(hi.x, hi.y, hi.z, 0.0f);
}

// Order-preserving float <-> uint maps for atomic min / max.
__device__ __forceinline__ uint32_t f2o(float f) {
  uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float o2f(uint32_t u) {
  return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

__global__ void k_bounds_init(uint32_t* b) {
  if (threadIdx.x < 3) b[threadIdx.x] = 0xFFFFFFFFu;
  else if (threadIdx.x < 6) b[threadIdx.x] = 0u;
}

// Bounds of the box centroids (the Morton quantisation domain).
__global__ void k_bounds(const float4* __restrict__ boxes, uint64_t n, uint32_t* b) {
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (uint64_t)gridDim.x * blockDim.x) {
    float4 lo = boxes[2 * t], hi = boxes[2 * t + 1];
    float c[3] = {0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y), 0.5f * (lo.z + hi.z)};
    for (int d = 0; d < 3; ++d) {
      mn[d] = fminf(mn[d], c[d]);
      mx[d] = fmaxf(mx[d], c[d]);
    }
  }
  for (int d = 0; d < 3; ++d)
    for (int o = 16; o; o >>= 1) {
      mn[d] = fminf(mn[d], __shfl_xor_sync(0xFFFFFFFFu, mn[d], o));
      mx[d] = fmaxf(mx[d], __shfl_xor_sync(0xFFFFFFFFu, mx[d], o));
    }
  if ((threadIdx.x & 31) == 0)
    for (int d = 0; d < 3; ++d) {
      atomicMin(&b[d], f2o(mn[d]));
      atomicMax(&b[3 + d], f2o(mx[d]));
    }
}

// 10-bit spread: bit i of x moves to bit 3i.
__device__ __forceinline__ uint32_t spread10(uint32_t x) {
  x &= 0x3FFu;
  x = (x | (x << 16)) & 0x030000FFu;
  x = (x | (x << 8)) & 0x0300F00Fu;
  x = (x | (x << 4)) & 0x030C30C3u;
  x = (x | (x << 2)) & 0x09249249u;
  return x;
}

__global__ void k_morton(const float4* __restrict__ boxes, uint64_t n, const uint32_t* b, uint32_t* keys,
                         uint32_t* vals) {
  uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  float4 lo = boxes[2 * t], hi = boxes[2 * t + 1];
  float c[3] = {0.5f * (lo.x + hi.x), 0.5f * (lo.y + hi.y), 0.5f * (lo.z + hi.z)};
  uint32_t q[3];
  for (int d = 0; d < 3; ++d) {
    float mn = o2f(b[d]), mx = o2f(b[3 + d]);
    float ext = mx - mn;
    float u = ext > 0.0f ? (c[d] - mn) / ext : 0.0f;
    u = fminf(fmaxf(u * 1024.0f, 0.0f), 1023.0f);
    q[d] = (uint32_t)u;
  }
  keys[t] = (spread10(q[0]) << 2) | (spread10(q[1]) << 1) | spread10(q[2]);
  vals[t] = (uint32_t)t;
}

// ---- exclusive scan (u32) --------------------------------------------------
constexpr int kScanItems = 4;
constexpr int kScanTile = kThreads * kScanItems;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* total) {
  __shared__ uint32_t warp_sums[kThreads / 32];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) warp_sums[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t s = lane < kThreads / 32 ? warp_sums[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xFFFFFFFFu, s, o);
      if (lane >= o) s += y;
    }
    if (lane < kThreads / 32) warp_sums[lane] = s;
  }
  __syncthreads();
  uint32_t prefix = warp ? warp_sums[warp - 1] : 0;
  *total = warp_sums[kThreads / 32 - 1];
  __syncthreads();
  return prefix + x - v;
}

__global__ void k_scan_tiles(const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* tile_sums) {
  uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
  uint32_t v[kScanItems], s = 0;
  for (int k = 0; k < kScanItems; ++k) {
    v[k] = base + k < n ? in[base + k] : 0;
    s += v[k];
  }
  uint32_t total;
  uint32_t ex = block_exclusive_scan(s, &total);
  for (int k = 0; k < kScanItems; ++k) {
    if (base + k < n) out[base + k] = ex;
    ex += v[k];
  }
  if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

__global__ void k_add_tiles(uint32_t* out, uint64_t n, const uint32_t* tile_offsets) {
  uint64_t base = (uint64_t)blockIdx.x * kScanTile + (uint64_t)threadIdx.x * kScanItems;
  uint32_t add = tile_offsets[blockIdx.x];
  for (int k = 0; k < kScanItems; ++k)
    if (base + k < n) out[base + k] += add;
}

// total = last exclusive prefix + last input (saved before an in-place scan).
__global__ void k_copy_total(const uint32_t* scanned, uint64_t n, const uint32_t* last_in, uint32_t* total) {
  *total = scanned[n - 1] + *last_in;
}

// ---- radix sort ------------------------------------------------------------
constexpr int kSortItems = 8;
constexpr int kSortTile = kThreads * kSortItems;
constexpr int kDigits = 256;

__global__ void k_hist(const uint32_t* __restrict__ keys, uint64_t n, int shift, uint32_t* hist, uint32_t nblocks) {
  __shared__ uint32_t h[kDigits];
  h[threadIdx.x] = 0;
  __syncthreads();
  uint64_t base = (uint64_t)blockIdx.x * kSortTile;
  for (int it = 0; it < kSortItems; ++it) {
    uint64_t k = base + (uint64_t)it * kThreads + threadIdx.x;
    if (k < n) atomicAdd(&h[(keys[k] >> shift) & 0xFFu], 1u);
  }
  __syncthreads();
  hist[(uint64_t)threadIdx.x * nblocks + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter: within a tile, keys keep their input order per digit.  The
// tile is first ordered by digit in shared memory (a key's place: the tile's
// start of its digit, from the scanned offsets, plus the same-digit keys
// before it), then each digit's run is written out contiguously, so
// neighbouring threads write neighbouring addresses.
__global__ void k_scatter(const uint32_t* __restrict__ kin, const uint32_t* __restrict__ vin, uint32_t* kout,
                          uint32_t* vout, uint64_t n, int shift, const uint32_t* offsets, uint32_t nblocks) {
  __shared__ uint32_t run[kDigits];
  __shared__ uint32_t wcnt[kThreads / 32][kDigits];
  __shared__ uint32_t base_off[kDigits];
  __shared__ uint32_t tile_start[kDigits];
  __shared__ uint32_t s_key[kSortTile], s_val[kSortTile];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint64_t base = (uint64_t)blockIdx.x * kSortTile;
  const uint32_t tile_n = (uint32_t)(n - base < (uint64_t)kSortTile ? n - base : (uint64_t)kSortTile);
  {
    // this tile's count of digit d: the next offset (digit-major) minus its own
    const uint64_t idx = (uint64_t)threadIdx.x * nblocks + blockIdx.x;
    const uint32_t off = offsets[idx];
    const uint32_t next = idx + 1 < (uint64_t)kDigits * nblocks ? offsets[idx + 1] : (uint32_t)n;
    base_off[threadIdx.x] = off;
    // exclusive scan of the counts over the 256 digits (one per thread)
    uint32_t c = next - off, incl = c;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, o);
      if (lane >= o) incl += y;
    }
    if (lane == 31) wcnt[0][warp] = incl;
    __syncthreads();
    uint32_t wbase = 0;
    for (int w = 0; w < warp; ++w) wbase += wcnt[0][w];
    tile_start[threadIdx.x] = wbase + incl - c;
    run[threadIdx.x] = 0;
    __syncthreads();
  }
  const uint32_t lt_mask = (1u << lane) - 1u;
  for (int it = 0; it < kSortItems; ++it) {
    for (int w = 0; w < kThreads / 32; ++w) wcnt[w][threadIdx.x] = 0;
    __syncthreads();
    const uint32_t t = (uint32_t)it * kThreads + threadIdx.x;
    const bool valid = t < tile_n;
    const uint32_t key = valid ? kin[base + t] : 0, val = valid ? vin[base + t] : 0;
    const uint32_t digit = valid ? (key >> shift) & 0xFFu : 0x100u;
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, digit);
    const uint32_t lrank = __popc(peers & lt_mask);
    if (valid && lrank == 0) wcnt[warp][digit] = __popc(peers);
    __syncthreads();
    if (valid) {
      uint32_t before = run[digit];
      for (int w = 0; w < warp; ++w) before += wcnt[w][digit];
      const uint32_t pos = tile_start[digit] + before + lrank;  // < tile_n
      s_key[pos] = key;
      s_val[pos] = val;
    }
    __syncthreads();
    uint32_t add = 0;
    for (int w = 0; w < kThreads / 32; ++w) add += wcnt[w][threadIdx.x];
    run[threadIdx.x] += add;
    __syncthreads();
  }
  for (uint32_t t = threadIdx.x; t < tile_n; t += kThreads) {
    const uint32_t key = s_key[t];
    const uint32_t d = (key >> shift) & 0xFFu;
    const uint32_t dst = base_off[d] + (t - tile_start[d]);
    kout[dst] = key;
    vout[dst] = s_val[t];
  }
}

// ---- Karras hierarchy --------------------------------------------------------
__device__ __forceinline__ int kdelta(const uint32_t* __restrict__ k, int n, int i, int j) {
  if (j < 0 || j >= n) return -1;
  uint32_t a = k[i], b = k[j];
  if (a == b) return 32 + __clz((uint32_t)(i ^ j));
  return __clz(a ^ b);
}

__global__ void k_karras(const uint32_t* __restrict__ keys, int n, BvhNode* nodes, uint32_t* node_parent,
                         uint32_t* leaf_parent) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  int d = (kdelta(keys, n, i, i + 1) - kdelta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
  int dmin = kdelta(keys, n, i, i - d);
  long lmax = 2;
  while (kdelta(keys, n, i, (int)(i + lmax * d)) > dmin) lmax *= 2;
  long l = 0;
  for (long t = lmax / 2; t >= 1; t /= 2)
    if (kdelta(keys, n, i, (int)(i + (l + t) * d)) > dmin) l += t;
  int j = (int)(i + l * d);
  int dnode = kdelta(keys, n, i, j);
  long s = 0, t = l;
  do {
    t = (t + 1) >> 1;
    if (kdelta(keys, n, i, (int)(i + (s + t) * d)) > dnode) s += t;
  } while (t > 1);
  int gamma = (int)(i + s * d + min(d, 0));
  uint32_t left = (min(i, j) == gamma) ? (LEAF_BIT | (uint32_t)gamma) : (uint32_t)gamma;
  uint32_t right = (max(i, j) == gamma + 1) ? (LEAF_BIT | (uint32_t)(gamma + 1)) : (uint32_t)(gamma + 1);
  nodes[i].l_lo.w = __uint_as_float(left);
  nodes[i].l_hi.w = __uint_as_float(right);
  if (left & LEAF_BIT) leaf_parent[gamma] = i;
  else node_parent[gamma] = i;
  if (right & LEAF_BIT) leaf_parent[gamma + 1] = i;
  else node_parent[gamma + 1] = i;
  if (i == 0) node_parent[0] = 0xFFFFFFFFu;
}

__global__ void k_gather_leaves(const TriRec* __restrict__ tris, const uint32_t* __restrict__ perm, int n,
                                TriRec* stris) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k < n) stris[k] = tris[perm[k]];
}

__device__ __forceinline__ void store_child_box(BvhNode* node, bool left, float4 lo, float4 hi) {
  float* f = reinterpret_cast<float*>(node);
  int o = left ? 0 : 8;
  __stcg(f + o + 0, lo.x);
  __stcg(f + o + 1, lo.y);
  __stcg(f + o + 2, lo.z);
  __stcg(f + o + 4, hi.x);
  __stcg(f + o + 5, hi.y);
  __stcg(f + o + 6, hi.z);
}

__global__ void k_refit(const float4* __restrict__ boxes, const uint32_t* __restrict__ perm, int n, BvhNode* nodes,
                        const uint32_t* __restrict__ node_parent, const uint32_t* __restrict__ leaf_parent,
                        uint32_t* counters) {
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= n) return;
  uint32_t tri = perm[k];
  float4 lo = boxes[2 * tri], hi = boxes[2 * tri + 1];
  uint32_t child = LEAF_BIT | (uint32_t)k;
  uint32_t p = leaf_parent[k];
  // At most n - 1 levels; the bound keeps a malformed tree from looping.
  for (int guard = 0; guard < n; ++guard) {
    BvhNode* node = &nodes[p];
    bool left = __float_as_uint(__ldcg(&node->l_lo.w)) == child;
    store_child_box(node, left, lo, hi);
    __threadfence();
    if (atomicAdd(&counters[p], 1u) == 0) return;
    __threadfence();
    float4 a = __ldcg(&node->l_lo), b = __ldcg(&node->l_hi), c = __ldcg(&node->r_lo), d = __ldcg(&node->r_hi);
    lo = make_float4(fminf(a.x, c.x), fminf(a.y, c.y), fminf(a.z, c.z), 0.0f);
    hi = make_float4(fmaxf(b.x, d.x), fmaxf(b.y, d.y), fmaxf(b.z, d.z), 0.0f);
    uint32_t up = node_parent[p];
    if (up == 0xFFFFFFFFu) return;
    child = p;
    p = up;
  }
}

inline unsigned grid_for(uint64_t n, int threads = kThreads) { return (unsigned)((n + threads - 1) / threads); }

}  // namespace

int exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* d_total, cudaStream_t s) {
  if (n == 0) {
    if (d_total) M2S_CUDA(cudaMemsetAsync(d_total, 0, 4, s));
    return M2S_OK;
  }
  uint64_t tiles = (n + kScanTile - 1) / kScanTile;
  DevBuf<uint32_t> sums;
  int st = sums.alloc(tiles + 1, s);
  if (st) return st;
  // The last input is needed for the total if the scan runs in place.
  DevBuf<uint32_t> last;
  if (d_total) {
    if ((st = last.alloc(1, s))) return st;
    M2S_CUDA(cudaMemcpyAsync(last.p, in + n - 1, 4, cudaMemcpyDeviceToDevice, s));
  }
  k_scan_tiles<<<(unsigned)tiles, kThreads, 0, s>>>(in, out, n, sums.p);
  M2S_CUDA(cudaGetLastError());
  if (tiles > 1) {
    if ((st = exclusive_scan_u32(sums.p, sums.p, tiles, nullptr, s))) return st;
    k_add_tiles<<<(unsigned)tiles, kThreads, 0, s>>>(out, n, sums.p);
    M2S_CUDA(cudaGetLastError());
  }
  if (d_total) {
    k_copy_total<<<1, 1, 0, s>>>(out, n, last.p, d_total);
    M2S_CUDA(cudaGetLastError());
  }
  return M2S_OK;
}

int radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint64_t n, int key_bits, cudaStream_t s) {
  if (n <= 1) return M2S_OK;
  if (key_bits <= 0 || key_bits > 32 || n > 0xFFFFFFFFull) return M2S_ERR_INVALID_ARGUMENT;
  uint32_t nblocks = (uint32_t)((n + kSortTile - 1) / kSortTile);
  DevBuf<uint32_t> k2, v2, hist;
  int st;
  if ((st = k2.alloc(n, s)) || (st = v2.alloc(n, s)) || (st = hist.alloc((uint64_t)kDigits * nblocks, s))) return st;
  uint32_t *ka = keys, *va = vals, *kb = k2.p, *vb = v2.p;
  int passes = (key_bits + 7) / 8;
  for (int p = 0; p < passes; ++p) {
    int shift = 8 * p;
    k_hist<<<nblocks, kThreads, 0, s>>>(ka, n, shift, hist.p, nblocks);
    M2S_CUDA(cudaGetLastError());
    if ((st = exclusive_scan_u32(hist.p, hist.p, (uint64_t)kDigits * nblocks, nullptr, s))) return st;
    k_scatter<<<nblocks, kThreads, 0, s>>>(ka, va, kb, vb, n, shift, hist.p, nblocks);
    M2S_CUDA(cudaGetLastError());
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  if (ka != keys) {
    M2S_CUDA(cudaMemcpyAsync(keys, ka, n * 4, cudaMemcpyDeviceToDevice, s));
    M2S_CUDA(cudaMemcpyAsync(vals, va, n * 4, cudaMemcpyDeviceToDevice, s));
  }
  return M2S_OK;
}

int build_device_mesh(const MeshInput& in, DeviceMesh* out, uint32_t* d_status, cudaStream_t s, bool with_tree) {
  if (in.n_tris > 0x7FFFFFFFull) return M2S_ERR_INVALID_ARGUMENT;
  const uint32_t T = (uint32_t)in.n_tris;
  out->n_tris = T;
  out->root = T == 1 ? LEAF_BIT : 0;
  int st;
  if ((st = out->tris.alloc(T, s))) return st;
  if (T == 0) return M2S_OK;
  DevBuf<float4> boxes;
  DevBuf<uint32_t> keys, perm, bounds;
  if ((st = boxes.alloc(2ull * T, s)) || (st = keys.alloc(T, s)) || (st = perm.alloc(T, s)) ||
      (st = bounds.alloc(6, s)))
    return st;
  k_setup<<<grid_for(T), kThreads, 0, s>>>(in, out->tris.p, boxes.p, d_status);
  M2S_CUDA(cudaGetLastError());
  if (!with_tree) return M2S_OK;
  k_bounds_init<<<1, 32, 0, s>>>(bounds.p);
  k_bounds<<<std::min(grid_for(T), 1184u), kThreads, 0, s>>>(boxes.p, T, bounds.p);
  k_morton<<<grid_for(T), kThreads, 0, s>>>(boxes.p, T, bounds.p, keys.p, perm.p);
  M2S_CUDA(cudaGetLastError());
  if ((st = radix_sort_pairs(keys.p, perm.p, T, 30, s))) return st;
  if ((st = out->stris.alloc(T, s))) return st;
  k_gather_leaves<<<grid_for(T), kThreads, 0, s>>>(out->tris.p, perm.p, (int)T, out->stris.p);
  M2S_CUDA(cudaGetLastError());
  if (T < 2) return M2S_OK;
  DevBuf<uint32_t> node_parent, leaf_parent, counters;
  if ((st = out->nodes.alloc(T - 1, s)) || (st = node_parent.alloc(T - 1, s)) || (st = leaf_parent.alloc(T, s)) ||
      (st = counters.alloc(T - 1, s)))
    return st;
  M2S_CUDA(cudaMemsetAsync(counters.p, 0, (T - 1) * sizeof(uint32_t), s));
  k_karras<<<grid_for(T - 1), kThreads, 0, s>>>(keys.p, (int)T, out->nodes.p, node_parent.p, leaf_parent.p);
  M2S_CUDA(cudaGetLastError());
  k_refit<<<grid_for(T), kThreads, 0, s>>>(boxes.p, perm.p, (int)T, out->nodes.p, node_parent.p, leaf_parent.p,
                                           counters.p);
  M2S_CUDA(cudaGetLastError());
  return M2S_OK;
}

}  // namespace m2s
