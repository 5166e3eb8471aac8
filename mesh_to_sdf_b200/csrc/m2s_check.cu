// check_mesh_triangle_list (generate/mesh_check.rs:24-81) on the device:
// O(E log E) sorts instead of the crate's O(E^2) edge loop, with the crate's
// verdict and the crate's first reported failure.
//
// The crate checks, in this order:
//  1. the index count is a multiple of 3;
//  2. no vertex repeats an earlier one, comparing the `{:?}` text of its
//     coordinates — the same as comparing f32 bit patterns with every NaN
//     equal — and reports the first repeat in vertex order;
//  3. no face repeats an earlier one as an ordered index triple, reporting the
//     first repeat;
//  4. the directed edges (a,b), (b,c), (c,a) of every face, in order, are
//     consumed from the end: the popped edge fails if another copy of it is
//     left ("duplicate edge") or if no reverse edge is left ("not
//     waterproof"); otherwise every copy of the reverse is removed.
// For step 4 note that, per unordered pair {u, v}, the first of its edges to
// be popped is the one at the pair's highest position; it is the only check
// the pair gets (a success removes the other direction, the popped
// direction has a single copy).  That check fails exactly when the popped
// direction occurs more than once, or the other direction never occurs (a
// self-loop u == u never has a reverse left).  The crate stops at the failing
// pair whose check position is highest.
//
// Device steps: repeats of steps 2 and 3 by a stable LSD sort of indices on
// the three coordinates (three radix sorts), then a scan of neighbours in
// sorted order; step 4 by a stable sort of edge positions on (min, max) of
// their endpoints and one pass over the resulting runs.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "m2s_internal.cuh"

namespace m2s {
namespace {

constexpr unsigned kThreads = 256;

unsigned grid_for(uint64_t n) { return (unsigned)std::max<uint64_t>(1, std::min<uint64_t>((n + kThreads - 1) / kThreads, 148ull * 16)); }

__device__ __forceinline__ uint32_t vertex_key(float f) { return isnan(f) ? 0x7FC00000u : __float_as_uint(f); }

// component k of element i: vertices (canonical f32 bits) or face indices
template <bool VERTS>
__device__ __forceinline__ uint32_t comp(const void* base, uint64_t i, int k) {
  if (VERTS) return vertex_key(((const float*)base)[3 * i + k]);
  return ((const uint32_t*)base)[3 * i + k];
}

__global__ void k_iota(uint32_t* v, uint64_t n) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    v[i] = (uint32_t)i;
}

template <bool VERTS>
__global__ void k_gather_comp(const void* base, const uint32_t* __restrict__ idx, uint64_t n, int k,
                              uint32_t* __restrict__ keys) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    keys[i] = comp<VERTS>(base, idx[i], k);
}

// In triple order with ties in index order, a repeat's earliest occurrence is
// the second element of its run: the smallest such index is the first repeat.
template <bool VERTS>
__global__ void k_first_repeat(const void* base, const uint32_t* __restrict__ idx, uint64_t n,
                               unsigned long long* first) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x + 1; i < n;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t a = idx[i - 1], b = idx[i];
    if (comp<VERTS>(base, a, 0) == comp<VERTS>(base, b, 0) && comp<VERTS>(base, a, 1) == comp<VERTS>(base, b, 1) &&
        comp<VERTS>(base, a, 2) == comp<VERTS>(base, b, 2))
      atomicMin(first, (unsigned long long)b);
  }
}

// Directed edge at position p = 3 f + k: (t[k], t[(k + 1) % 3]).
__device__ __forceinline__ void edge_at(const uint32_t* faces, uint32_t p, uint32_t* from, uint32_t* to) {
  const uint32_t f = p / 3, k = p - 3 * f;
  *from = faces[3 * f + k];
  *to = faces[3 * f + (k == 2 ? 0 : k + 1)];
}

__global__ void k_edge_keys(const uint32_t* __restrict__ faces, const uint32_t* __restrict__ pos, uint64_t n, int hi,
                            uint32_t* __restrict__ keys) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t a, b;
    edge_at(faces, pos[i], &a, &b);
    keys[i] = hi ? max(a, b) : min(a, b);
  }
}

// One pass over the runs of equal {min, max}: the thread at a run's start
// walks it.  Failing pairs compete for the highest check position.
__global__ void k_edge_runs(const uint32_t* __restrict__ faces, const uint32_t* __restrict__ pos, uint64_t n,
                            unsigned long long* worst, uint32_t* run_kind, uint32_t* run_from, uint32_t* run_to) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    uint32_t a, b;
    edge_at(faces, pos[i], &a, &b);
    const uint32_t lo = min(a, b), hi = max(a, b);
    if (i > 0) {
      uint32_t pa, pb;
      edge_at(faces, pos[i - 1], &pa, &pb);
      if (min(pa, pb) == lo && max(pa, pb) == hi) continue;  // not a run start
    }
    uint32_t n_up = 0, n_down = 0;  // lo -> hi, hi -> lo
    uint32_t last_up = 0, last_down = 0;
    bool any_up = false, any_down = false;
    for (uint64_t j = i; j < n; ++j) {
      uint32_t c, d;
      const uint32_t p = pos[j];
      edge_at(faces, p, &c, &d);
      if (min(c, d) != lo || max(c, d) != hi) break;
      if (c == lo) {  // includes self-loops
        ++n_up;
        last_up = any_up ? max(last_up, p) : p;
        any_up = true;
      } else {
        ++n_down;
        last_down = any_down ? max(last_down, p) : p;
        any_down = true;
      }
    }
    uint32_t kind = 0, from, to, at;
    if (lo == hi) {
      at = last_up;
      from = to = lo;
      kind = n_up >= 2 ? 4 : 5;
    } else {
      const bool up_first = any_up && (!any_down || last_up > last_down);
      const uint32_t n_first = up_first ? n_up : n_down, n_other = up_first ? n_down : n_up;
      at = up_first ? last_up : last_down;
      from = up_first ? lo : hi;
      to = up_first ? hi : lo;
      kind = n_first >= 2 ? 4 : (n_other == 0 ? 5 : 0);
    }
    if (kind) {
      run_kind[i] = kind;
      run_from[i] = from;
      run_to[i] = to;
      atomicMax(worst, ((unsigned long long)at << 32) | (unsigned long long)i);
    }
  }
}

// Stable sort of idx[0..n) by the triple (comp 0, comp 1, comp 2).
template <bool VERTS>
int sort_triples(const void* base, uint64_t n, uint32_t* idx, uint32_t* keys, cudaStream_t s) {
  k_iota<<<grid_for(n), kThreads, 0, s>>>(idx, n);
  for (int k = 2; k >= 0; --k) {
    k_gather_comp<VERTS><<<grid_for(n), kThreads, 0, s>>>(base, idx, n, k, keys);
    M2S_CUDA(cudaGetLastError());
    int st = radix_sort_pairs(keys, idx, n, 32, s);
    if (st) return st;
  }
  return M2S_OK;
}

template <bool VERTS>
int first_repeat(const void* base, uint64_t n, cudaStream_t s, uint64_t* out) {
  *out = UINT64_MAX;
  if (n < 2) return M2S_OK;
  DevBuf<uint32_t> idx, keys;
  DevBuf<unsigned long long> first;
  int st;
  if ((st = idx.alloc(n, s)) || (st = keys.alloc(n, s)) || (st = first.alloc(1, s))) return st;
  if ((st = sort_triples<VERTS>(base, n, idx.p, keys.p, s))) return st;
  M2S_CUDA(cudaMemsetAsync(first.p, 0xFF, 8, s));
  k_first_repeat<VERTS><<<grid_for(n), kThreads, 0, s>>>(base, idx.p, n, first.p);
  M2S_CUDA(cudaGetLastError());
  unsigned long long h = 0;
  M2S_CUDA(cudaMemcpyAsync(&h, first.p, 8, cudaMemcpyDeviceToHost, s));
  M2S_CUDA(cudaStreamSynchronize(s));
  *out = h;
  return M2S_OK;
}

}  // namespace

int check_mesh_triangle_list(const float* d_vertices, uint64_t nv, const uint32_t* d_faces, uint64_t n_idx, int* kind,
                             uint64_t detail[2], cudaStream_t s) {
  *kind = 0;
  detail[0] = detail[1] = 0;
  if (n_idx % 3 != 0) {
    *kind = 1;
    return M2S_OK;
  }
  if (nv > 0xFFFFFFFFull || n_idx > 0xFFFFFFFFull) return M2S_ERR_INVALID_ARGUMENT;  // 32-bit sort values
  int st;
  uint64_t rep;
  if ((st = first_repeat<true>(d_vertices, nv, s, &rep))) return st;
  if (rep != UINT64_MAX) {
    *kind = 2;
    detail[0] = rep;
    return M2S_OK;
  }
  const uint64_t F = n_idx / 3, E = n_idx;
  if ((st = first_repeat<false>(d_faces, F, s, &rep))) return st;
  if (rep != UINT64_MAX) {
    *kind = 3;
    detail[0] = rep;
    return M2S_OK;
  }
  if (E == 0) return M2S_OK;
  DevBuf<uint32_t> pos, keys, rk, rf, rt;
  DevBuf<unsigned long long> worst;
  if ((st = pos.alloc(E, s)) || (st = keys.alloc(E, s)) || (st = rk.alloc(E, s)) || (st = rf.alloc(E, s)) ||
      (st = rt.alloc(E, s)) || (st = worst.alloc(1, s)))
    return st;
  k_iota<<<grid_for(E), kThreads, 0, s>>>(pos.p, E);
  for (int hi = 1; hi >= 0; --hi) {  // by max, then (stably) by min
    k_edge_keys<<<grid_for(E), kThreads, 0, s>>>(d_faces, pos.p, E, hi, keys.p);
    M2S_CUDA(cudaGetLastError());
    if ((st = radix_sort_pairs(keys.p, pos.p, E, 32, s))) return st;
  }
  M2S_CUDA(cudaMemsetAsync(worst.p, 0, 8, s));
  M2S_CUDA(cudaMemsetAsync(rk.p, 0, 4 * E, s));
  k_edge_runs<<<grid_for(E), kThreads, 0, s>>>(d_faces, pos.p, E, worst.p, rk.p, rf.p, rt.p);
  M2S_CUDA(cudaGetLastError());
  unsigned long long w = 0;
  M2S_CUDA(cudaMemcpyAsync(&w, worst.p, 8, cudaMemcpyDeviceToHost, s));
  M2S_CUDA(cudaStreamSynchronize(s));
  const uint32_t run = (uint32_t)w;
  uint32_t k = 0, from = 0, to = 0;
  M2S_CUDA(cudaMemcpyAsync(&k, rk.p + run, 4, cudaMemcpyDeviceToHost, s));
  M2S_CUDA(cudaMemcpyAsync(&from, rf.p + run, 4, cudaMemcpyDeviceToHost, s));
  M2S_CUDA(cudaMemcpyAsync(&to, rt.p + run, 4, cudaMemcpyDeviceToHost, s));
  M2S_CUDA(cudaStreamSynchronize(s));
  if (k) {
    *kind = (int)k;
    detail[0] = from;
    detail[1] = to;
  }
  return M2S_OK;
}

}  // namespace m2s

using namespace m2s;

extern "C" int m2s_check_mesh_triangle_list(const float* vertices, uint64_t n_vertices, const uint32_t* faces,
                                            uint64_t n_face_indices, int* result, uint64_t detail[2], void* stream) {
  if (!result || !detail || (n_vertices && !vertices) || (n_face_indices && !faces)) return M2S_ERR_INVALID_ARGUMENT;
  *result = 0;
  detail[0] = detail[1] = 0;
  if (n_face_indices % 3 != 0) {  // mesh_check.rs:29-31, before anything touches the device
    *result = 1;
    return M2S_OK;
  }
  int st;
  if ((st = require_device())) return st;
  cudaStream_t s = (cudaStream_t)stream;
  DevBuf<float> v;
  DevBuf<uint32_t> f;
  if ((st = v.alloc(3 * n_vertices, s)) || (st = f.alloc(n_face_indices, s))) return st;
  if (n_vertices) M2S_CUDA(cudaMemcpyAsync(v.p, vertices, 12 * n_vertices, cudaMemcpyHostToDevice, s));
  if (n_face_indices) M2S_CUDA(cudaMemcpyAsync(f.p, faces, 4 * n_face_indices, cudaMemcpyHostToDevice, s));
  return check_mesh_triangle_list(v.p, n_vertices, f.p, n_face_indices, result, detail, s);
}
