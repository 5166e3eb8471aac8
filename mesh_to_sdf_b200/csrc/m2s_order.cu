// Distance-ordered cell list: the voxel viewer's index buffer
// (mesh_to_sdf_client/src/sdf.rs:63-71) computed on the device.
//
// The client sorts 0..n by `data[i].total_cmp(&data[j])` with rayon's stable
// `par_sort_by`, then takes `minmax` of the data as its iso limits.  Here each
// distance becomes a 32-bit key that orders like total_cmp (negative floats:
// all bits flipped; others: sign bit set), and the (key, index) pairs go
// through the library's stable LSD radix sort starting from indices in order
// — equal distances keep index order, as in the stable sort.
#include <cuda_runtime.h>

#include <algorithm>
#include <cfloat>

#include "m2s_internal.cuh"

namespace m2s {
namespace {

__device__ __forceinline__ uint32_t total_order_key(float f) {
  const uint32_t b = __float_as_uint(f);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

__global__ void k_order_keys(const float* __restrict__ d, uint64_t n, uint32_t* __restrict__ keys,
                             uint32_t* __restrict__ idx) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    keys[i] = total_order_key(d[i]);
    idx[i] = (uint32_t)i;
  }
}

// min / max of the non-NaN values (the order keys of the extremes).
__global__ void k_minmax(const float* __restrict__ d, uint64_t n, unsigned int* mm) {
  float lo = FLT_MAX, hi = -FLT_MAX;
  bool any = false;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
    const float v = d[i];
    if (isnan(v)) continue;
    lo = fminf(lo, v);
    hi = fmaxf(hi, v);
    any = true;
  }
  unsigned int klo = any ? total_order_key(lo) : 0xFFFFFFFFu, khi = any ? total_order_key(hi) : 0u;
  for (int o = 16; o; o >>= 1) {
    klo = min(klo, __shfl_xor_sync(0xFFFFFFFFu, klo, o));
    khi = max(khi, __shfl_xor_sync(0xFFFFFFFFu, khi, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&mm[0], klo);
    atomicMax(&mm[1], khi);
  }
}

__global__ void k_minmax_out(const unsigned int* mm, float* out) {
  for (int k = 0; k < 2; ++k) {
    const uint32_t key = mm[k];
    const uint32_t b = (key & 0x80000000u) ? (key & 0x7FFFFFFFu) : ~key;  // inverse of total_order_key
    out[k] = __uint_as_float(b);
  }
}

}  // namespace

int sort_cells_by_distance(const float* d_sdf, uint64_t n, uint32_t* d_order, float* d_minmax, cudaStream_t s) {
  if (n == 0) return M2S_OK;
  if (n > 0xFFFFFFFFull) return M2S_ERR_INVALID_ARGUMENT;
  DevBuf<uint32_t> keys;
  int st;
  if ((st = keys.alloc(n, s))) return st;
  const unsigned blocks = (unsigned)std::min<uint64_t>((n + 255) / 256, 148ull * 16);
  k_order_keys<<<blocks, 256, 0, s>>>(d_sdf, n, keys.p, d_order);
  M2S_CUDA(cudaGetLastError());
  if ((st = radix_sort_pairs(keys.p, d_order, n, 32, s))) return st;
  if (d_minmax) {
    DevBuf<unsigned int> mm;
    if ((st = mm.alloc(2, s))) return st;
    const unsigned int init[2] = {0xFFFFFFFFu, 0u};
    M2S_CUDA(cudaMemcpyAsync(mm.p, init, sizeof(init), cudaMemcpyHostToDevice, s));
    k_minmax<<<blocks, 256, 0, s>>>(d_sdf, n, mm.p);
    k_minmax_out<<<1, 1, 0, s>>>(mm.p, d_minmax);
    M2S_CUDA(cudaGetLastError());
  }
  return M2S_OK;
}

}  // namespace m2s

using namespace m2s;

extern "C" {

int m2s_sort_cells_by_distance_device(const float* d_sdf, uint64_t n, uint32_t* d_order, float* d_minmax,
                                      void* stream) {
  if (n && (!d_sdf || !d_order)) return M2S_ERR_INVALID_ARGUMENT;
  int st;
  if ((st = require_device())) return st;
  return sort_cells_by_distance(d_sdf, n, d_order, d_minmax, (cudaStream_t)stream);
}

int m2s_sort_cells_by_distance(const float* sdf, uint64_t n, uint32_t* order, float minmax[2], void* stream) {
  if (n && (!sdf || !order)) return M2S_ERR_INVALID_ARGUMENT;
  if (n > 0xFFFFFFFFull) return M2S_ERR_INVALID_ARGUMENT;
  int st;
  if ((st = require_device())) return st;
  if (n == 0) return M2S_OK;
  cudaStream_t s = (cudaStream_t)stream;
  DevBuf<float> d, mm;
  DevBuf<uint32_t> o;
  if ((st = d.alloc(n, s)) || (st = o.alloc(n, s)) || (st = mm.alloc(2, s))) return st;
  M2S_CUDA(cudaMemcpyAsync(d.p, sdf, 4 * n, cudaMemcpyHostToDevice, s));
  if ((st = sort_cells_by_distance(d.p, n, o.p, minmax ? mm.p : nullptr, s))) return st;
  M2S_CUDA(cudaMemcpyAsync(order, o.p, 4 * n, cudaMemcpyDeviceToHost, s));
  if (minmax) M2S_CUDA(cudaMemcpyAsync(minmax, mm.p, 8, cudaMemcpyDeviceToHost, s));
  M2S_CUDA(cudaStreamSynchronize(s));
  return M2S_OK;
}

}  // extern "C"
