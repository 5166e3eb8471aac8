// m2s_generate_sdf_none_noalloc: generate_sdf with AccelerationMethod::None
// for callers that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc at query time: a real-time render loop
// (cudaMalloc may synchronise the whole device and stall every other stream
// for an unbounded time), or an application that has already handed its
// entire device-memory budget to its own pool, leaving nothing for a library
// to allocate.  This entry point therefore takes every input and output as a
// caller-owned device pointer and keeps its only scratch — the triangle
// records of the mesh and a status word — in a file-scope __device__ array of
// fixed size, allocated by the CUDA module when the library is loaded.
//
// Limits and behaviour:
//  * at most kMaxTriangles triangles (larger meshes are rejected with
//    M2S_ERR_INVALID_ARGUMENT and a message naming the limit);
//  * the array exists once per device that loads the library and stays
//    allocated until the process exits;
//  * every call on a device reuses the same array, so calls whose work
//    overlaps on the GPU (different streams or threads) race and must be
//    serialised by the caller;
//  * the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress) with that device current; make that first call
//    before any stream capture;
//  * the call returns after the result is in d_out (it waits for its stream
//    to read the status word back into a host stack variable).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>

#include "m2s_internal.cuh"

namespace m2s {
namespace {

constexpr uint64_t kMaxTriangles = 1ull << 18;  // 262,144 triangles
constexpr size_t kRecordBytes = kMaxTriangles * sizeof(TriRec);
constexpr size_t kScratchBytes = kRecordBytes + 256;  // records, then the status word

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_mu;
constexpr int kMaxDevices = 64;  // devices whose scratch address is remembered
void* g_scratch_ptr[kMaxDevices];

// Device address of g_scratch on the current device (looked up once per device).
int scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) {
    set_error("m2s_generate_sdf_none_noalloc serves devices 0..63; the current device is " + std::to_string(dev));
    return M2S_ERR_INVALID_ARGUMENT;
  }
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(g_scratch)");
    g_scratch_ptr[dev] = p;
  }
  *out = g_scratch_ptr[dev];
  return M2S_OK;
}

__device__ __forceinline__ uint32_t index_at(const void* idx, int bits, uint64_t k) {
  if (bits == 16) return ((const uint16_t*)idx)[k];
  if (bits == 32) return ((const uint32_t*)idx)[k];
  return (uint32_t)k;
}

// Triangle records of Topology::get_triangles (lib.rs:193-215); out-of-range
// indices raise M2S_ERR_INDEX_RANGE.
__global__ void k_records(const float* __restrict__ v, uint64_t nv, const void* __restrict__ idx, int bits, int topo,
                          uint64_t n_tris, TriRec* __restrict__ out, uint32_t* status) {
  uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n_tris) return;
  uint64_t base = topo == M2S_TOPOLOGY_TRIANGLE_LIST ? 3 * t : t;
  uint64_t i[3];
  for (int k = 0; k < 3; ++k) i[k] = bits ? index_at(idx, bits, base + k) : base + k;
  if (i[0] >= nv || i[1] >= nv || i[2] >= nv) {
    atomicOr(status, bit(M2S_ERR_INDEX_RANGE));
    i[0] = i[1] = i[2] = 0;
  }
  float a[3], b[3], c[3];
  for (int d = 0; d < 3; ++d) {
    a[d] = v[3 * i[0] + d];
    b[d] = v[3 * i[1] + d];
    c[d] = v[3 * i[2] + d];
  }
  TriRec r;
  r.a = make_float4(a[0], a[1], a[2], __int_as_float(degenerate_kind(a[0], a[1], a[2], b[0], b[1], b[2], c[0], c[1], c[2])));
  r.b = make_float4(b[0], b[1], b[2], __uint_as_float((uint32_t)t));
  r.c = make_float4(c[0], c[1], c[2], 0.0f);
  out[t] = r;
}

// lib.rs:374-376: every query coordinate must be finite.
__global__ void k_finite(const float* __restrict__ q, uint64_t n, uint32_t* status) {
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
    if (!isfinite(q[i])) atomicOr(status, bit(M2S_ERR_NONFINITE_QUERY));
}

}  // namespace
}  // namespace m2s

using namespace m2s;

extern "C" int m2s_generate_sdf_none_noalloc(const float* d_vertices, uint64_t n_vertices, const void* d_indices,
                                             uint64_t n_indices, int index_bits, int topology,
                                             const float* d_query_points, uint64_t n_queries, int sign, float* d_out,
                                             void* stream) {
  if (index_bits != M2S_INDEX_NONE && index_bits != M2S_INDEX_U16 && index_bits != M2S_INDEX_U32)
    return M2S_ERR_INVALID_ARGUMENT;
  if (topology != M2S_TOPOLOGY_TRIANGLE_LIST && topology != M2S_TOPOLOGY_TRIANGLE_STRIP) return M2S_ERR_INVALID_ARGUMENT;
  if (sign != M2S_SIGN_RAYCAST && sign != M2S_SIGN_NORMAL) return M2S_ERR_INVALID_ARGUMENT;
  const uint64_t n = index_bits == M2S_INDEX_NONE ? n_vertices : n_indices;
  uint64_t T;
  if (topology == M2S_TOPOLOGY_TRIANGLE_LIST) {
    if (n % 3 != 0) return M2S_ERR_INDEX_COUNT;  // lib.rs:203, lib.rs:207
    T = n / 3;
  } else {
    T = n >= 3 ? n - 2 : 0;
  }
  if (T > kMaxTriangles) {
    set_error("m2s_generate_sdf_none_noalloc: the mesh has more than 262144 triangles, the size of its fixed scratch");
    return M2S_ERR_INVALID_ARGUMENT;
  }
  if ((T && (!d_vertices || (index_bits != M2S_INDEX_NONE && !d_indices))) || (n_queries && (!d_query_points || !d_out)))
    return M2S_ERR_INVALID_ARGUMENT;
  if (T > 0 && n_vertices == 0) return M2S_ERR_INDEX_RANGE;
  if (n_queries == 0) return M2S_OK;
  int st;
  void* scratch = nullptr;
  if ((st = scratch_address(&scratch))) return st;
  cudaStream_t s = (cudaStream_t)stream;
  TriRec* recs = reinterpret_cast<TriRec*>(scratch);
  uint32_t* d_status = reinterpret_cast<uint32_t*>(static_cast<unsigned char*>(scratch) + kRecordBytes);
  M2S_CUDA(cudaMemsetAsync(d_status, 0, sizeof(uint32_t), s));  // the array keeps the last call's contents
  if (T) {
    k_records<<<(unsigned)((T + 255) / 256), 256, 0, s>>>(d_vertices, n_vertices, d_indices, index_bits, topology, T,
                                                           recs, d_status);
    M2S_CUDA(cudaGetLastError());
  }
  k_finite<<<(unsigned)std::min<uint64_t>((3 * n_queries + 255) / 256, 148u * 16u), 256, 0, s>>>(d_query_points,
                                                                                               3 * n_queries, d_status);
  M2S_CUDA(cudaGetLastError());
  MeshView view{recs, nullptr, nullptr, (uint32_t)T, 0};
  if ((st = brute_force_sdf(view, sign, d_query_points, n_queries, d_out, d_status, s, /*allow_alloc=*/false)))
    return st;
  uint32_t bits = 0;  // host stack: the copy from pageable memory completes before it returns
  M2S_CUDA(cudaMemcpyAsync(&bits, d_status, sizeof(bits), cudaMemcpyDeviceToHost, s));
  M2S_CUDA(cudaStreamSynchronize(s));
  for (int code = 1; code < 32; ++code)
    if (bits & (1u << code)) return code;
  return M2S_OK;
}
