// Internal declarations shared by the mesh_to_sdf_b200 CUDA sources.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/m2s.h"
#include "m2s_geo.cuh"

namespace m2s {

// Kernels OR (1u << status) into a device word; the host maps the lowest set
// bit back to a status code.
__host__ __device__ constexpr uint32_t bit(int status) { return 1u << status; }

// One triangle, 48 bytes, read with three 128-bit loads.
//   a.w : degenerate kind (TRI_*), as int bits
//   b.w : triangle index in the crate's triangle order, as uint bits
//   c.w : unused (0)
struct __align__(16) TriRec {
  float4 a, b, c;
};

// Internal LBVH node, 64 bytes: both child boxes live in the parent so one
// node fetch tests both children.  l_lo.w / l_hi.w hold the left / right
// child references (uint bits); LEAF_BIT marks a leaf (index into the
// LBVH-ordered triangle array).
struct __align__(16) BvhNode {
  float4 l_lo, l_hi, r_lo, r_hi;
};
constexpr uint32_t LEAF_BIT = 0x80000000u;

// Device view of a resident mesh.
struct MeshView {
  const TriRec* tris;    // crate triangle order
  const TriRec* stris;   // LBVH leaf order
  const BvhNode* nodes;  // n_tris - 1 internal nodes (node 0 is the root)
  uint32_t n_tris;
  uint32_t root;  // 0, or LEAF_BIT | 0 for a single triangle
};

// Thread-local error detail for m2s_last_error().
void set_error(const std::string& msg);
int cuda_fail(cudaError_t e, const char* what);

#define M2S_CUDA(call)                                    \
  do {                                                    \
    cudaError_t e_ = (call);                              \
    if (e_ != cudaSuccess) return ::m2s::cuda_fail(e_, #call); \
  } while (0)

// Stream-ordered device allocation from the library's memory pool.
int dev_alloc(void** p, size_t bytes, cudaStream_t s);
void dev_free(void* p, cudaStream_t s);

template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  cudaStream_t s = nullptr;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : p(o.p), n(o.n), s(o.s) { o.p = nullptr; }
  DevBuf& operator=(DevBuf&& o) noexcept {
    release();
    p = o.p, n = o.n, s = o.s;
    o.p = nullptr;
    return *this;
  }
  int alloc(size_t count, cudaStream_t st) {
    release();
    s = st;
    n = count;
    if (count == 0) return M2S_OK;
    return dev_alloc((void**)&p, count * sizeof(T), st);
  }
  void release() {
    if (p) dev_free(p, s);
    p = nullptr;
    n = 0;
  }
  ~DevBuf() { release(); }
};

// ---- LBVH build (m2s_lbvh.cu) ----------------------------------------------

struct MeshInput {
  const float* d_vertices;  // device, 3 * n_vertices
  uint64_t n_vertices;
  const void* d_indices;  // device or NULL
  int index_bits;         // 0 / 16 / 32
  int topology;           // 0 list / 1 strip
  uint64_t n_tris;
};

struct DeviceMesh {
  DevBuf<TriRec> tris, stris;
  DevBuf<BvhNode> nodes;
  uint32_t n_tris = 0;
  uint32_t root = 0;
  MeshView view() const { return {tris.p, stris.p, nodes.p, n_tris, root}; }
};

// Builds the triangle records and the LBVH.  d_status receives status bits.
// with_tree = false builds the triangle records only (grid path, brute force).
int build_device_mesh(const MeshInput& in, DeviceMesh* out, uint32_t* d_status, cudaStream_t s,
                      bool with_tree = true);

// Stable LSD radix sort of (key, value) pairs over the low key_bits bits.
int radix_sort_pairs(uint32_t* keys, uint32_t* vals, uint64_t n, int key_bits, cudaStream_t s);

// Exclusive scan of n uint32 (in place allowed); returns the total via *d_total if non-null.
int exclusive_scan_u32(const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* d_total, cudaStream_t s);

// ---- point queries (m2s_query.cu) -------------------------------------------

int query_points(const MeshView& m, int accel, int sign, const float* d_q, uint64_t nq, float* d_out,
                 float* d_vec, uint8_t* d_inside, uint32_t* d_status, cudaStream_t s);

// Node visits a query may spend in the one-thread-per-query pass before it is
// continued one warp per query (0 disables the second pass).
extern uint32_t g_query_budget;

// allow_alloc = false keeps the brute force in one pass with no scratch buffer.
int brute_force_sdf(const MeshView& m, int sign, const float* d_q, uint64_t nq, float* d_out,
                    uint32_t* d_status, cudaStream_t s, bool allow_alloc = true);

// ---- grid (m2s_grid.cu) ------------------------------------------------------

struct GridDesc {
  float first[3];
  float size[3];
  uint64_t n[3];
  uint64_t cells() const { return n[0] * n[1] * n[2]; }
};

// stats: [seed updates, rounds, states relaxed, neighbour evaluations, ray hits,
// overflow recoveries, kernel launches, relax rounds launched].  phase_ms (may be
// NULL) receives device time of [seeding, propagation, rays, finalize].
constexpr int kGridStats = 8;
int grid_sdf(const MeshView& m, const GridDesc& g, int sign, float* d_out, uint32_t* d_status, cudaStream_t s,
             uint64_t stats[kGridStats], float phase_ms[4]);

}  // namespace m2s
