// C ABI of mesh_to_sdf_b200 (declared in include/m2s.h).
//
// Host-pointer entry points mirror the Rust crate's public functions: they
// validate like the crate (returning a status where it panics), upload the
// inputs to HBM, run the device path and copy the result back.  There is no
// CPU fallback: without an sm_100 device every compute call fails with
// M2S_ERR_NO_DEVICE.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "m2s_internal.cuh"

namespace m2s {
namespace {

thread_local std::string t_last_error;
thread_local uint64_t t_grid_stats[kGridStats];
thread_local float t_grid_phase_ms[4];
thread_local bool t_profile = false;
thread_local uint64_t t_query_stats[12];
thread_local std::vector<uint32_t> t_round_log;

std::mutex g_pool_mu;
cudaMemPool_t g_pools[64];
bool g_pool_ready[64];

int current_pool(cudaMemPool_t* out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= 64) return M2S_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (!g_pool_ready[dev]) {
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    e = cudaMemPoolCreate(&g_pools[dev], &props);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemPoolCreate");
    // Keep freed blocks cached in the pool between calls.
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(g_pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
    // A block freed on one stream is not handed to another stream before the
    // free has run: otherwise the pool makes the new stream wait for the old
    // one's queued work, and independent callers (a point query and a grid
    // job on their own streams) wait for each other.
    int no = 0;
    cudaMemPoolSetAttribute(g_pools[dev], cudaMemPoolReuseAllowInternalDependencies, &no);
    g_pool_ready[dev] = true;
  }
  *out = g_pools[dev];
  return M2S_OK;
}

// Triangle count of a topology (lib.rs:193-215); M2S_ERR_INDEX_COUNT where the
// crate asserts len % 3 == 0.
int triangle_count(uint64_t nv, const void* idx, uint64_t ni, int bits, int topo, uint64_t* T) {
  if (bits != M2S_INDEX_NONE && bits != M2S_INDEX_U16 && bits != M2S_INDEX_U32) return M2S_ERR_INVALID_ARGUMENT;
  if (topo != M2S_TOPOLOGY_TRIANGLE_LIST && topo != M2S_TOPOLOGY_TRIANGLE_STRIP) return M2S_ERR_INVALID_ARGUMENT;
  if (bits != M2S_INDEX_NONE && ni > 0 && !idx) return M2S_ERR_INVALID_ARGUMENT;
  uint64_t n = bits == M2S_INDEX_NONE ? nv : ni;
  if (topo == M2S_TOPOLOGY_TRIANGLE_LIST) {
    if (n % 3 != 0) return M2S_ERR_INDEX_COUNT;
    *T = n / 3;
  } else {
    *T = n >= 3 ? n - 2 : 0;
  }
  if (*T > 0 && nv == 0) return M2S_ERR_INDEX_RANGE;  // every index is out of range
  if (*T > 0x7FFFFFFFull) return M2S_ERR_INVALID_ARGUMENT;
  return M2S_OK;
}

bool all_finite(const float* q, uint64_t n) {
  for (uint64_t i = 0; i < 3 * n; ++i)
    if (!std::isfinite(q[i])) return false;
  return true;
}

// Device copies of a host mesh, kept alive for the duration of a call.
struct Upload {
  DevBuf<float> v;
  DevBuf<uint8_t> idx;
};

int upload_mesh(const float* vertices, uint64_t nv, const void* indices, uint64_t ni, int bits, Upload* up,
                cudaStream_t s) {
  int st;
  if (nv && !vertices) return M2S_ERR_INVALID_ARGUMENT;
  if ((st = up->v.alloc(3 * nv, s))) return st;
  if (nv) M2S_CUDA(cudaMemcpyAsync(up->v.p, vertices, 12 * nv, cudaMemcpyHostToDevice, s));
  if (bits != M2S_INDEX_NONE && ni) {
    size_t bytes = ni * (bits / 8);
    if ((st = up->idx.alloc(bytes, s))) return st;
    M2S_CUDA(cudaMemcpyAsync(up->idx.p, indices, bytes, cudaMemcpyHostToDevice, s));
  }
  return M2S_OK;
}

// A pinned status word per host thread, allocated once: freeing pinned memory
// waits for the whole device, which would stall a caller's other streams.
struct PinnedWord {
  uint32_t* p = nullptr;
  ~PinnedWord() {
    if (p) cudaFreeHost(p);
  }
};

struct StatusWord {
  DevBuf<uint32_t> d;
  uint32_t* h = nullptr;
  int init(cudaStream_t s) {
    thread_local PinnedWord pw;
    if (!pw.p) M2S_CUDA(cudaMallocHost(&pw.p, 4));
    h = pw.p;
    int st = d.alloc(1, s);
    if (st) return st;
    M2S_CUDA(cudaMemsetAsync(d.p, 0, 4, s));
    *h = 0;
    return M2S_OK;
  }
  // Synchronises the stream and returns the status the kernels raised.
  int read(cudaStream_t s) {
    M2S_CUDA(cudaMemcpyAsync(h, d.p, 4, cudaMemcpyDeviceToHost, s));
    M2S_CUDA(cudaStreamSynchronize(s));
    return status_from_bits(*h);
  }
};

}  // namespace

void set_error(const std::string& msg) { t_last_error = msg; }

int cuda_fail(cudaError_t e, const char* what) {
  t_last_error = std::string(what) + ": " + cudaGetErrorString(e);
  cudaGetLastError();
  return e == cudaErrorMemoryAllocation ? M2S_ERR_OUT_OF_MEMORY : M2S_ERR_CUDA;
}

// Device check, cached per device: compute capability 10.x (sm_100a build).
int g_dev_ok[64];  // 0 unknown, 1 ok, 2 unusable

int require_device() {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
    cudaGetLastError();
    set_error("no CUDA device");
    return M2S_ERR_NO_DEVICE;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return M2S_ERR_NO_DEVICE;
  if (g_dev_ok[dev] == 0) {
    cudaDeviceProp p;
    if (cudaGetDeviceProperties(&p, dev) != cudaSuccess) return M2S_ERR_NO_DEVICE;
    g_dev_ok[dev] = p.major == 10 ? 1 : 2;
  }
  if (g_dev_ok[dev] != 1) {
    set_error("the CUDA device is not compute capability 10.x (this library is built for sm_100a)");
    return M2S_ERR_NO_DEVICE;
  }
  return M2S_OK;
}

int status_from_bits(uint32_t bits) {
  if (!bits) return M2S_OK;
  for (int s = 1; s < 32; ++s)
    if (bits & (1u << s)) return s;
  return M2S_ERR_CUDA;
}

void record_grid_stats(const uint64_t stats[kGridStats]) {
  for (int i = 0; i < kGridStats; ++i) t_grid_stats[i] = stats[i];
}

float* grid_phase_slot() { return t_profile ? t_grid_phase_ms : nullptr; }

bool profiling_enabled() { return t_profile; }

void record_query_stats(const uint64_t stats[12]) {
  for (int i = 0; i < 12; ++i) t_query_stats[i] = stats[i];
}

void record_round_log(const std::vector<uint32_t>& log) { t_round_log = log; }

int dev_alloc(void** p, size_t bytes, cudaStream_t s) {
  cudaMemPool_t pool = nullptr;
  int st = current_pool(&pool);
  if (st) return st;
  cudaError_t e = cudaMallocFromPoolAsync(p, bytes, pool, s);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMallocFromPoolAsync");
  return M2S_OK;
}

void dev_free(void* p, cudaStream_t s) { cudaFreeAsync(p, s); }

}  // namespace m2s

using namespace m2s;

namespace {

int build_mesh_handle(const float* vertices, uint64_t nv, const void* indices, uint64_t ni, int bits, int topo,
                      int accel, int sign, uint64_t T, m2s_mesh* h, cudaStream_t s) {
  Upload up;
  int st = upload_mesh(vertices, nv, indices, ni, bits, &up, s);
  if (st) return st;
  StatusWord sw;
  if ((st = sw.init(s))) return st;
  MeshInput in{up.v.p, nv, bits != M2S_INDEX_NONE ? (const void*)up.idx.p : nullptr, bits, topo, T};
  h->accel = accel;
  h->sign = sign;
  cudaGetDevice(&h->device);
  if ((st = build_device_mesh(in, &h->mesh, sw.d.p, s, accel != M2S_ACCEL_NONE))) return st;
  return sw.read(s);
}

}  // namespace

extern "C" {

int m2s_version(void) { return 100; }

const char* m2s_last_error(void) { return t_last_error.c_str(); }

const char* m2s_status_string(int status) {
  switch (status) {
    case M2S_OK: return "ok";
    case M2S_ERR_INVALID_ARGUMENT: return "invalid argument";
    case M2S_ERR_NONFINITE_QUERY: return "query point contains non-finite values";
    case M2S_ERR_INDEX_COUNT: return "TriangleList length must be divisible by 3";
    case M2S_ERR_INDEX_RANGE: return "vertex index out of range";
    case M2S_ERR_NAN_DISTANCE: return "NaN distance";
    case M2S_ERR_EMPTY_MESH: return "mesh has no triangles";
    case M2S_ERR_CUDA: return "CUDA error";
    case M2S_ERR_OUT_OF_MEMORY: return "out of device memory";
    case M2S_ERR_LIMIT: return "a bounded device loop hit its limit";
    case M2S_ERR_NO_DEVICE: return "no usable sm_100 CUDA device";
    case M2S_ERR_FORMAT: return "malformed serialized signed distance field";
    default: return "unknown status";
  }
}

int m2s_device_available(void) { return require_device() == M2S_OK ? 1 : 0; }

void m2s_set_query_budget(uint32_t node_visits) { g_query_budget = node_visits; }
uint32_t m2s_query_budget(void) { return g_query_budget; }

int m2s_last_grid_stats(uint64_t out[10]) {
  if (!out) return M2S_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < 10; ++i) out[i] = t_grid_stats[i];
  return M2S_OK;
}

int m2s_pool_usage(uint64_t out[2]) {
  if (!out) return M2S_ERR_INVALID_ARGUMENT;
  out[0] = out[1] = 0;
  int dev = 0;
  M2S_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return M2S_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lk(g_pool_mu);
  if (!g_pool_ready[dev]) return M2S_OK;  // nothing allocated on this device yet
  M2S_CUDA(cudaMemPoolGetAttribute(g_pools[dev], cudaMemPoolAttrUsedMemCurrent, &out[0]));
  M2S_CUDA(cudaMemPoolGetAttribute(g_pools[dev], cudaMemPoolAttrReservedMemCurrent, &out[1]));
  return M2S_OK;
}

int m2s_last_query_audit(uint64_t out[7]) {
  if (!out) return M2S_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < 7; ++i) out[i] = t_query_stats[5 + i];
  return M2S_OK;
}

int m2s_last_grid_audit(uint64_t out[7]) {
  if (!out) return M2S_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < 7; ++i) out[i] = t_grid_stats[12 + i];
  return M2S_OK;
}

int m2s_last_grid_filter_stats(uint64_t out[2]) {
  if (!out) return M2S_ERR_INVALID_ARGUMENT;
  out[0] = t_grid_stats[10];
  out[1] = t_grid_stats[11];
  return M2S_OK;
}

void m2s_set_profiling(int enable) { t_profile = enable != 0; }

int m2s_last_query_stats(uint64_t out[5]) {
  if (!out) return M2S_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < 5; ++i) out[i] = t_query_stats[i];
  return M2S_OK;
}

uint32_t m2s_last_grid_round_log(uint32_t* out, uint32_t capacity) {
  const uint32_t n = (uint32_t)(t_round_log.size() / 2);
  if (out)
    for (uint32_t i = 0; i < n && i < capacity; ++i) {
      out[2 * i] = t_round_log[2 * i];
      out[2 * i + 1] = t_round_log[2 * i + 1];
    }
  return n;
}

int m2s_last_grid_phase_ms(float out[4]) {
  if (!out) return M2S_ERR_INVALID_ARGUMENT;
  for (int i = 0; i < 4; ++i) out[i] = t_grid_phase_ms[i];
  return M2S_OK;
}

int m2s_generate_sdf(const float* vertices, uint64_t nv, const void* indices, uint64_t ni, int bits, int topo,
                     const float* q, uint64_t nq, int accel, int sign, float* out, uint64_t* out_len, void* stream) {
  if (out_len) *out_len = 0;
  if (accel < M2S_ACCEL_NONE || accel > M2S_ACCEL_RTREE_BVH || sign < 0 || sign > 1) return M2S_ERR_INVALID_ARGUMENT;
  if (nq && (!q || !out)) return M2S_ERR_INVALID_ARGUMENT;
  if (!all_finite(q, nq)) return M2S_ERR_NONFINITE_QUERY;  // lib.rs:374-376
  uint64_t T = 0;
  int st = triangle_count(nv, indices, ni, bits, topo, &T);
  if (st) return st;
  if ((st = require_device())) return st;
  cudaStream_t s = (cudaStream_t)stream;
  m2s_mesh h;
  if ((st = build_mesh_handle(vertices, nv, indices, ni, bits, topo, accel, sign, T, &h, s))) {
    // generate_sdf_default never reads a vertex when there is no query.
    if (!(st == M2S_ERR_INDEX_RANGE && accel == M2S_ACCEL_NONE && nq == 0)) return st;
  }
  if (T == 0 && accel == M2S_ACCEL_RTREE_BVH) return M2S_OK;  // rtree_bvh.rs:96-97: empty Vec
  if (T == 0 && accel != M2S_ACCEL_NONE && nq > 0) return M2S_ERR_EMPTY_MESH;
  if (nq == 0) return M2S_OK;
  DevBuf<float> dq, dout;
  if ((st = dq.alloc(3 * nq, s)) || (st = dout.alloc(nq, s))) return st;
  M2S_CUDA(cudaMemcpyAsync(dq.p, q, 12 * nq, cudaMemcpyHostToDevice, s));
  StatusWord sw;
  if ((st = sw.init(s))) return st;
  if ((st = query_points(h.mesh.view(), accel, sign, dq.p, nq, dout.p, nullptr, nullptr, sw.d.p, s))) return st;
  M2S_CUDA(cudaMemcpyAsync(out, dout.p, 4 * nq, cudaMemcpyDeviceToHost, s));
  if ((st = sw.read(s))) return st;
  if (out_len) *out_len = nq;
  return M2S_OK;
}

int m2s_build_sdf_acceleration(const float* vertices, uint64_t nv, const void* indices, uint64_t ni, int bits,
                               int topo, int accel, int sign, m2s_mesh** out_mesh, void* stream) {
  if (!out_mesh) return M2S_ERR_INVALID_ARGUMENT;
  *out_mesh = nullptr;
  if (accel < M2S_ACCEL_NONE || accel > M2S_ACCEL_RTREE_BVH || sign < 0 || sign > 1) return M2S_ERR_INVALID_ARGUMENT;
  uint64_t T = 0;
  int st = triangle_count(nv, indices, ni, bits, topo, &T);
  if (st) return st;
  if ((st = require_device())) return st;
  if (T == 0 && accel == M2S_ACCEL_RTREE_BVH) return M2S_OK;  // rtree_bvh.rs:124-126: None
  cudaStream_t s = (cudaStream_t)stream;
  m2s_mesh* h = new m2s_mesh();
  if ((st = build_mesh_handle(vertices, nv, indices, ni, bits, topo, accel, sign, T, h, s))) {
    delete h;
    return st;
  }
  *out_mesh = h;
  return M2S_OK;
}

void m2s_mesh_free(m2s_mesh* mesh) {
  if (!mesh) return;
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(mesh->device);
  cudaDeviceSynchronize();
  delete mesh;
  cudaSetDevice(prev);
}

uint64_t m2s_mesh_triangle_count(const m2s_mesh* mesh) { return mesh ? mesh->mesh.n_tris : 0; }
int m2s_mesh_accel(const m2s_mesh* mesh) { return mesh ? mesh->accel : -1; }

int m2s_query_sdf(const m2s_mesh* mesh, const float* q, uint64_t nq, float* out, uint64_t* out_len, void* stream) {
  if (out_len) *out_len = 0;
  if (!mesh || (nq && (!q || !out))) return M2S_ERR_INVALID_ARGUMENT;
  if (!all_finite(q, nq)) return M2S_ERR_NONFINITE_QUERY;
  int st;
  if ((st = require_device())) return st;
  if (nq == 0) return M2S_OK;
  if (mesh->mesh.n_tris == 0 && mesh->accel != M2S_ACCEL_NONE) return M2S_ERR_EMPTY_MESH;
  cudaStream_t s = (cudaStream_t)stream;
  DevBuf<float> dq, dout;
  if ((st = dq.alloc(3 * nq, s)) || (st = dout.alloc(nq, s))) return st;
  M2S_CUDA(cudaMemcpyAsync(dq.p, q, 12 * nq, cudaMemcpyHostToDevice, s));
  StatusWord sw;
  if ((st = sw.init(s))) return st;
  if ((st = query_points(mesh->mesh.view(), mesh->accel, mesh->sign, dq.p, nq, dout.p, nullptr, nullptr, sw.d.p, s)))
    return st;
  M2S_CUDA(cudaMemcpyAsync(out, dout.p, 4 * nq, cudaMemcpyDeviceToHost, s));
  if ((st = sw.read(s))) return st;
  if (out_len) *out_len = nq;
  return M2S_OK;
}

int m2s_query_vector_to_closest_point(const m2s_mesh* mesh, const float* q, uint64_t nq, float* out_vec,
                                      uint8_t* out_inside, uint64_t* out_len, void* stream) {
  if (out_len) *out_len = 0;
  if (!mesh || (nq && (!q || !out_vec || !out_inside))) return M2S_ERR_INVALID_ARGUMENT;
  if (mesh->accel != M2S_ACCEL_RTREE_BVH) return M2S_ERR_INVALID_ARGUMENT;
  if (!all_finite(q, nq)) return M2S_ERR_NONFINITE_QUERY;
  int st;
  if ((st = require_device())) return st;
  if (nq == 0) return M2S_OK;
  cudaStream_t s = (cudaStream_t)stream;
  DevBuf<float> dq, dvec;
  DevBuf<uint8_t> din;
  if ((st = dq.alloc(3 * nq, s)) || (st = dvec.alloc(3 * nq, s)) || (st = din.alloc(nq, s))) return st;
  M2S_CUDA(cudaMemcpyAsync(dq.p, q, 12 * nq, cudaMemcpyHostToDevice, s));
  StatusWord sw;
  if ((st = sw.init(s))) return st;
  if ((st = query_points(mesh->mesh.view(), M2S_ACCEL_RTREE_BVH, M2S_SIGN_RAYCAST, dq.p, nq, nullptr, dvec.p, din.p,
                         sw.d.p, s)))
    return st;
  M2S_CUDA(cudaMemcpyAsync(out_vec, dvec.p, 12 * nq, cudaMemcpyDeviceToHost, s));
  M2S_CUDA(cudaMemcpyAsync(out_inside, din.p, nq, cudaMemcpyDeviceToHost, s));
  if ((st = sw.read(s))) return st;
  if (out_len) *out_len = nq;
  return M2S_OK;
}

int m2s_generate_grid_sdf(const float* vertices, uint64_t nv, const void* indices, uint64_t ni, int bits, int topo,
                          const float first_cell[3], const float cell_size[3], const uint64_t cell_count[3], int sign,
                          float* out, uint64_t* out_len, void* stream) {
  if (out_len) *out_len = 0;
  if (!first_cell || !cell_size || !cell_count || sign < 0 || sign > 1) return M2S_ERR_INVALID_ARGUMENT;
  uint64_t T = 0;
  int st = triangle_count(nv, indices, ni, bits, topo, &T);
  if (st) return st;
  GridDesc g;
  for (int d = 0; d < 3; ++d) {
    g.first[d] = first_cell[d];
    g.size[d] = cell_size[d];
    g.n[d] = cell_count[d];
  }
  const uint64_t N = g.cells();
  if (N == 0) return T ? M2S_ERR_INVALID_ARGUMENT : M2S_OK;  // zero count: the crate's clamp panics
  if (!out) return M2S_ERR_INVALID_ARGUMENT;
  if ((st = require_device())) return st;
  cudaStream_t s = (cudaStream_t)stream;
  Upload up;
  if ((st = upload_mesh(vertices, nv, indices, ni, bits, &up, s))) return st;
  StatusWord sw;
  if ((st = sw.init(s))) return st;
  MeshInput in{up.v.p, nv, bits != M2S_INDEX_NONE ? (const void*)up.idx.p : nullptr, bits, topo, T};
  DeviceMesh mesh;
  // The grid path needs the triangle records only (seeding and lattice rays
  // walk triangles directly), so no LBVH is built here.
  if ((st = build_device_mesh(in, &mesh, sw.d.p, s, /*with_tree=*/false))) return st;
  if ((st = sw.read(s))) return st;  // index errors stop the call before the grid runs
  DevBuf<float> dout;
  if ((st = dout.alloc(N, s))) return st;
  uint64_t stats[kGridStats] = {};
  if ((st = grid_sdf(mesh.view(), g, sign, dout.p, sw.d.p, s, stats, t_profile ? t_grid_phase_ms : nullptr)))
    return st;
  for (int i = 0; i < kGridStats; ++i) t_grid_stats[i] = stats[i];
  M2S_CUDA(cudaMemcpyAsync(out, dout.p, 4 * N, cudaMemcpyDeviceToHost, s));
  if ((st = sw.read(s))) return st;
  if (out_len) *out_len = N;
  return M2S_OK;
}

int m2s_query_sdf_device(const m2s_mesh* mesh, const float* d_q, uint64_t nq, float* d_out, uint32_t* d_status,
                         void* stream) {
  if (!mesh || (nq && (!d_q || !d_out))) return M2S_ERR_INVALID_ARGUMENT;
  int st;
  if ((st = require_device())) return st;
  if (nq == 0) return M2S_OK;
  if (mesh->mesh.n_tris == 0 && mesh->accel != M2S_ACCEL_NONE) return M2S_ERR_EMPTY_MESH;
  cudaStream_t s = (cudaStream_t)stream;
  DevBuf<uint32_t> own;
  if (!d_status) {
    if ((st = own.alloc(1, s))) return st;
    M2S_CUDA(cudaMemsetAsync(own.p, 0, 4, s));
    d_status = own.p;
  }
  return query_points(mesh->mesh.view(), mesh->accel, mesh->sign, d_q, nq, d_out, nullptr, nullptr, d_status, s);
}

int m2s_query_autotune(const m2s_mesh* mesh, const float* d_q, uint64_t nq, void* stream, uint32_t* out_budget,
                       float out_ms[kQueryBudgetCandidates]) {
  if (!mesh || !d_q || nq == 0) return M2S_ERR_INVALID_ARGUMENT;
  int st;
  if ((st = require_device())) return st;
  if (mesh->mesh.n_tris == 0 || mesh->accel == M2S_ACCEL_NONE) return M2S_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  DevBuf<float> out;
  DevBuf<uint32_t> status;
  if ((st = out.alloc(nq, s)) || (st = status.alloc(1, s))) return st;
  M2S_CUDA(cudaMemsetAsync(status.p, 0, 4, s));
  cudaEvent_t e0, e1;
  M2S_CUDA(cudaEventCreate(&e0));
  M2S_CUDA(cudaEventCreate(&e1));
  // Candidates are passed to each timed call, never published while timing:
  // concurrent queries keep the current budget, and a budget set by another
  // thread meanwhile wins over the result below.
  uint32_t saved = g_query_budget.load();
  float best_ms = INFINITY;
  uint32_t best = saved;
  for (int c = 0; c < kQueryBudgetCandidates && !st; ++c) {
    float ms = INFINITY;
    // one warm-up, then the faster of two timed runs
    for (int rep = 0; rep < 3 && !st; ++rep) {
      if (rep && cudaEventRecord(e0, s) != cudaSuccess) st = M2S_ERR_CUDA;
      if (!st) st = query_points(mesh->mesh.view(), mesh->accel, mesh->sign, d_q, nq, out.p, nullptr, nullptr,
                                 status.p, s, kQueryBudgets[c]);
      if (!st && rep) {
        float t = 0.0f;
        if (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
            cudaEventElapsedTime(&t, e0, e1) != cudaSuccess)
          st = M2S_ERR_CUDA;
        ms = std::min(ms, t);
      }
    }
    if (out_ms) out_ms[c] = ms;
    if (ms < best_ms) {
      best_ms = ms;
      best = kQueryBudgets[c];
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!st) g_query_budget.compare_exchange_strong(saved, best);  // unless it was set meanwhile
  if (out_budget) *out_budget = st ? saved : best;
  return st;
}

int m2s_grid_sdf_device(const m2s_mesh* mesh, const float first_cell[3], const float cell_size[3],
                        const uint64_t cell_count[3], int sign, float* d_out, uint32_t* d_status, void* stream) {
  if (!mesh || !first_cell || !cell_size || !cell_count || sign < 0 || sign > 1) return M2S_ERR_INVALID_ARGUMENT;
  int st;
  if ((st = require_device())) return st;
  GridDesc g;
  for (int d = 0; d < 3; ++d) {
    g.first[d] = first_cell[d];
    g.size[d] = cell_size[d];
    g.n[d] = cell_count[d];
  }
  if (g.cells() == 0) return mesh->mesh.n_tris ? M2S_ERR_INVALID_ARGUMENT : M2S_OK;
  if (!d_out) return M2S_ERR_INVALID_ARGUMENT;
  cudaStream_t s = (cudaStream_t)stream;
  DevBuf<uint32_t> own;
  if (!d_status) {
    if ((st = own.alloc(1, s))) return st;
    M2S_CUDA(cudaMemsetAsync(own.p, 0, 4, s));
    d_status = own.p;
  }
  uint64_t stats[kGridStats] = {};
  st = grid_sdf(mesh->mesh.view(), g, sign, d_out, d_status, s, stats, t_profile ? t_grid_phase_ms : nullptr);
  for (int i = 0; i < kGridStats; ++i) t_grid_stats[i] = stats[i];
  return st;
}

int m2s_radix_sort_pairs_device(uint32_t* d_keys, uint32_t* d_values, uint64_t n, int key_bits, void* stream) {
  int st;
  if ((st = require_device())) return st;
  if (n && (!d_keys || !d_values)) return M2S_ERR_INVALID_ARGUMENT;
  return radix_sort_pairs(d_keys, d_values, n, key_bits, (cudaStream_t)stream);
}

}  // extern "C"
