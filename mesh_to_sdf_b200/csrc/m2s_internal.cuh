// Internal declarations shared by the mesh_to_sdf_b200 CUDA sources.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cmath>
#include <memory>
#include <string>
#include <vector>

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

// budget >= 0 overrides the process-wide node budget (g_query_budget) for
// this call only: the autotuner times candidates without publishing them.
int query_points(const MeshView& m, int accel, int sign, const float* d_q, uint64_t nq, float* d_out,
                 float* d_vec, uint8_t* d_inside, uint32_t* d_status, cudaStream_t s, int64_t budget = -1);

// Node visits a query may spend in the one-thread-per-query pass before it is
// continued one warp per query (0 disables the second pass).
extern std::atomic<uint32_t> g_query_budget;
// The budget a batch of nq queries uses: `base` from 2^20 queries up,
// base * sqrt(nq / 2^20) from 2^18, and base / 16 below, at least 64 (0 stays
// 0: no warp pass).  Below 2^18 queries every query has a thread from the
// start and the batch waits for its longest searches, which the warp pass
// finishes sooner (star s6 mixed points, Rtree, base 1024: 50,000 queries
// 1.30 -> 1.08 ms, 100,000 1.68 -> 1.51 ms); from 2^18 on, the thread pass's
// throughput counts (400,000: 3.32 ms at 632 against 3.83 at 316 and 3.99 at 158).
inline uint32_t effective_query_budget(uint32_t base, uint64_t nq) {
  if (base == 0) return 0;
  const double f = nq >= (1ull << 20) ? 1.0
                   : nq >= (1ull << 18) ? std::sqrt((double)nq / (double)(1ull << 20))
                                        : 1.0 / 16.0;
  const uint32_t b = (uint32_t)(base * f + 0.5);
  return b < 64 ? std::min<uint32_t>(64, base) : b;
}
// Node budgets the query autotuner tries (64 also moves Bvh(Normal) batches
// of 2^18 queries and more to the warp hand-off: see query_points).
constexpr int kQueryBudgetCandidates = 8;
constexpr uint32_t kQueryBudgets[kQueryBudgetCandidates] = {0, 64, 256, 512, 1024, 1536, 2048, 4096};
// Base budgets at or below this hand Bvh(Normal) searches and band folds to
// the warp pass at every batch size; larger ones keep batches of 2^18
// queries and more in one pass.
constexpr uint32_t kNormalHandoffMaxBudget = 64;

// Profiling (m2s_set_profiling, per host thread): whether it is on, and the
// traversal counts of the last point query made with it on:
// [queries, search node fetches, search triangle tests, sign node fetches,
// sign triangle tests].
bool profiling_enabled();
// [queries, the four traversal counts, the seven FP64-audit counts]
void record_query_stats(const uint64_t stats[12]);

// allow_alloc = false keeps the brute force in one pass with no scratch buffer.
int brute_force_sdf(const MeshView& m, int sign, const float* d_q, uint64_t nq, float* d_out,
                    uint32_t* d_status, cudaStream_t s, bool allow_alloc = true);

// ---- grid (m2s_grid.cu) ------------------------------------------------------

struct GridDesc {
  float first[3];
  float size[3];
  uint64_t n[3];
  // Cell count, saturated at UINT64_MAX when the product overflows.
  uint64_t cells() const {
    unsigned __int128 c = (unsigned __int128)n[0] * n[1];
    if (c > UINT64_MAX) return UINT64_MAX;
    c *= n[2];
    return c > UINT64_MAX ? UINT64_MAX : (uint64_t)c;
  }
};

// stats: [seed updates, relax rounds, states relaxed, neighbour proposals,
// ray hits, overflow restarts, kernel launches, far-list redistributions,
// rounds relaxed by one block alone, largest list relaxed in one round,
// proposals dropped because the neighbour holds the proposing triangle,
// proposals dropped by the distance bound, then the FP64 audit's seven
// counters (zero unless GridTuning::fp64_audit): ray tests, ambiguous ray
// tests, ray tests FP64 decides otherwise, cells whose Raycast vote the FP64
// decisions flip, cells whose Voronoi region was audited, ambiguous region
// choices, region choices FP64 makes otherwise].  phase_ms (may be NULL)
// receives device time of [seeding, propagation, rays, finalize].
constexpr int kGridStats = 19;
int grid_sdf(const MeshView& m, const GridDesc& g, int sign, float* d_out, uint32_t* d_status, cudaStream_t s,
             uint64_t stats[kGridStats], float phase_ms[4]);

// Knobs that change speed, never results.
struct GridTuning {
  int blocks_per_sm = 0;             // cooperative blocks per SM (0: occupancy limit)
  uint32_t cells_per_block = 1024;   // cooperative grid = ceil(cells / this) blocks, at least one per SM
  uint32_t list_capacity = 0;        // entries per bucket list (0: derived from the cell count)
  // A batch runs as jobs ("waves") of at most this many cells each (a larger
  // grid alone), which bounds a job's keys (8 bytes per cell) and lists.
  uint64_t wave_cells = 1ull << 27;
  // Relax rounds of at most this many states run on one block, with block
  // barriers only (0: every round on every block).
  uint32_t solo_max = 64;
  // Drop proposals that a per-triangle distance bound proves cannot win
  // before their closest-point evaluation, in the filtered kernel variant
  // (off: the plain variant; results are identical either way).
  bool bound_filter = false;
  // Audit every ray test and every cell's Voronoi region against an f32
  // error bound and re-decide the ambiguous ones in FP64 (counts only; the
  // output does not change).
  bool fp64_audit = false;
};

struct GridRunInfo {
  bool overflow = false;
  uint64_t seeds = 0, rounds = 0, entries = 0, evals = 0, ray_hits = 0, far_phases = 0, launches = 0, solo_rounds = 0,
           max_list = 0, log_n = 0, filter_same = 0, filter_bound = 0;
  uint64_t audit[7] = {0, 0, 0, 0, 0, 0, 0};
};

// A set of (mesh, grid) pairs computed together: one cell index space (grid k
// starts at the sum of the cells of grids 0..k-1, which is also where its
// output starts in d_out) and one triangle array.  prepare() allocates and
// uploads everything; enqueue() queues the whole pipeline on a stream with no
// host synchronisation, so it can be captured into a CUDA graph; read_state()
// waits for the stream and reports whether the bucket lists overflowed, in
// which case the caller raises the capacity and runs enqueue() again (the
// rerun starts from scratch, so results never depend on the capacity).
class GridJob {
 public:
  GridJob();
  ~GridJob();
  GridJob(const GridJob&) = delete;
  GridJob& operator=(const GridJob&) = delete;
  // out_offsets[k] (NULL: back to back from 0) is where grid k's values start in d_out.
  int prepare(const MeshView* meshes, uint32_t n, const GridDesc* grids, int sign, float* d_out, uint32_t* d_status,
              cudaStream_t s, const GridTuning& tune, const uint64_t* out_offsets = nullptr);
  int alloc_lists(cudaStream_t s);
  int enqueue(cudaStream_t s, cudaEvent_t* ev5);
  int read_state(cudaStream_t s, GridRunInfo* info);
  uint32_t capacity() const;
  void set_capacity(uint32_t cap);
  uint64_t cells() const;
  uint64_t device_bytes() const;  // workspace held by the job (lists included)
  unsigned cooperative_blocks() const;
  unsigned max_cooperative_blocks() const;
  void set_cooperative_blocks(unsigned blocks);  // clamped to [1, max_cooperative_blocks()]
  int sign() const;
  uint32_t grids() const;
  // Profiling: record every propagation step (kind and size, and the time it
  // was chosen) in a device log of `cap` steps.
  int enable_round_log(uint32_t cap, cudaStream_t s);
  int read_round_log(std::vector<uint32_t>* out, uint32_t n, cudaStream_t s);

 private:
  struct Impl;
  Impl* p;
};

// Runs a job to completion (restarting with larger lists on overflow).
int run_grid_job(GridJob& job, cudaStream_t s, uint64_t stats[kGridStats], float phase_ms[4]);

// Waves of a batch: grid indices per job, largest grids first, first fit into
// jobs of at most wave_cells cells (a larger grid alone).
std::vector<std::vector<uint32_t>> plan_waves(const GridDesc* grids, uint32_t n, uint64_t wave_cells);

// One prepared job per wave of a batch (outputs back to back in d_out, in the
// order of `grids`).
int prepare_waves(const MeshView* meshes, uint32_t n, const GridDesc* grids, int sign, float* d_out,
                  uint32_t* d_status, cudaStream_t s, const GridTuning& tune,
                  std::vector<std::unique_ptr<GridJob>>* jobs);

// n (mesh, grid) pairs, wave by wave; results back to back in d_out.
int grid_sdf_batch(const MeshView* meshes, uint32_t n, const GridDesc* grids, int sign, float* d_out,
                   uint32_t* d_status, cudaStream_t s, uint64_t stats[kGridStats], float phase_ms[4],
                   const GridTuning& tune);

// Validates a grid description for the device path (32-bit cell indices).
int check_grid(const GridDesc& g);

// Blocks of the propagation kernel that fit on one SM (its occupancy limit).
int propagate_blocks_per_sm(int sign);

// Entries per bucket list of a job of `cells` cells (before any overflow
// restart), and the device bytes of such a job's workspace.
uint32_t default_list_capacity(uint64_t cells);
uint64_t grid_job_bytes(uint64_t cells);

// Process-wide grid knobs (m2s_set_grid_tuning), read as a copy under a lock:
// a caller may change them while other threads (the server's) run grids.
GridTuning grid_tuning();
void set_grid_tuning(const GridTuning& t);

// ---- host API helpers (m2s_api.cu) -------------------------------------------

// M2S_OK when the current device is compute capability 10.x.
int require_device();
// Records the counters / phase times of the last grid call of this thread.
void record_grid_stats(const uint64_t stats[kGridStats]);
float* grid_phase_slot();  // NULL unless profiling is on
void record_round_log(const std::vector<uint32_t>& log);
int status_from_bits(uint32_t bits);

}  // namespace m2s

// Resident mesh behind the m2s_mesh handle.
struct m2s_mesh {
  int device = 0;
  int accel = 0;
  int sign = 0;
  m2s::DeviceMesh mesh;
};

namespace m2s {

}  // namespace m2s
