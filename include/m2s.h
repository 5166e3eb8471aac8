/* mesh_to_sdf_b200 — C ABI of the B200 (sm_100a) signed-distance library.
 *
 * This is the drop-in boundary for the Rust crate `mesh_to_sdf`: every entry
 * point below replaces one public function of that crate (citations are
 * `mesh_to_sdf/src/<file>:<line>`), with the crate's arguments flattened to
 * plain pointers and sizes.  A Rust shim maps `Topology`, `SignMethod`,
 * `AccelerationMethod`, `Grid` and `Point` (flattened to float[3]) onto these
 * calls and turns non-zero status codes back into the crate's panics.
 *
 * Conventions
 *  - vertices / query points: float[3 * n], x y z interleaved (a `[f32; 3]`
 *    slice, or any `Point` copied out through x()/y()/z()).
 *  - indices: NULL with index_bits = M2S_INDEX_NONE (the crate's `None`), or
 *    uint16_t* / uint32_t* with index_bits = 16 / 32.
 *  - outputs are caller-allocated; *out_len receives the number of results,
 *    which is 0 exactly when the crate returns an empty Vec.
 *  - `stream` is a cudaStream_t (NULL = the legacy default stream).  Host-
 *    pointer entry points block until their results are in host memory.
 *    `_device` entry points take device pointers, enqueue on `stream` and
 *    return without synchronising; their status arrives in `d_status`.
 *  - every call runs on the calling thread's current CUDA device.
 *  - there is no CPU path: without a usable sm_100 device every compute entry
 *    point returns M2S_ERR_NO_DEVICE.
 */
#ifndef M2S_H
#define M2S_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  The crate panics where these are non-zero. */
enum m2s_status {
  M2S_OK = 0,
  M2S_ERR_INVALID_ARGUMENT = 1,
  M2S_ERR_NONFINITE_QUERY = 2, /* lib.rs:374-376 assert!(point.is_finite()) */
  M2S_ERR_INDEX_COUNT = 3,     /* lib.rs:203, lib.rs:207 list length % 3 != 0 */
  M2S_ERR_INDEX_RANGE = 4,     /* slice indexing panic (test at lib.rs:557-566) */
  M2S_ERR_NAN_DISTANCE = 5,    /* lib.rs:330 expect("NaN distance") */
  M2S_ERR_EMPTY_MESH = 6,      /* rtree.rs:148 nearest.unwrap() on an empty tree */
  M2S_ERR_CUDA = 7,
  M2S_ERR_OUT_OF_MEMORY = 8,
  M2S_ERR_LIMIT = 9, /* a bounded device loop (stack, worklist, rounds) hit its limit */
  M2S_ERR_NO_DEVICE = 10,
  M2S_ERR_FORMAT = 11 /* serde.rs: SerdeError::DeserializationFailed */
};

enum { M2S_TOPOLOGY_TRIANGLE_LIST = 0, M2S_TOPOLOGY_TRIANGLE_STRIP = 1 }; /* lib.rs:156-171 */
enum { M2S_INDEX_NONE = 0, M2S_INDEX_U16 = 16, M2S_INDEX_U32 = 32 };
enum { M2S_SIGN_RAYCAST = 0, M2S_SIGN_NORMAL = 1 }; /* lib.rs:252-263 */
enum {                                              /* lib.rs:272-286 */
       M2S_ACCEL_NONE = 0,
       M2S_ACCEL_BVH = 1,
       M2S_ACCEL_RTREE = 2,
       M2S_ACCEL_RTREE_BVH = 3
};

/* Resident acceleration structure: `SdfAccelerationMesh` (lib.rs:303-312).
 * Owns device copies of the mesh and its LBVH; immutable after build and safe
 * to query from several streams at once. */
typedef struct m2s_mesh m2s_mesh;

/* generate_sdf (lib.rs:364-391).  `sign` is ignored for RTREE (always the
 * normal sign, rtree.rs:137-157) and RTREE_BVH (always the 3-ray vote,
 * rtree_bvh.rs:143-201).  out: n_queries floats. */
int m2s_generate_sdf(const float* vertices, uint64_t n_vertices, const void* indices,
                     uint64_t n_indices, int index_bits, int topology, const float* query_points,
                     uint64_t n_queries, int accel, int sign, float* out, uint64_t* out_len,
                     void* stream);

/* generate_grid_sdf (generate/grid.rs:265-378).  The grid is `Grid::new(first_cell,
 * cell_size, cell_count)` (grid.rs:43-49); out holds the cell_count product of
 * floats in the crate's order, index = z + y*nz + x*ny*nz (grid.rs:122-124). */
int m2s_generate_grid_sdf(const float* vertices, uint64_t n_vertices, const void* indices,
                          uint64_t n_indices, int index_bits, int topology,
                          const float first_cell[3], const float cell_size[3],
                          const uint64_t cell_count[3], int sign, float* out, uint64_t* out_len,
                          void* stream);

/* build_sdf_acceleration (lib.rs:410-433).  *out_mesh is NULL (and M2S_OK is
 * returned) exactly where the crate returns None: RTREE_BVH on an empty mesh
 * (rtree_bvh.rs:124-126). */
int m2s_build_sdf_acceleration(const float* vertices, uint64_t n_vertices, const void* indices,
                               uint64_t n_indices, int index_bits, int topology, int accel,
                               int sign, m2s_mesh** out_mesh, void* stream);

/* query_sdf (lib.rs:463-485).  Non-finite query points are rejected with
 * M2S_ERR_NONFINITE_QUERY (the crate does not check them here). */
int m2s_query_sdf(const m2s_mesh* mesh, const float* query_points, uint64_t n_queries,
                  float* out, uint64_t* out_len, void* stream);

/* query_vector_to_closest_point_rtree_bvh (rtree_bvh.rs:217-276, exported at
 * lib.rs:150).  The mesh must have been built with M2S_ACCEL_RTREE_BVH.
 * out_vectors: 3 floats per query (closest point - query); out_inside: 1 byte
 * per query (1 = inside by the 3-ray vote). */
int m2s_query_vector_to_closest_point(const m2s_mesh* mesh, const float* query_points,
                                      uint64_t n_queries, float* out_vectors,
                                      uint8_t* out_inside, uint64_t* out_len, void* stream);

/* Releases a handle from m2s_build_sdf_acceleration (NULL is a no-op). */
void m2s_mesh_free(m2s_mesh* mesh);

/* Triangle count and acceleration method of a handle. */
uint64_t m2s_mesh_triangle_count(const m2s_mesh* mesh);
int m2s_mesh_accel(const m2s_mesh* mesh);

/* ---- device-resident variants (HBM in, HBM out, asynchronous) ----------- */

/* query_sdf over device arrays.  d_status: device uint32 that receives the
 * OR of status bits (1 << code) raised by the kernels; may be NULL. */
int m2s_query_sdf_device(const m2s_mesh* mesh, const float* d_query_points, uint64_t n_queries,
                         float* d_out, uint32_t* d_status, void* stream);

/* generate_grid_sdf against a resident mesh (built with any method; the grid
 * path uses its triangles only).  d_out: device floats.  Unlike the other
 * _device calls it returns once d_out is written: the host reads back whether
 * the propagation lists overflowed (and reruns with larger ones if so). */
int m2s_grid_sdf_device(const m2s_mesh* mesh, const float first_cell[3],
                        const float cell_size[3], const uint64_t cell_count[3], int sign,
                        float* d_out, uint32_t* d_status, void* stream);

/* ---- batches of grids (no counterpart in the reference) ------------------ */

/* The crate computes one grid per call (generate/grid.rs:265-274); a server
 * with many small requests would pay each call's fixed cost — propagation
 * rounds that each end in a device-wide barrier — once per grid.  These calls
 * compute n_grids (mesh, grid) pairs in one job instead.  Grid k uses
 * meshes[k] (a resident handle; all on the current device) and
 * first_cells[3k..3k+2], cell_sizes[3k..3k+2], cell_counts[3k..3k+2]; its
 * cells start at d_out + (cells of grids 0..k-1).  Every grid's result is
 * bit-identical to m2s_grid_sdf_device on that mesh and grid alone.  The job
 * addresses cells with 32-bit indices: fewer than 2^32 - 1 cells in total.
 * Returns once d_out is written. */
int m2s_grid_sdf_batch_device(const m2s_mesh* const* meshes, uint32_t n_grids,
                              const float* first_cells, const float* cell_sizes,
                              const uint64_t* cell_counts, int sign, float* d_out,
                              uint32_t* d_status, void* stream);

/* A batch prepared once (workspace allocated, pipeline captured into a CUDA
 * graph) and replayed by m2s_grid_plan_run.  The meshes, d_out and d_status
 * (required here; the kernels OR status bits into it, the caller clears it)
 * are bound at creation and must outlive the plan.  `stream` is unused at
 * creation (the plan allocates and captures on a stream of its own). */
typedef struct m2s_grid_plan m2s_grid_plan;
int m2s_grid_plan_create(const m2s_mesh* const* meshes, uint32_t n_grids,
                         const float* first_cells, const float* cell_sizes,
                         const uint64_t* cell_counts, int sign, float* d_out,
                         uint32_t* d_status, void* stream, m2s_grid_plan** out_plan);
/* Replays the plan on `stream`; returns once d_out is written. */
int m2s_grid_plan_run(m2s_grid_plan* plan, void* stream);
/* Times the plan's waves at several cooperative grid sizes (results are
 * identical at every size) and keeps the fastest per class of wave (device,
 * sign, one grid or several, log2 of the cell count), for this plan and for
 * later plans.  *out_blocks (may be NULL) receives the first wave's choice. */
int m2s_grid_plan_autotune(m2s_grid_plan* plan, void* stream, uint32_t* out_blocks);
uint64_t m2s_grid_plan_cells(const m2s_grid_plan* plan);
uint64_t m2s_grid_plan_device_bytes(const m2s_grid_plan* plan);
uint32_t m2s_grid_plan_blocks(const m2s_grid_plan* plan);
/* Number of jobs ("waves") the plan's batch was split into (see below). */
uint32_t m2s_grid_plan_waves(const m2s_grid_plan* plan);
void m2s_grid_plan_free(m2s_grid_plan* plan);
/* Forgets every autotuned choice. */
void m2s_clear_grid_autotune(void);

/* Process-wide grid knobs; they change speed, never results.  blocks_per_sm:
 * cooperative propagation blocks per SM (0 = occupancy limit; the server's
 * grid waves then run 3 per SM, leaving room for point queries);
 * cells_per_block: the propagation launch uses ceil(cells / this) blocks, at
 * least one per SM (0 = 1024); wave_cells: a batch runs as jobs of at most this many
 * cells, largest grids first (a larger grid alone); grids in one job share its
 * rounds (0 = 128M; the server keeps its waves at 4M for latency); solo_max: propagation rounds of at most this
 * many states run on one block with block barriers only (0 = never, negative
 * = the default 64, at most 64). */
void m2s_set_grid_tuning(int blocks_per_sm, uint32_t cells_per_block, uint64_t wave_cells, int solo_max);
/* Process-wide (no counterpart in the reference): with enable != 0, grid
 * propagation runs its filtered kernel variant, which drops, before their
 * closest-point evaluation, the proposals that a per-triangle distance bound
 * (the triangle's plane and edge lines, with a slack far above f32 rounding)
 * proves cannot beat the cell's value (on the star s6 256^3 grid: half of
 * them); 0 (the default) runs the plain variant.  Results are identical
 * either way.  The propagation is bound by dependent memory trips, not by
 * the evaluations, so the filter pays only on some inputs (the star s6 Normal
 * grid 13.9 -> 13.3 ms; the Raycast grid and the terrain slightly slower). */
void m2s_set_grid_bound_filter(int enable);

/* generate_sdf with AccelerationMethod::None for callers that cannot allocate
 * device memory.  No counterpart in the reference: the crate allocates freely.
 * Every input and output is a caller-owned device pointer; the only scratch
 * (the mesh's triangle records and a status word) is a fixed 12 MiB
 * `static __device__` array inside this library, so the call itself performs
 * no cudaMalloc/cudaFree.  Callers that need this: real-time loops that cannot
 * risk the device-wide synchronisation an allocation may cause, and
 * applications that have already given their whole device-memory budget to
 * their own pool.  Limits: at most 262,144 triangles (more returns
 * M2S_ERR_INVALID_ARGUMENT); devices 0..63 only (a higher current device
 * returns M2S_ERR_INVALID_ARGUMENT); the array is held by every device that loads the
 * library until the process exits; all calls share it, so calls that overlap
 * on the GPU race and must be serialised by the caller.  The first call on a
 * device looks up the array's address with that device current — make it
 * before any stream capture.  Returns once d_out is written, with the status
 * of the kernels (same codes and checks as m2s_generate_sdf). */
int m2s_generate_sdf_none_noalloc(const float* d_vertices, uint64_t n_vertices,
                                  const void* d_indices, uint64_t n_indices, int index_bits,
                                  int topology, const float* d_query_points, uint64_t n_queries,
                                  int sign, float* d_out, void* stream);

/* ---- serving loop (no counterpart in the reference) ----------------------- */

/* The crate's resident API (build_sdf_acceleration / query_sdf, lib.rs:410-485)
 * answers one call at a time on the caller's thread.  A server owns resident
 * meshes and worker threads (uploads, point requests, and two grid lanes)
 * and admits requests against a device-memory budget: each reserves an
 * estimate of what it will hold and waits, in arrival order per kind, until
 * that fits.  Point requests on different meshes overlap on a pool of
 * `point_streams` streams (0 = 4); a free grid lane takes the grid requests
 * waiting at that moment (up to 4M cells) as one wave, so a request is
 * admitted at the next wave boundary, and the two lanes' waves run side by
 * side (each on half the propagation blocks per SM; a wave that starts while
 * the other lane is idle and nothing else waits takes all but one).  Every result equals the one the single-request
 * calls give (m2s_query_sdf with the mesh's method; m2s_grid_sdf_device).
 * Submissions return a ticket at once; the caller's host buffers (queries,
 * outputs) must stay valid until m2s_server_wait returns for that ticket.
 * Pinned host buffers let copies overlap kernels.  Free the server only
 * after every ticket was waited for. */
typedef struct m2s_server m2s_server;
int m2s_server_create(uint64_t hbm_budget_bytes, uint32_t point_streams, m2s_server** out);
void m2s_server_free(m2s_server* server);
/* Copies the mesh now; its triangle records and LBVH are built by the server.
 * *mesh_id is valid at once: requests on it wait until the build is done.
 * An upload that does not fit first evicts idle meshes (no queued or running
 * request), least recently used first. */
int m2s_server_submit_upload(m2s_server* server, const float* vertices, uint64_t n_vertices,
                             const void* indices, uint64_t n_indices, int index_bits, int topology,
                             int accel, int sign, uint32_t* mesh_id, uint64_t* ticket);
/* query_sdf on a resident mesh: out receives n_queries floats. */
int m2s_server_submit_points(m2s_server* server, uint32_t mesh_id, const float* query_points,
                             uint64_t n_queries, float* out, uint64_t* ticket);
/* generate_grid_sdf on a resident mesh: out receives the grid's cells. */
int m2s_server_submit_grid(m2s_server* server, uint32_t mesh_id, const float first_cell[3],
                           const float cell_size[3], const uint64_t cell_count[3], int sign,
                           float* out, uint64_t* ticket);
/* Waits for a ticket (timeout_s < 0: no limit; M2S_ERR_LIMIT if it is still
 * pending at the timeout, the ticket staying valid); *status receives the
 * request's status and *latency_s the time from submission to completion. */
int m2s_server_wait(m2s_server* server, uint64_t ticket, double timeout_s, int* status,
                    double* latency_s);
/* Frees a resident mesh that no queued or running request uses. */
int m2s_server_remove_mesh(m2s_server* server, uint32_t mesh_id);
/* [uploads, point requests, grid requests completed; failed; grid waves;
 *  grid requests in waves; most requests in one wave; reserved bytes; peak reserved bytes;
 *  resident meshes; queued requests; evicted meshes]. */
int m2s_server_stats(m2s_server* server, uint64_t out[12]);

/* ---- results for the viewer and on disk ----------------------------------- */

/* The voxel viewer's index buffer (mesh_to_sdf_client/src/sdf.rs:63-71): the
 * indices 0..n-1 stably sorted by f32::total_cmp of the distances, and the
 * (min, max) of the distances as its iso limits.  Device arrays, asynchronous
 * on `stream`; d_minmax (2 floats) may be NULL.  n < 2^32. */
int m2s_sort_cells_by_distance_device(const float* d_sdf, uint64_t n, uint32_t* d_order, float* d_minmax,
                                      void* stream);
/* The same from and into host memory (returns when done). */
int m2s_sort_cells_by_distance(const float* sdf, uint64_t n, uint32_t* order, float minmax[2], void* stream);

/* The crate's on-disk format V1 (serde.rs:106-221, rmp-serde encoding):
 * save_to_file writes these bytes, read_from_file reads them.  Host memory
 * only, no device needed.  With out = NULL, *out_len receives the size. */
int m2s_serialize_generic(const float* query_points, uint64_t n_points, const float* distances,
                          uint64_t n_distances, uint8_t* out, uint64_t capacity, uint64_t* out_len);
int m2s_serialize_grid(const float first_cell[3], const float cell_size[3], const uint64_t cell_count[3],
                       const float* distances, uint64_t n_distances, uint8_t* out, uint64_t capacity,
                       uint64_t* out_len);
/* *kind: 0 generic, 1 grid.  Call with NULL arrays to learn the counts, then
 * again with arrays of 3 * n_points and n_distances floats.  Malformed data:
 * M2S_ERR_FORMAT. */
int m2s_deserialize(const uint8_t* data, uint64_t len, int* kind, uint64_t* n_points, uint64_t* n_distances,
                    float* query_points, float* distances, float grid_first[3], float grid_size[3],
                    uint64_t grid_count[3]);

/* check_mesh_triangle_list (generate/mesh_check.rs:24-81) on the device, by
 * sorting (O(E log E); the crate's edge loop is O(E^2)), with the crate's
 * verdict and the crate's first reported failure: *result 0 = Ok; 1 = the
 * index count is not a multiple of 3; 2 = duplicate vertex (detail[0] = its
 * index); 3 = duplicate face (detail[0] = its face index); 4 = duplicate edge
 * detail[0] -> detail[1]; 5 = edge detail[0] -> detail[1] without a reverse
 * edge.  Host arrays; returns when done. */
int m2s_check_mesh_triangle_list(const float* vertices, uint64_t n_vertices, const uint32_t* faces,
                                 uint64_t n_face_indices, int* result, uint64_t detail[2], void* stream);

/* ---- utilities ----------------------------------------------------------- */

/* Stable LSD radix sort of (uint32 key, uint32 value) pairs on the device, the
 * sort behind the LBVH build; exposed so tests can compare it bit for bit with
 * a CPU stable sort.  Arrays are device pointers; results overwrite them. */
int m2s_radix_sort_pairs_device(uint32_t* d_keys, uint32_t* d_values, uint64_t n, int key_bits,
                                void* stream);

/* Diagnostics of the last grid call on this thread: [seed updates, relax
 * rounds, states relaxed, neighbour proposals (the on-grid cells of the 26
 * around each relaxed state; a proposal dropped unevaluated, see
 * m2s_last_grid_filter_stats, is counted too), ray hits, propagation
 * restarts, kernel launches, far-list redistributions, rounds relaxed by one
 * block alone, largest bucket list relaxed in one round]. */
int m2s_last_grid_stats(uint64_t out[10]);
/* Of the neighbour proposals of the last grid call on this thread: [dropped
 * because the neighbour already holds the proposing triangle, dropped by the
 * distance bound (m2s_set_grid_bound_filter)]; the rest were evaluated. */
int m2s_last_grid_filter_stats(uint64_t out[2]);

/* FP64 audit (no counterpart in the reference; a report, never a change of
 * output).  Results are the reference's f32 arithmetic, decision for
 * decision.  With enable != 0 (process-wide), grid calls and point queries
 * also check every aligned ray test (geo.rs:165-216) and the Voronoi-region
 * choice behind each result (geo.rs:97-128) against a forward-error bound of
 * the f32 arithmetic, and re-decide in FP64, on the device, only those whose
 * compared quantity lies within the bound.  Point queries run their counting
 * kernels then (as with m2s_set_profiling) and synchronise their stream.
 * m2s_last_grid_audit / m2s_last_query_audit read the last call's counts on
 * this thread: [ray tests, ambiguous ray tests, ray tests FP64 decides the
 * other way, cells / queries whose 2-of-3 vote the FP64 decisions flip,
 * cells / queries whose nearest triangle's region was audited (proper
 * triangles), ambiguous region choices, region choices FP64 makes
 * otherwise].  Point counts cover the LBVH methods (Bvh, Rtree, RtreeBvh). */
void m2s_set_fp64_audit(int enable);
int m2s_last_grid_audit(uint64_t out[7]);
int m2s_last_query_audit(uint64_t out[7]);

/* When enabled (per thread), grid calls time their phases with CUDA events on
 * their stream — the points the crate logs at generate/grid.rs:303-307,
 * 342-346 and 369-373 — readable with m2s_last_grid_phase_ms as
 * [seeding, propagation, rays, finalize] in milliseconds. */
void m2s_set_profiling(int enable);

/* Traversal counts of the last point query made on this thread with
 * profiling on (LBVH methods; no counterpart in the reference):
 * [queries, nearest-triangle search node fetches, search triangle tests,
 * sign-step node fetches, sign-step triangle tests].  The sign step is the
 * three axis rays (Bvh Raycast, RtreeBvh) or the Normal tie band (Bvh
 * Normal); Rtree has none.  Counting runs separate kernel instantiations and
 * reads the totals back, so a profiled query synchronises its stream. */
int m2s_last_query_stats(uint64_t out[5]);

/* Diagnostics of the grid propagation's barrier bound (no counterpart in the
 * reference): launches `blocks` blocks (1..64) that wait at one grid barrier
 * expecting `expected` blocks (1..64).  With blocks == expected all pass; with
 * fewer, every wait gives up after the barrier's two-second limit and raises
 * the abort flag, and the kernel returns.  out[0] = blocks that passed,
 * out[1] = blocks that gave up.  Synchronous. */
int m2s_test_grid_barrier(uint32_t blocks, uint32_t expected, uint32_t out[2]);
int m2s_last_grid_phase_ms(float out[4]);
/* With profiling on, the last grid call on this thread also records its
 * propagation steps in order, two words each: the step — the number of states
 * of a relaxed bucket list (bit 30 set when one block relaxed it alone), or
 * (bit 31 set) the number of far states of a redistribution, or 0xC0000000
 * for the end — and the nanoseconds from the kernel's start to the moment the
 * step was chosen.  Returns the number of steps recorded (at most 65,536),
 * copying up to `capacity` steps (2 * capacity words) to `out` (may be NULL). */
uint32_t m2s_last_grid_round_log(uint32_t* out, uint32_t capacity);

/* Point queries run one thread per query (from 2^19 queries the 32 queries of
 * a warp walk the tree together, the budget still counted per query); a
 * query that visits more than its node budget is continued by a whole warp
 * (points deep inside a closed mesh
 * see most triangles at nearly the same distance).  `node_visits` is the
 * budget of batches of 2^20 queries and more; a batch of nq queries from 2^18
 * uses node_visits * sqrt(nq / 2^20), and a smaller one node_visits / 16,
 * at least 64 either way, since a small batch's time is its longest
 * single-thread search.  0 keeps every query on one thread.
 * Bvh(Normal) hands searches and band folds over the budget to the warp pass
 * in batches under 2^18 queries, and at every size when node_visits is 64 or
 * less (a win on closed meshes with many deep-interior points, a loss on open
 * surfaces; the autotuner tries it).
 * Process-wide tuning knob; the autotuner sets it. */
void m2s_set_query_budget(uint32_t node_visits);
uint32_t m2s_query_budget(void);

/* The query autotuner (no counterpart in the reference): times the resident
 * mesh's LBVH query on the caller's device queries d_q[0..nq) with each
 * base budget of {0, 64, 256, 512, 1024, 1536, 2048, 4096} (see
 * m2s_set_query_budget: where a query moves from one thread to one warp,
 * scaled down for batches under 2^20 queries) and sets the fastest.  Results
 * do not depend on the budget.  Candidates are timed on this call alone:
 * queries running meanwhile on other threads keep the current budget, and if
 * another thread sets a budget while the tuner runs, that setting stands and
 * the tuner's choice is not published.  out_budget (may be NULL) receives the
 * choice, out_ms (may be NULL, 8 entries) each candidate's time.  Synchronous;
 * meshes built with AccelerationMethod::None have no traversal to tune
 * (M2S_ERR_INVALID_ARGUMENT). */
int m2s_query_autotune(const m2s_mesh* mesh, const float* d_q, uint64_t nq, void* stream, uint32_t* out_budget,
                       float out_ms[8]);

/* Diagnostics (no counterpart in the reference): [bytes in use, bytes
 * reserved] of this library's device-memory pool on the current device (both
 * 0 before the library's first allocation there).  Every allocating entry
 * point draws its workspace from this pool. */
int m2s_pool_usage(uint64_t out[2]);

const char* m2s_status_string(int status);
/* Detail of the last failure on the calling thread ("" if none). */
const char* m2s_last_error(void);
/* 1 if a CUDA device of compute capability 10.x is usable, else 0. */
int m2s_device_available(void);
int m2s_version(void);

#ifdef __cplusplus
}
#endif
#endif /* M2S_H */
