/* C ABI of the CPU oracle (test infrastructure only).
 *
 * liboracle restates the Rust crate `mesh_to_sdf` on the CPU.  It is the
 * checker for the CUDA library and the timed CPU baseline; the shipped library
 * never links or calls it.  Status codes are the same numbers as include/m2s.h.
 *
 * Ordering semantics that the reference leaves to third-party crates (the
 * bvh crate's candidate order for Bvh+Normal, rstar's choice among exactly tied
 * nearest triangles) are pinned here to "lowest triangle index first"; the
 * reference's own choice there is not observable from this container, so those
 * two cases are parity-unpinned and the tests count them separately.
 */
#ifndef M2S_ORACLE_H
#define M2S_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Geometry primitives (geo.rs). p/a/b/c/out are float[3]. */
void orc_closest_point_triangle(const float* p, const float* a, const float* b, const float* c,
                                float* out);
float orc_point_triangle_distance(const float* p, const float* a, const float* b, const float* c);
float orc_point_triangle_distance2(const float* p, const float* a, const float* b, const float* c);
float orc_point_triangle_signed_distance(const float* p, const float* a, const float* b,
                                         const float* c);
/* returns 1 and writes *t on a hit (t > 0), else 0 */
int orc_ray_triangle_intersection_aligned(const float* o, const float* a, const float* b,
                                          const float* c, int axis, float* t);
void orc_triangle_bounding_box(const float* a, const float* b, const float* c, float* mn,
                               float* mx);
/* -1 Less, 0 Equal, 1 Greater, 2 = the reference would panic (NaN) */
int orc_compare_distances(float a, float b);

/* Topology::get_triangles (lib.rs:193-215).  index_bits: 0 = no index buffer,
 * 16 = uint16, 32 = uint32.  topology: 0 = TriangleList, 1 = TriangleStrip.
 * Writes 3*n_tris uint32 into tris_out (may be NULL to just count) and returns a
 * status; *n_tris receives the triangle count. */
int orc_expand_topology(uint64_t n_vertices, const void* indices, uint64_t n_indices,
                        int index_bits, int topology, uint32_t* tris_out, uint64_t* n_tris);

/* generate_sdf (lib.rs:364-391).  accel: 0 None, 1 Bvh, 2 Rtree, 3 RtreeBvh.
 * sign: 0 Raycast, 1 Normal (ignored for Rtree/RtreeBvh).  out holds n_queries
 * floats; *out_len is n_queries, or 0 when the reference returns an empty Vec
 * (RtreeBvh on an empty mesh).  n_threads <= 0 uses every core. */
int orc_generate_sdf(const float* vertices, uint64_t n_vertices, const void* indices,
                     uint64_t n_indices, int index_bits, int topology, const float* queries,
                     uint64_t n_queries, int accel, int sign, float* out, uint64_t* out_len,
                     int n_threads);

/* query_vector_to_closest_point_rtree_bvh (rtree_bvh.rs:217-276): out_vec gets
 * 3 floats per query (closest - p), out_inside one byte per query. */
int orc_query_vector_to_closest_point(const float* vertices, uint64_t n_vertices,
                                      const void* indices, uint64_t n_indices, int index_bits,
                                      int topology, const float* queries, uint64_t n_queries,
                                      float* out_vec, uint8_t* out_inside, uint64_t* out_len,
                                      int n_threads);

/* generate_grid_sdf (generate/grid.rs:265-378).  n_threads = 1 is the
 * deterministic single-heap run; n_threads > 1 splits the heap round-robin
 * across threads exactly like the reference (grid.rs:318-339) and is as
 * order-dependent as the reference itself.  stats (may be NULL) receives
 * [seed updates, heap pops, rays cast, ray hits]. */
int orc_generate_grid_sdf(const float* vertices, uint64_t n_vertices, const void* indices,
                          uint64_t n_indices, int index_bits, int topology,
                          const float* first_cell, const float* cell_size,
                          const uint64_t* cell_count, int sign, float* out, uint64_t* out_len,
                          int n_threads, uint64_t* stats);

/* FP64 brute force: exact-as-double unsigned distance to the mesh and the
 * 3-axis ray vote evaluated in double.  Used for max/RMS error reports only. */
int orc_generate_sdf_f64(const float* vertices, uint64_t n_vertices, const void* indices,
                         uint64_t n_indices, int index_bits, int topology, const float* queries,
                         uint64_t n_queries, double* out_unsigned, uint8_t* out_inside_vote,
                         int n_threads);

/* Grid helpers (grid.rs). */
void orc_grid_from_bounding_box(const float* bbox_min, const float* bbox_max,
                                const uint64_t* cell_count, float* first_cell, float* cell_size);
void orc_grid_cell_center(const float* first_cell, const float* cell_size, const uint64_t* cell,
                          float* out);
/* returns 1 for SnapResult::Inside, 0 for Outside; cell_out gets the cell */
int orc_grid_snap_point(const float* first_cell, const float* cell_size,
                        const uint64_t* cell_count, const float* p, uint64_t* cell_out);

/* check_mesh_triangle_list (generate/mesh_check.rs:24-81): kind 0 ok, 1 length
 * not a multiple of 3, 2 duplicate vertex (detail[0]), 3 duplicate face
 * (detail[0]), 4 duplicate edge, 5 edge without its reverse (detail[0] ->
 * detail[1]). */
int orc_check_mesh_triangle_list(const float* vertices, uint64_t n_vertices, const uint32_t* faces,
                                 uint64_t n_face_indices, int* kind, uint64_t* detail);

#ifdef __cplusplus
}
#endif
#endif
