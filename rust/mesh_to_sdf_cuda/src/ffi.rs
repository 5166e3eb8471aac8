//! Raw bindings of include/m2s.h, one `extern "C"` item per declaration.
//! NOT COMPILED HERE: see Cargo.toml.
#![allow(non_camel_case_types)]

use core::ffi::{c_char, c_int, c_void};

pub const M2S_OK: c_int = 0;
pub const M2S_ERR_INVALID_ARGUMENT: c_int = 1;
pub const M2S_ERR_NONFINITE_QUERY: c_int = 2;
pub const M2S_ERR_INDEX_COUNT: c_int = 3;
pub const M2S_ERR_INDEX_RANGE: c_int = 4;
pub const M2S_ERR_NAN_DISTANCE: c_int = 5;
pub const M2S_ERR_EMPTY_MESH: c_int = 6;
pub const M2S_ERR_CUDA: c_int = 7;
pub const M2S_ERR_OUT_OF_MEMORY: c_int = 8;
pub const M2S_ERR_LIMIT: c_int = 9;
pub const M2S_ERR_NO_DEVICE: c_int = 10;
pub const M2S_ERR_FORMAT: c_int = 11;

pub const M2S_TOPOLOGY_TRIANGLE_LIST: c_int = 0;
pub const M2S_TOPOLOGY_TRIANGLE_STRIP: c_int = 1;
pub const M2S_INDEX_NONE: c_int = 0;
pub const M2S_INDEX_U16: c_int = 16;
pub const M2S_INDEX_U32: c_int = 32;
pub const M2S_SIGN_RAYCAST: c_int = 0;
pub const M2S_SIGN_NORMAL: c_int = 1;
pub const M2S_ACCEL_NONE: c_int = 0;
pub const M2S_ACCEL_BVH: c_int = 1;
pub const M2S_ACCEL_RTREE: c_int = 2;
pub const M2S_ACCEL_RTREE_BVH: c_int = 3;

#[repr(C)]
pub struct m2s_mesh {
    _private: [u8; 0],
}
#[repr(C)]
pub struct m2s_grid_plan {
    _private: [u8; 0],
}
#[repr(C)]
pub struct m2s_server {
    _private: [u8; 0],
}

extern "C" {
    // ---- the crate's entry points
    pub fn m2s_generate_sdf(vertices: *const f32, n_vertices: u64, indices: *const c_void, n_indices: u64,
                            index_bits: c_int, topology: c_int, query_points: *const f32, n_queries: u64,
                            accel: c_int, sign: c_int, out: *mut f32, out_len: *mut u64,
                            stream: *mut c_void) -> c_int;
    pub fn m2s_generate_grid_sdf(vertices: *const f32, n_vertices: u64, indices: *const c_void, n_indices: u64,
                                 index_bits: c_int, topology: c_int, first_cell: *const f32,
                                 cell_size: *const f32, cell_count: *const u64, sign: c_int, out: *mut f32,
                                 out_len: *mut u64, stream: *mut c_void) -> c_int;
    pub fn m2s_build_sdf_acceleration(vertices: *const f32, n_vertices: u64, indices: *const c_void,
                                      n_indices: u64, index_bits: c_int, topology: c_int, accel: c_int,
                                      sign: c_int, out_mesh: *mut *mut m2s_mesh, stream: *mut c_void) -> c_int;
    pub fn m2s_query_sdf(mesh: *const m2s_mesh, query_points: *const f32, n_queries: u64, out: *mut f32,
                         out_len: *mut u64, stream: *mut c_void) -> c_int;
    pub fn m2s_query_vector_to_closest_point(mesh: *const m2s_mesh, query_points: *const f32, n_queries: u64,
                                             out_vectors: *mut f32, out_inside: *mut u8, out_len: *mut u64,
                                             stream: *mut c_void) -> c_int;
    pub fn m2s_mesh_free(mesh: *mut m2s_mesh);
    pub fn m2s_mesh_triangle_count(mesh: *const m2s_mesh) -> u64;
    pub fn m2s_mesh_accel(mesh: *const m2s_mesh) -> c_int;

    // ---- device-resident variants
    pub fn m2s_query_sdf_device(mesh: *const m2s_mesh, d_query_points: *const f32, n_queries: u64,
                                d_out: *mut f32, d_status: *mut u32, stream: *mut c_void) -> c_int;
    pub fn m2s_grid_sdf_device(mesh: *const m2s_mesh, first_cell: *const f32, cell_size: *const f32,
                               cell_count: *const u64, sign: c_int, d_out: *mut f32, d_status: *mut u32,
                               stream: *mut c_void) -> c_int;

    // ---- batches of grids
    pub fn m2s_grid_sdf_batch_device(meshes: *const *const m2s_mesh, n_grids: u32, first_cells: *const f32,
                                     cell_sizes: *const f32, cell_counts: *const u64, sign: c_int,
                                     d_out: *mut f32, d_status: *mut u32, stream: *mut c_void) -> c_int;
    pub fn m2s_grid_plan_create(meshes: *const *const m2s_mesh, n_grids: u32, first_cells: *const f32,
                                cell_sizes: *const f32, cell_counts: *const u64, sign: c_int, d_out: *mut f32,
                                d_status: *mut u32, stream: *mut c_void, out_plan: *mut *mut m2s_grid_plan)
                                -> c_int;
    pub fn m2s_grid_plan_run(plan: *mut m2s_grid_plan, stream: *mut c_void) -> c_int;
    pub fn m2s_grid_plan_autotune(plan: *mut m2s_grid_plan, stream: *mut c_void, out_blocks: *mut u32) -> c_int;
    pub fn m2s_grid_plan_cells(plan: *const m2s_grid_plan) -> u64;
    pub fn m2s_grid_plan_device_bytes(plan: *const m2s_grid_plan) -> u64;
    pub fn m2s_grid_plan_blocks(plan: *const m2s_grid_plan) -> u32;
    pub fn m2s_grid_plan_waves(plan: *const m2s_grid_plan) -> u32;
    pub fn m2s_grid_plan_free(plan: *mut m2s_grid_plan);
    pub fn m2s_clear_grid_autotune();
    pub fn m2s_set_grid_tuning(blocks_per_sm: c_int, cells_per_block: u32, wave_cells: u64, solo_max: c_int);
    pub fn m2s_set_grid_bound_filter(enable: c_int);
    pub fn m2s_set_fp64_audit(enable: c_int);
    pub fn m2s_last_grid_audit(out: *mut u64) -> c_int;
    pub fn m2s_last_query_audit(out: *mut u64) -> c_int;

    // ---- callers that cannot allocate device memory
    pub fn m2s_generate_sdf_none_noalloc(d_vertices: *const f32, n_vertices: u64, d_indices: *const c_void,
                                         n_indices: u64, index_bits: c_int, topology: c_int,
                                         d_query_points: *const f32, n_queries: u64, sign: c_int,
                                         d_out: *mut f32, stream: *mut c_void) -> c_int;

    // ---- serving loop
    pub fn m2s_server_create(hbm_budget_bytes: u64, point_streams: u32, out: *mut *mut m2s_server) -> c_int;
    pub fn m2s_server_free(server: *mut m2s_server);
    pub fn m2s_server_submit_upload(server: *mut m2s_server, vertices: *const f32, n_vertices: u64,
                                    indices: *const c_void, n_indices: u64, index_bits: c_int, topology: c_int,
                                    accel: c_int, sign: c_int, mesh_id: *mut u32, ticket: *mut u64) -> c_int;
    pub fn m2s_server_submit_points(server: *mut m2s_server, mesh_id: u32, query_points: *const f32,
                                    n_queries: u64, out: *mut f32, ticket: *mut u64) -> c_int;
    pub fn m2s_server_submit_grid(server: *mut m2s_server, mesh_id: u32, first_cell: *const f32,
                                  cell_size: *const f32, cell_count: *const u64, sign: c_int, out: *mut f32,
                                  ticket: *mut u64) -> c_int;
    pub fn m2s_server_wait(server: *mut m2s_server, ticket: u64, timeout_s: f64, status: *mut c_int,
                           latency_s: *mut f64) -> c_int;
    pub fn m2s_server_remove_mesh(server: *mut m2s_server, mesh_id: u32) -> c_int;
    pub fn m2s_server_stats(server: *mut m2s_server, out: *mut u64) -> c_int;

    // ---- results for the viewer and on disk
    pub fn m2s_sort_cells_by_distance_device(d_sdf: *const f32, n: u64, d_order: *mut u32, d_minmax: *mut f32,
                                             stream: *mut c_void) -> c_int;
    pub fn m2s_sort_cells_by_distance(sdf: *const f32, n: u64, order: *mut u32, minmax: *mut f32,
                                      stream: *mut c_void) -> c_int;
    pub fn m2s_serialize_generic(query_points: *const f32, n_points: u64, distances: *const f32,
                                 n_distances: u64, out: *mut u8, capacity: u64, out_len: *mut u64) -> c_int;
    pub fn m2s_serialize_grid(first_cell: *const f32, cell_size: *const f32, cell_count: *const u64,
                              distances: *const f32, n_distances: u64, out: *mut u8, capacity: u64,
                              out_len: *mut u64) -> c_int;
    pub fn m2s_deserialize(data: *const u8, len: u64, kind: *mut c_int, n_points: *mut u64,
                           n_distances: *mut u64, query_points: *mut f32, distances: *mut f32,
                           grid_first: *mut f32, grid_size: *mut f32, grid_count: *mut u64) -> c_int;
    pub fn m2s_check_mesh_triangle_list(vertices: *const f32, n_vertices: u64, faces: *const u32,
                                        n_face_indices: u64, result: *mut c_int, detail: *mut u64,
                                        stream: *mut c_void) -> c_int;

    // ---- utilities and diagnostics
    pub fn m2s_radix_sort_pairs_device(d_keys: *mut u32, d_values: *mut u32, n: u64, key_bits: c_int,
                                       stream: *mut c_void) -> c_int;
    pub fn m2s_last_grid_stats(out: *mut u64) -> c_int;
    pub fn m2s_last_grid_filter_stats(out: *mut u64) -> c_int;
    pub fn m2s_set_profiling(enable: c_int);
    pub fn m2s_last_query_stats(out: *mut u64) -> c_int;
    pub fn m2s_test_grid_barrier(blocks: u32, expected: u32, out: *mut u32) -> c_int;
    pub fn m2s_last_grid_phase_ms(out: *mut f32) -> c_int;
    pub fn m2s_last_grid_round_log(out: *mut u32, capacity: u32) -> u32;
    pub fn m2s_set_query_budget(node_visits: u32);
    pub fn m2s_query_budget() -> u32;
    pub fn m2s_query_autotune(mesh: *const m2s_mesh, d_q: *const f32, nq: u64, stream: *mut c_void,
                              out_budget: *mut u32, out_ms: *mut f32) -> c_int;
    pub fn m2s_pool_usage(out: *mut u64) -> c_int;
    pub fn m2s_status_string(status: c_int) -> *const c_char;
    pub fn m2s_last_error() -> *const c_char;
    pub fn m2s_device_available() -> c_int;
    pub fn m2s_version() -> c_int;
}
