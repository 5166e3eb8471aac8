//! `mesh_to_sdf_cuda`: the public API of the `mesh_to_sdf` crate (0.4) —
//! `generate_sdf`, `generate_grid_sdf`, `build_sdf_acceleration` /
//! `query_sdf`, `query_vector_to_closest_point_rtree_bvh`,
//! `check_mesh_triangle_list` and their types — computed on an NVIDIA B200
//! by the library of this repository (include/m2s.h).
//!
//! NOT COMPILED HERE: the image this repository is built on has no Rust
//! toolchain.  The C ABI it binds is compiled and tested from C++
//! (tests/test_abi.py) and from Python (tests/).
//!
//! Item by item (paths in the reference crate `mesh_to_sdf/src/`):
//! * `Point`, `Grid`, `SnapResult` — re-exported from the original crate
//!   (`point.rs:22`, `grid.rs:10-173`): plain data and f32 arithmetic that the
//!   device code reproduces bit for bit.
//! * `Topology`, `OwnedTopology`, `SignMethod`, `AccelerationMethod`,
//!   `ALL_SDF_ACCELERATION_METHODS` — `lib.rs:156-296`, same variants, same
//!   derives.
//! * `SdfAccelerationMesh` and its four variant types — `lib.rs:303-312`;
//!   each variant holds a resident device mesh (an `m2s_mesh` handle).
//! * `generate_sdf` (`lib.rs:364-391`), `build_sdf_acceleration`
//!   (`lib.rs:410-433`), `query_sdf` (`lib.rs:463-485`),
//!   `generate_grid_sdf` (`generate/grid.rs:265-378`),
//!   `query_vector_to_closest_point_rtree_bvh` (`rtree_bvh.rs:217-276`),
//!   `check_mesh_triangle_list` (`generate/mesh_check.rs:24-81`).
//! * `serde` (feature "serde") — the original crate's module
//!   (`serde.rs`), re-exported.
//!
//! Where the crate panics, these functions panic too, with the library's
//! status message (a non-finite query point, an index list whose length is
//! not a multiple of 3, an index out of range, a NaN distance, an empty mesh
//! under `Rtree`).  Empty-mesh results follow the crate: `None` gives
//! `f32::MAX` per query, `RtreeBvh` an empty `Vec`, and
//! `build_sdf_acceleration(.., RtreeBvh)` on an empty mesh `None`.
use core::ffi::{c_int, c_void};
use core::marker::PhantomData;
use std::ffi::CStr;

pub mod ffi;

pub use mesh_to_sdf::{Grid, Point, SnapResult};

#[cfg(feature = "serde")]
pub use mesh_to_sdf::serde;

/// Mesh topology: how indices are stored (`lib.rs:156-171`).
#[derive(Copy, Clone)]
pub enum Topology<'a, I>
where
    I: Into<u32>,
{
    /// Every three indices (or vertices, without indices) form a triangle.
    TriangleList(Option<&'a [I]>),
    /// Every three adjacent indices (or vertices) form a triangle; windows are
    /// taken as they come, with no winding flip.
    TriangleStrip(Option<&'a [I]>),
}

/// Owned version of `Topology` (`lib.rs:177-186`).
#[derive(Clone)]
pub enum OwnedTopology<I>
where
    I: Into<u32>,
{
    OwnedTriangleList(Option<Vec<I>>),
    OwnedTriangleStrip(Option<Vec<I>>),
}

impl<I> OwnedTopology<I>
where
    I: Into<u32> + Copy + Sync + Send,
{
    fn as_topology(&self) -> Topology<I> {
        match self {
            Self::OwnedTriangleList(i) => Topology::TriangleList(i.as_deref()),
            Self::OwnedTriangleStrip(i) => Topology::TriangleStrip(i.as_deref()),
        }
    }
}

/// Sign method (`lib.rs:252-263`).
#[derive(Debug, Clone, Copy, Default, PartialEq, Eq, PartialOrd, Ord, Hash)]
pub enum SignMethod {
    /// Parity of the crossings of axis-aligned rays (the mesh must be watertight).
    #[default]
    Raycast,
    /// The sign of the nearest triangle's normal side.
    Normal,
}

/// Acceleration method (`lib.rs:272-286`).  On the device every method but
/// `None` runs on one LBVH built on the GPU; the names keep the crate's
/// semantics (`Rtree`: nearest triangle, normal sign; `RtreeBvh`: nearest
/// triangle, 3-ray vote; `Bvh(sign)`: the crate's candidate fold).
#[derive(Default, Debug, Clone, Copy, PartialEq, Eq, PartialOrd, Ord, Hash)]
pub enum AccelerationMethod {
    None(SignMethod),
    Bvh(SignMethod),
    Rtree,
    #[default]
    RtreeBvh,
}

/// Every acceleration method (`lib.rs:289-296`).
pub const ALL_SDF_ACCELERATION_METHODS: [AccelerationMethod; 6] = [
    AccelerationMethod::None(SignMethod::Raycast),
    AccelerationMethod::None(SignMethod::Normal),
    AccelerationMethod::Bvh(SignMethod::Raycast),
    AccelerationMethod::Bvh(SignMethod::Normal),
    AccelerationMethod::Rtree,
    AccelerationMethod::RtreeBvh,
];

// ---------------------------------------------------------------------------
// conversions to the C ABI

fn panic_on(status: c_int, what: &str) {
    if status != ffi::M2S_OK {
        let msg = unsafe { CStr::from_ptr(ffi::m2s_status_string(status)) }.to_string_lossy().into_owned();
        let detail = unsafe { CStr::from_ptr(ffi::m2s_last_error()) }.to_string_lossy().into_owned();
        if detail.is_empty() {
            panic!("{what}: {msg}");
        }
        panic!("{what}: {msg} ({detail})");
    }
}

/// The coordinates of points as one f32 array (no copy needed when `V` is
/// `[f32; 3]`, but `Point` is a trait, so the general path flattens).
fn flatten<V: Point>(points: &[V]) -> Vec<f32> {
    let mut out = Vec::with_capacity(3 * points.len());
    for p in points {
        out.extend_from_slice(&[p.x(), p.y(), p.z()]);
    }
    out
}

/// Index buffer of a topology, widened to u32 (`I: Into<u32>` covers u16 and
/// u32); (indices, index_bits, topology code).
fn indices<I: Copy + Into<u32>>(t: Topology<I>) -> (Option<Vec<u32>>, c_int, c_int) {
    let (slice, topo) = match t {
        Topology::TriangleList(s) => (s, ffi::M2S_TOPOLOGY_TRIANGLE_LIST),
        Topology::TriangleStrip(s) => (s, ffi::M2S_TOPOLOGY_TRIANGLE_STRIP),
    };
    match slice {
        Some(s) => (Some(s.iter().map(|x| (*x).into()).collect()), ffi::M2S_INDEX_U32, topo),
        None => (None, ffi::M2S_INDEX_NONE, topo),
    }
}

fn method_codes(m: AccelerationMethod) -> (c_int, c_int) {
    let sign = |s: SignMethod| if s == SignMethod::Raycast { ffi::M2S_SIGN_RAYCAST } else { ffi::M2S_SIGN_NORMAL };
    match m {
        AccelerationMethod::None(s) => (ffi::M2S_ACCEL_NONE, sign(s)),
        AccelerationMethod::Bvh(s) => (ffi::M2S_ACCEL_BVH, sign(s)),
        AccelerationMethod::Rtree => (ffi::M2S_ACCEL_RTREE, ffi::M2S_SIGN_NORMAL),
        AccelerationMethod::RtreeBvh => (ffi::M2S_ACCEL_RTREE_BVH, ffi::M2S_SIGN_RAYCAST),
    }
}

fn idx_ptr(i: &Option<Vec<u32>>) -> (*const c_void, u64) {
    match i {
        Some(v) => (v.as_ptr().cast(), v.len() as u64),
        None => (core::ptr::null(), 0),
    }
}

// ---------------------------------------------------------------------------
// generate_sdf / generate_grid_sdf

/// `generate_sdf` (`lib.rs:364-391`): signed distances of `query_points` to
/// the mesh, one per point (an empty `Vec` for `RtreeBvh` on an empty mesh).
pub fn generate_sdf<V, I>(vertices: &[V], indices: Topology<I>, query_points: &[V],
                          acceleration_method: AccelerationMethod) -> Vec<f32>
where
    V: Point + 'static,
    I: Copy + Into<u32> + Sync + Send,
{
    let v = flatten(vertices);
    let q = flatten(query_points);
    let (idx, bits, topo) = self::indices(indices);
    let (ip, ni) = idx_ptr(&idx);
    let (accel, sign) = method_codes(acceleration_method);
    let mut out = vec![0f32; query_points.len()];
    let mut n = 0u64;
    let st = unsafe {
        ffi::m2s_generate_sdf(v.as_ptr(), vertices.len() as u64, ip, ni, bits, topo, q.as_ptr(),
                              query_points.len() as u64, accel, sign, out.as_mut_ptr(), &mut n,
                              core::ptr::null_mut())
    };
    panic_on(st, "generate_sdf");
    out.truncate(n as usize);
    out
}

/// `generate_grid_sdf` (`generate/grid.rs:265-378`): one distance per cell of
/// `grid`, index = z + y * nz + x * ny * nz.
pub fn generate_grid_sdf<V, I>(vertices: &[V], indices: Topology<I>, grid: &Grid<V>,
                               sign_method: SignMethod) -> Vec<f32>
where
    V: Point + 'static,
    I: Copy + Into<u32> + Sync + Send,
{
    let v = flatten(vertices);
    let (idx, bits, topo) = self::indices(indices);
    let (ip, ni) = idx_ptr(&idx);
    let f = grid.get_first_cell();
    let s = grid.get_cell_size();
    let first = [f.x(), f.y(), f.z()];
    let size = [s.x(), s.y(), s.z()];
    let c = grid.get_cell_count();
    let count = [c[0] as u64, c[1] as u64, c[2] as u64];
    let sign = if sign_method == SignMethod::Raycast { ffi::M2S_SIGN_RAYCAST } else { ffi::M2S_SIGN_NORMAL };
    let mut out = vec![0f32; grid.get_total_cell_count()];
    let mut n = 0u64;
    let st = unsafe {
        ffi::m2s_generate_grid_sdf(v.as_ptr(), vertices.len() as u64, ip, ni, bits, topo, first.as_ptr(),
                                   size.as_ptr(), count.as_ptr(), sign, out.as_mut_ptr(), &mut n,
                                   core::ptr::null_mut())
    };
    panic_on(st, "generate_grid_sdf");
    out.truncate(n as usize);
    out
}

// ---------------------------------------------------------------------------
// resident meshes: build_sdf_acceleration / query_sdf

/// A resident device mesh (device copies of the triangles and, but for
/// `None`, the LBVH); freed on drop.  Immutable after build; queries from
/// several threads at once are safe.
struct Resident {
    handle: *mut ffi::m2s_mesh,
}
unsafe impl Send for Resident {}
unsafe impl Sync for Resident {}
impl Drop for Resident {
    fn drop(&mut self) {
        unsafe { ffi::m2s_mesh_free(self.handle) }
    }
}

/// The `None` variant (`generate/generic/default.rs:11`).
pub struct SdfAccelerationDefault<V: Point, I: Copy + Into<u32> + Sync + Send> {
    mesh: std::sync::Arc<Resident>,
    _types: PhantomData<(V, I)>,
}
/// The `Bvh` variant (`generate/generic/bvh.rs:52`).
pub struct SdfAccelerationBvh<V: Point> {
    mesh: std::sync::Arc<Resident>,
    _types: PhantomData<V>,
}
/// The `Rtree` variant (`generate/generic/rtree.rs:84`).
pub struct SdfAccelerationRtree<V: Point> {
    mesh: std::sync::Arc<Resident>,
    _types: PhantomData<V>,
}
/// The `RtreeBvh` variant (`generate/generic/rtree_bvh.rs:73`).
pub struct SdfAccelerationRtreeBvh<V: Point> {
    mesh: std::sync::Arc<Resident>,
    _types: PhantomData<V>,
}

macro_rules! clone_resident {
    ($t:ident < $($g:ident),* >) => {
        impl<V: Point, $($g: Copy + Into<u32> + Sync + Send),*> Clone for $t<V, $($g),*> {
            fn clone(&self) -> Self { Self { mesh: self.mesh.clone(), _types: PhantomData } }
        }
    };
    ($t:ident) => {
        impl<V: Point> Clone for $t<V> {
            fn clone(&self) -> Self { Self { mesh: self.mesh.clone(), _types: PhantomData } }
        }
    };
}
clone_resident!(SdfAccelerationDefault<I>);
clone_resident!(SdfAccelerationBvh);
clone_resident!(SdfAccelerationRtree);
clone_resident!(SdfAccelerationRtreeBvh);

/// `SdfAccelerationMesh` (`lib.rs:303-312`).
#[derive(Clone)]
pub enum SdfAccelerationMesh<V: Point, I: Copy + Into<u32> + Sync + Send> {
    None(SdfAccelerationDefault<V, I>),
    Bvh(SdfAccelerationBvh<V>),
    Rtree(SdfAccelerationRtree<V>),
    RtreeBvh(SdfAccelerationRtreeBvh<V>),
}

impl<V: Point, I: Copy + Into<u32> + Sync + Send> SdfAccelerationMesh<V, I> {
    fn handle(&self) -> *const ffi::m2s_mesh {
        match self {
            Self::None(a) => a.mesh.handle,
            Self::Bvh(a) => a.mesh.handle,
            Self::Rtree(a) => a.mesh.handle,
            Self::RtreeBvh(a) => a.mesh.handle,
        }
    }
}

/// `build_sdf_acceleration` (`lib.rs:410-433`): uploads the mesh and builds
/// its LBVH on the device.  `None` exactly where the crate returns `None`
/// (`RtreeBvh` on an empty mesh).
pub fn build_sdf_acceleration<V, I>(vertices: &[V], indices: Topology<I>,
                                    acceleration_method: AccelerationMethod)
                                    -> Option<SdfAccelerationMesh<V, I>>
where
    V: Point + 'static,
    I: Copy + Into<u32> + Sync + Send,
{
    let v = flatten(vertices);
    let (idx, bits, topo) = self::indices(indices);
    let (ip, ni) = idx_ptr(&idx);
    let (accel, sign) = method_codes(acceleration_method);
    let mut h: *mut ffi::m2s_mesh = core::ptr::null_mut();
    let st = unsafe {
        ffi::m2s_build_sdf_acceleration(v.as_ptr(), vertices.len() as u64, ip, ni, bits, topo, accel, sign, &mut h,
                                        core::ptr::null_mut())
    };
    panic_on(st, "build_sdf_acceleration");
    if h.is_null() {
        return None;
    }
    let mesh = std::sync::Arc::new(Resident { handle: h });
    Some(match acceleration_method {
        AccelerationMethod::None(_) => SdfAccelerationMesh::None(SdfAccelerationDefault { mesh, _types: PhantomData }),
        AccelerationMethod::Bvh(_) => SdfAccelerationMesh::Bvh(SdfAccelerationBvh { mesh, _types: PhantomData }),
        AccelerationMethod::Rtree => SdfAccelerationMesh::Rtree(SdfAccelerationRtree { mesh, _types: PhantomData }),
        AccelerationMethod::RtreeBvh => {
            SdfAccelerationMesh::RtreeBvh(SdfAccelerationRtreeBvh { mesh, _types: PhantomData })
        }
    })
}

/// `query_sdf` (`lib.rs:463-485`).  Unlike the crate, a non-finite query
/// point panics here too (the crate leaves the result unspecified).
pub fn query_sdf<V, I>(acceleration: &SdfAccelerationMesh<V, I>, query_points: &[V]) -> Vec<f32>
where
    V: Point + 'static,
    I: Copy + Into<u32> + Sync + Send,
{
    let q = flatten(query_points);
    let mut out = vec![0f32; query_points.len()];
    let mut n = 0u64;
    let st = unsafe {
        ffi::m2s_query_sdf(acceleration.handle(), q.as_ptr(), query_points.len() as u64, out.as_mut_ptr(), &mut n,
                           core::ptr::null_mut())
    };
    panic_on(st, "query_sdf");
    out.truncate(n as usize);
    out
}

/// `query_vector_to_closest_point_rtree_bvh` (`rtree_bvh.rs:217-276`): per
/// query point, the vector to the closest point on the nearest triangle and
/// whether the point is inside (3-ray vote).
pub fn query_vector_to_closest_point_rtree_bvh<V>(acceleration: &SdfAccelerationRtreeBvh<V>,
                                                  query_points: &[V]) -> Vec<(V, bool)>
where
    V: Point + 'static,
{
    let q = flatten(query_points);
    let mut vec = vec![0f32; 3 * query_points.len()];
    let mut inside = vec![0u8; query_points.len()];
    let mut n = 0u64;
    let st = unsafe {
        ffi::m2s_query_vector_to_closest_point(acceleration.mesh.handle, q.as_ptr(), query_points.len() as u64,
                                               vec.as_mut_ptr(), inside.as_mut_ptr(), &mut n, core::ptr::null_mut())
    };
    panic_on(st, "query_vector_to_closest_point_rtree_bvh");
    (0..n as usize).map(|k| (V::new(vec[3 * k], vec[3 * k + 1], vec[3 * k + 2]), inside[k] != 0)).collect()
}

// ---------------------------------------------------------------------------
// check_mesh_triangle_list

/// Face index types the device check takes: anything that widens to u32.
/// (The crate accepts any `Copy + Eq + Hash + Debug` index; its callers pass
/// u16, u32 or usize.)
pub trait FaceIndex: Copy + Eq + core::hash::Hash + core::fmt::Debug {
    fn to_u32(self) -> u32;
}
impl FaceIndex for u16 {
    fn to_u32(self) -> u32 { self as u32 }
}
impl FaceIndex for u32 {
    fn to_u32(self) -> u32 { self }
}
impl FaceIndex for usize {
    fn to_u32(self) -> u32 { u32::try_from(self).expect("face index above u32::MAX") }
}

/// `check_mesh_triangle_list` (`generate/mesh_check.rs:24-81`): the crate's
/// verdict and first reported failure, in the crate's words, computed on the
/// device by sorting.
pub fn check_mesh_triangle_list<V, U>(vertices: &[V], faces: &[U]) -> Result<(), String>
where
    V: Copy + Point,
    U: FaceIndex,
{
    let v = flatten(vertices);
    let f: Vec<u32> = faces.iter().map(|x| x.to_u32()).collect();
    let mut result: c_int = 0;
    let mut detail = [0u64; 2];
    let st = unsafe {
        ffi::m2s_check_mesh_triangle_list(v.as_ptr(), vertices.len() as u64, f.as_ptr(), f.len() as u64,
                                          &mut result, detail.as_mut_ptr(), core::ptr::null_mut())
    };
    panic_on(st, "check_mesh_triangle_list");
    // detail: the vertex (2), the face (3), or the edge's two vertex indices (4, 5)
    let (a, b) = (detail[0] as usize, detail[1] as usize);
    match result {
        0 => Ok(()),
        1 => Err("Faces must be a multiple of 3".to_string()),
        2 => {
            let p = vertices[a];
            Err(format!("Duplicate vertex found at ({:?}, {:?}, {:?})", p.x(), p.y(), p.z()))
        }
        3 => Err(format!("Duplicate face found: {:?}", faces[3 * a..3 * a + 3].to_vec())),
        4 => Err(format!("Duplicate edge {a:?} -> {b:?} - do you have an inverted normal?")),
        _ => Err(format!(
            "Mesh is not waterproof - edge {a:?} -> {b:?} does not have a corresponding edge {b:?} -> {a:?}"
        )),
    }
}

// Kept from the crate's surface: OwnedTopology is constructible and
// convertible, as in lib.rs:177-244.
impl<'a, I> Topology<'a, I>
where
    I: Into<u32> + Copy + Sync + Send,
{
    /// An owned copy of this topology.
    pub fn to_owned_topology(self) -> OwnedTopology<I> {
        match self {
            Topology::TriangleList(i) => OwnedTopology::OwnedTriangleList(i.map(|s| s.to_vec())),
            Topology::TriangleStrip(i) => OwnedTopology::OwnedTriangleStrip(i.map(|s| s.to_vec())),
        }
    }
}

impl<I> OwnedTopology<I>
where
    I: Into<u32> + Copy + Sync + Send,
{
    /// A borrowed view of this topology.
    pub fn topology(&self) -> Topology<I> {
        self.as_topology()
    }
}
