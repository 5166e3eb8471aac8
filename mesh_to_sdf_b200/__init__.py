"""mesh_to_sdf_b200 — signed distance fields from triangle meshes on NVIDIA B200.

A drop-in for the two entry points of the Rust crate ``mesh_to_sdf``
(``generate_sdf`` and ``generate_grid_sdf``) plus its resident-mesh API
(``build_sdf_acceleration`` / ``query_sdf``), computed by hand-written CUDA
kernels for sm_100a behind the C ABI of ``include/m2s.h``.  Names, arguments
and error behaviour follow the crate (file:line citations are to
``mesh_to_sdf/src/``); where the crate panics, this module raises
:class:`M2SError` carrying the C status code.

There is no CPU implementation here: every compute call runs on the GPU and
fails loudly when ``libm2s.so`` or an sm_100 device is missing.
"""
from __future__ import annotations

import ctypes
import enum
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _lib

__all__ = [
    "SignMethod", "AccelerationMethod", "Topology", "Grid", "SnapResult", "SdfAccelerationMesh", "M2SError",
    "generate_sdf", "generate_grid_sdf", "build_sdf_acceleration", "query_sdf",
    "query_vector_to_closest_point_rtree_bvh", "ALL_SDF_ACCELERATION_METHODS", "device_available",
    "grid_sdf_batch_device", "GridPlan", "grid_offsets", "set_grid_tuning", "set_grid_bound_filter", "set_fp64_audit", "last_grid_audit", "last_query_audit", "clear_grid_autotune", "Server",
    "sort_cells_by_distance", "sort_cells_by_distance_device", "check_mesh_triangle_list",
]

F32 = np.float32

STATUS = {
    0: "OK", 1: "INVALID_ARGUMENT", 2: "NONFINITE_QUERY", 3: "INDEX_COUNT", 4: "INDEX_RANGE",
    5: "NAN_DISTANCE", 6: "EMPTY_MESH", 7: "CUDA", 8: "OUT_OF_MEMORY", 9: "LIMIT", 10: "NO_DEVICE", 11: "FORMAT",
}


class M2SError(RuntimeError):
    """A non-zero status from the C ABI (the crate panics in these cases)."""

    def __init__(self, status: int, what: str):
        L = _lib.lib()
        detail = (L.m2s_last_error() or b"").decode(errors="replace")
        msg = (L.m2s_status_string(status) or b"").decode()
        super().__init__(f"{what}: {STATUS.get(status, status)} ({msg}){' — ' + detail if detail else ''}")
        self.status = status


def _check(st: int, what: str):
    if st != 0:
        raise M2SError(st, what)


class SignMethod(enum.IntEnum):
    """lib.rs:252-263."""
    Raycast = 0
    Normal = 1


@dataclass(frozen=True)
class AccelerationMethod:
    """lib.rs:272-286: None(sign), Bvh(sign), Rtree, RtreeBvh (the default)."""
    kind: int
    sign: SignMethod = SignMethod.Raycast

    NONE = 0
    BVH = 1
    RTREE = 2
    RTREE_BVH = 3

    @classmethod
    def none(cls, sign: SignMethod = SignMethod.Raycast):
        return cls(cls.NONE, SignMethod(sign))

    @classmethod
    def bvh(cls, sign: SignMethod = SignMethod.Raycast):
        return cls(cls.BVH, SignMethod(sign))

    @classmethod
    def rtree(cls):
        return cls(cls.RTREE, SignMethod.Normal)

    @classmethod
    def rtree_bvh(cls):
        return cls(cls.RTREE_BVH, SignMethod.Raycast)

    @classmethod
    def default(cls):
        return cls.rtree_bvh()

    def __repr__(self):
        name = {0: "None", 1: "Bvh", 2: "Rtree", 3: "RtreeBvh"}[self.kind]
        return f"AccelerationMethod.{name}({self.sign.name})" if self.kind in (0, 1) else f"AccelerationMethod.{name}"


# lib.rs:289-296
ALL_SDF_ACCELERATION_METHODS = (
    AccelerationMethod.none(SignMethod.Raycast), AccelerationMethod.none(SignMethod.Normal),
    AccelerationMethod.bvh(SignMethod.Raycast), AccelerationMethod.bvh(SignMethod.Normal),
    AccelerationMethod.rtree(), AccelerationMethod.rtree_bvh(),
)


@dataclass(frozen=True)
class Topology:
    """lib.rs:156-171: TriangleList(Option<&[I]>) / TriangleStrip(Option<&[I]>), I = u16 or u32."""
    strip: bool
    indices: Optional[np.ndarray] = None

    @classmethod
    def TriangleList(cls, indices=None):
        return cls(False, None if indices is None else np.asarray(indices))

    @classmethod
    def TriangleStrip(cls, indices=None):
        return cls(True, None if indices is None else np.asarray(indices))

    def _ffi(self):
        """(pointer-owner array or None, n_indices, index_bits, topology code)."""
        if self.indices is None:
            return None, 0, 0, int(self.strip)
        idx = self.indices
        if idx.dtype == np.uint16:
            arr, bits = np.ascontiguousarray(idx.reshape(-1)), 16
        else:
            if idx.size and (idx.min() < 0 or idx.max() > 0xFFFFFFFF):
                raise ValueError("indices must fit in u32")
            arr, bits = np.ascontiguousarray(idx.reshape(-1).astype(np.uint32)), 32
        return arr, len(arr), bits, int(self.strip)


@dataclass(frozen=True)
class SnapResult:
    """grid.rs:10-17."""
    inside: bool
    cell: tuple

    @classmethod
    def Inside(cls, cell):
        return cls(True, tuple(int(c) for c in cell))

    @classmethod
    def Outside(cls, cell):
        return cls(False, tuple(int(c) for c in cell))


class Grid:
    """grid.rs:30-173.  All arithmetic is float32, in the crate's operation order."""

    def __init__(self, first_cell, cell_size, cell_count):
        self.first_cell = np.asarray(first_cell, F32).reshape(3).copy()
        self.cell_size = np.asarray(cell_size, F32).reshape(3).copy()
        self.cell_count = tuple(int(c) for c in cell_count)
        if any(c < 0 for c in self.cell_count):
            raise ValueError("cell counts must be non-negative")

    @classmethod
    def new(cls, first_cell, cell_size, cell_count):
        return cls(first_cell, cell_size, cell_count)

    @classmethod
    def from_bounding_box(cls, bbox_min, bbox_max, cell_count):
        # grid.rs:59-74
        mn = np.asarray(bbox_min, F32).reshape(3)
        mx = np.asarray(bbox_max, F32).reshape(3)
        fc = np.array([F32(c) for c in cell_count], F32)
        size = ((mx - mn).astype(F32) / fc).astype(F32)
        first = (mn + (size * F32(0.5)).astype(F32)).astype(F32)
        return cls(first, size, cell_count)

    def get_first_cell(self):
        return self.first_cell.copy()

    def get_last_cell(self):
        # grid.rs:82-88
        n = np.array(self.cell_count, F32)
        return (self.first_cell + (n * self.cell_size).astype(F32)).astype(F32)

    def get_cell_size(self):
        return self.cell_size.copy()

    def get_cell_count(self):
        return list(self.cell_count)

    def get_total_cell_count(self):
        return self.cell_count[0] * self.cell_count[1] * self.cell_count[2]

    def get_bounding_box(self):
        # grid.rs:110-119
        mn = (self.first_cell - (self.cell_size * F32(0.5)).astype(F32)).astype(F32)
        n = np.array(self.cell_count, F32)
        mx = (mn + (n * self.cell_size).astype(F32)).astype(F32)
        return mn, mx

    def get_cell_idx(self, cell):
        # grid.rs:122-124 (z fastest)
        return int(cell[2]) + int(cell[1]) * self.cell_count[2] + int(cell[0]) * self.cell_count[1] * self.cell_count[2]

    def get_cell_integer_coordinates(self, idx):
        # grid.rs:127-132
        nz, ny = self.cell_count[2], self.cell_count[1]
        return [idx // (ny * nz), (idx // nz) % ny, idx % nz]

    def get_cell_center(self, cell):
        # grid.rs:135-141
        c = np.array([F32(int(x)) for x in cell], F32)
        return (self.first_cell + (c * self.cell_size).astype(F32)).astype(F32)

    def cell_centers(self):
        """All cell centres, (n, 3) float32, in output order."""
        nx, ny, nz = self.cell_count
        ix, iy, iz = np.meshgrid(np.arange(nx, dtype=F32), np.arange(ny, dtype=F32), np.arange(nz, dtype=F32),
                                 indexing="ij")
        c = np.stack([ix, iy, iz], -1).reshape(-1, 3)
        return (self.first_cell + (c * self.cell_size).astype(F32)).astype(F32)

    def snap_point_to_grid(self, point):
        # grid.rs:145-170
        p = np.asarray(point, F32).reshape(3)
        rel = ((p - self.get_bounding_box()[0]).astype(F32) / self.cell_size).astype(F32)
        out, inside = [], True
        for d in range(3):
            f = float(np.floor(rel[d]))
            c = 0 if np.isnan(f) else int(max(min(f, 9.2e18), -9.2e18))
            cl = min(max(c, 0), self.cell_count[d] - 1)
            inside &= cl == c
            out.append(cl)
        return SnapResult.Inside(out) if inside else SnapResult.Outside(out)

    def __repr__(self):
        return f"Grid(first_cell={self.first_cell.tolist()}, cell_size={self.cell_size.tolist()}, " \
               f"cell_count={list(self.cell_count)})"


def _points(x, what="points"):
    a = np.ascontiguousarray(np.asarray(x, dtype=F32).reshape(-1, 3))
    return a


def _vp(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def device_available() -> bool:
    return bool(_lib.lib().m2s_device_available())


def generate_sdf(vertices, indices: Topology, query_points, acceleration_method: AccelerationMethod = None):
    """lib.rs:364-391: signed distance of every query point (positive outside)."""
    am = acceleration_method or AccelerationMethod.default()
    v = _points(vertices)
    q = _points(query_points)
    idx, ni, bits, topo = indices._ffi()
    out = np.empty(len(q), F32)
    n = ctypes.c_uint64(0)
    st = _lib.lib().m2s_generate_sdf(_vp(v), len(v), _vp(idx), ni, bits, topo, _vp(q), len(q), am.kind,
                                     int(am.sign), _vp(out), ctypes.byref(n), None)
    _check(st, "generate_sdf")
    return out[: n.value]


def generate_grid_sdf(vertices, indices: Topology, grid: Grid, sign_method: SignMethod = SignMethod.Raycast):
    """generate/grid.rs:265-378: signed distances of every cell centre, z fastest."""
    v = _points(vertices)
    idx, ni, bits, topo = indices._ffi()
    first = np.ascontiguousarray(grid.first_cell, F32)
    size = np.ascontiguousarray(grid.cell_size, F32)
    count = np.ascontiguousarray(np.array(grid.cell_count, np.uint64))
    out = np.empty(grid.get_total_cell_count(), F32)
    n = ctypes.c_uint64(0)
    st = _lib.lib().m2s_generate_grid_sdf(_vp(v), len(v), _vp(idx), ni, bits, topo, _vp(first), _vp(size),
                                          _vp(count), int(sign_method), _vp(out), ctypes.byref(n), None)
    _check(st, "generate_grid_sdf")
    return out[: n.value]


GRID_STATS = ("seed_updates", "rounds", "states_relaxed", "neighbour_evals", "ray_hits", "restarts",
              "kernel_launches", "far_phases", "solo_rounds", "max_list")


def last_grid_stats():
    """Counters of the last grid call on this thread (names in GRID_STATS),
    plus how many neighbour proposals were dropped unevaluated: `dropped_same`
    (the neighbour held the proposing triangle) and `dropped_bound` (the
    distance bound proved they cannot win)."""
    L = _lib.lib()
    a = np.zeros(len(GRID_STATS), np.uint64)
    L.m2s_last_grid_stats(_vp(a))
    d = dict(zip(GRID_STATS, (int(x) for x in a)))
    f = np.zeros(2, np.uint64)
    L.m2s_last_grid_filter_stats(_vp(f))
    d["dropped_same"], d["dropped_bound"] = int(f[0]), int(f[1])
    return d


AUDIT_STATS = ("ray_tests", "ray_ambiguous", "ray_fp64_disagrees", "vote_flips", "regions", "region_ambiguous",
               "region_fp64_disagrees")


def set_fp64_audit(enable: bool):
    """Process-wide: audit every f32 ray test and Voronoi-region choice against
    a forward-error bound and re-decide the ambiguous ones in FP64 on the
    device (counts only; results do not change).  See last_grid_audit() and
    last_query_audit()."""
    _lib.lib().m2s_set_fp64_audit(1 if enable else 0)


def last_grid_audit():
    """The FP64 audit counts of the last grid call on this thread (names in AUDIT_STATS)."""
    a = np.zeros(len(AUDIT_STATS), np.uint64)
    _lib.lib().m2s_last_grid_audit(_vp(a))
    return dict(zip(AUDIT_STATS, (int(x) for x in a)))


def last_query_audit():
    """The FP64 audit counts of the last point query on this thread (names in AUDIT_STATS)."""
    a = np.zeros(len(AUDIT_STATS), np.uint64)
    _lib.lib().m2s_last_query_audit(_vp(a))
    return dict(zip(AUDIT_STATS, (int(x) for x in a)))


def set_grid_bound_filter(enable: bool):
    """Process-wide: run grid propagation's filtered variant, which drops the
    proposals a per-triangle distance bound proves cannot win before their
    evaluation (off by default).  Results are identical either way."""
    _lib.lib().m2s_set_grid_bound_filter(1 if enable else 0)


QUERY_STATS = ("queries", "search_node_fetches", "search_triangle_tests", "sign_node_fetches", "sign_triangle_tests")


def last_query_stats():
    """With profiling on (set_profiling): traversal counts of the last point
    query on this thread (names in QUERY_STATS), plus per-query averages."""
    a = np.zeros(len(QUERY_STATS), np.uint64)
    _lib.lib().m2s_last_query_stats(_vp(a))
    d = dict(zip(QUERY_STATS, (int(x) for x in a)))
    n = max(d["queries"], 1)
    for k in QUERY_STATS[1:]:
        d[k + "_per_query"] = d[k] / n
    return d


def last_grid_round_log():
    """With profiling on: the last grid call's propagation steps in order, as
    (kind, size, t_ns) rows — kind 0 a relax round on every block, 2 a relax
    round on one block, 1 a far-list redistribution, 3 the end; size in states;
    t_ns the time from the kernel's start at which the step was chosen."""
    L = _lib.lib()
    n = int(L.m2s_last_grid_round_log(None, 0))
    a = np.zeros(2 * n, np.uint32)
    if n:
        L.m2s_last_grid_round_log(_vp(a), n)
    v, t = a[0::2], a[1::2]
    kind = np.where(v >> 31, np.where((v >> 30) & 1, 3, 1), np.where((v >> 30) & 1, 2, 0))
    return np.stack([kind.astype(np.int64), (v & 0x3FFFFFFF).astype(np.int64), t.astype(np.int64)], 1)


def set_profiling(enable: bool):
    """Time grid phases with CUDA events (per thread); see last_grid_phase_ms()."""
    _lib.lib().m2s_set_profiling(1 if enable else 0)


def last_grid_phase_ms():
    """{seeding, propagation, rays, finalize} device milliseconds of the last profiled grid call."""
    a = np.zeros(4, np.float32)
    _lib.lib().m2s_last_grid_phase_ms(_vp(a))
    return dict(zip(("seeding", "propagation", "rays", "finalize"), (float(x) for x in a)))


class SdfAccelerationMesh:
    """lib.rs:303-312: a mesh and its LBVH resident in HBM (owns an m2s_mesh*)."""

    def __init__(self, handle, method: AccelerationMethod):
        self._h = ctypes.c_void_p(handle)
        self.method = method

    @property
    def handle(self):
        return self._h

    @property
    def triangle_count(self):
        return int(_lib.lib().m2s_mesh_triangle_count(self._h))

    def close(self):
        if self._h and self._h.value:
            _lib.lib().m2s_mesh_free(self._h)
            self._h = ctypes.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- device-resident variants (torch tensors on cuda) -----------------
    def query_device(self, q, out, status=None, stream=None):
        """query_sdf on device tensors: q (n,3) float32, out (n,) float32; asynchronous."""
        st = _lib.lib().m2s_query_sdf_device(self._h, ctypes.c_void_p(q.data_ptr()), q.shape[0],
                                             ctypes.c_void_p(out.data_ptr()),
                                             None if status is None else ctypes.c_void_p(status.data_ptr()),
                                             None if stream is None else ctypes.c_void_p(stream))
        _check(st, "query_sdf_device")

    QUERY_BUDGETS = (0, 64, 256, 512, 1024, 1536, 2048, 4096)

    def autotune_queries(self, q, stream=None):
        """The query autotuner: times this mesh's query on the device tensor q
        (n,3) float32 at each node budget of QUERY_BUDGETS (where a query moves
        from one thread to one warp), sets the process-wide budget to the
        fastest and returns (budget, {budget: ms}).  Results do not depend on
        the budget."""
        b = ctypes.c_uint32(0)
        ms = np.zeros(len(self.QUERY_BUDGETS), np.float32)
        st = _lib.lib().m2s_query_autotune(self._h, ctypes.c_void_p(q.data_ptr()), q.shape[0],
                                           None if stream is None else ctypes.c_void_p(stream), ctypes.byref(b),
                                           _vp(ms))
        _check(st, "query_autotune")
        return int(b.value), {k: float(v) for k, v in zip(self.QUERY_BUDGETS, ms)}

    def grid_device(self, grid: Grid, sign_method: SignMethod, out, status=None, stream=None):
        """generate_grid_sdf into a device tensor `out` of grid.get_total_cell_count() float32."""
        first = np.ascontiguousarray(grid.first_cell, F32)
        size = np.ascontiguousarray(grid.cell_size, F32)
        count = np.ascontiguousarray(np.array(grid.cell_count, np.uint64))
        st = _lib.lib().m2s_grid_sdf_device(self._h, _vp(first), _vp(size), _vp(count), int(sign_method),
                                            ctypes.c_void_p(out.data_ptr()),
                                            None if status is None else ctypes.c_void_p(status.data_ptr()),
                                            None if stream is None else ctypes.c_void_p(stream))
        _check(st, "grid_sdf_device")


def build_sdf_acceleration(vertices, indices: Topology, acceleration_method: AccelerationMethod = None):
    """lib.rs:410-433; returns None where the crate does (RtreeBvh on an empty mesh)."""
    am = acceleration_method or AccelerationMethod.default()
    v = _points(vertices)
    idx, ni, bits, topo = indices._ffi()
    h = ctypes.c_void_p(None)
    st = _lib.lib().m2s_build_sdf_acceleration(_vp(v), len(v), _vp(idx), ni, bits, topo, am.kind, int(am.sign),
                                               ctypes.byref(h), None)
    _check(st, "build_sdf_acceleration")
    if not h.value:
        return None
    return SdfAccelerationMesh(h.value, am)


def query_sdf(acceleration: SdfAccelerationMesh, query_points):
    """lib.rs:463-485."""
    q = _points(query_points)
    out = np.empty(len(q), F32)
    n = ctypes.c_uint64(0)
    st = _lib.lib().m2s_query_sdf(acceleration.handle, _vp(q), len(q), _vp(out), ctypes.byref(n), None)
    _check(st, "query_sdf")
    return out[: n.value]


def query_vector_to_closest_point_rtree_bvh(acceleration: SdfAccelerationMesh, query_points):
    """rtree_bvh.rs:217-276: (closest point - query, inside) per query."""
    q = _points(query_points)
    vec = np.empty((len(q), 3), F32)
    inside = np.empty(len(q), np.uint8)
    n = ctypes.c_uint64(0)
    st = _lib.lib().m2s_query_vector_to_closest_point(acceleration.handle, _vp(q), len(q), _vp(vec), _vp(inside),
                                                      ctypes.byref(n), None)
    _check(st, "query_vector_to_closest_point_rtree_bvh")
    return vec[: n.value], inside[: n.value].astype(bool)


# ---- batches of grids (no counterpart in the crate) ---------------------------

def _grid_batch_args(meshes, grids):
    if len(meshes) != len(grids) or not grids:
        raise ValueError("one grid per mesh, at least one")
    handles = (ctypes.c_void_p * len(meshes))(*[m.handle.value for m in meshes])
    first = np.ascontiguousarray(np.array([g.first_cell for g in grids], F32).reshape(-1))
    size = np.ascontiguousarray(np.array([g.cell_size for g in grids], F32).reshape(-1))
    count = np.ascontiguousarray(np.array([g.cell_count for g in grids], np.uint64).reshape(-1))
    return handles, first, size, count


def grid_offsets(grids):
    """Start of each grid's cells in a batch output, and the total."""
    sizes = [int(g.get_total_cell_count()) for g in grids]
    return np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)


def grid_sdf_batch_device(meshes, grids, sign_method: SignMethod, out, status=None, stream=None):
    """Grid SDFs of (meshes[k], grids[k]) pairs in one job, into the device
    tensor `out` (the grids' cells back to back, in order, see grid_offsets).
    Every grid's values are bit-identical to SdfAccelerationMesh.grid_device on
    that mesh and grid alone; the job runs as many propagation rounds as its
    slowest grid instead of their sum."""
    handles, first, size, count = _grid_batch_args(meshes, grids)
    st = _lib.lib().m2s_grid_sdf_batch_device(handles, len(grids), _vp(first), _vp(size), _vp(count),
                                              int(sign_method), ctypes.c_void_p(out.data_ptr()),
                                              None if status is None else ctypes.c_void_p(status.data_ptr()),
                                              None if stream is None else ctypes.c_void_p(stream))
    _check(st, "grid_sdf_batch_device")


class GridPlan:
    """A batch of grids captured once into a CUDA graph and replayed with run().
    The meshes and the device tensors `out` (float32, all cells) and `status`
    (uint32, cleared by the caller) stay bound to the plan."""

    def __init__(self, meshes, grids, sign_method: SignMethod, out, status):
        handles, first, size, count = _grid_batch_args(meshes, grids)
        self._keep = (list(meshes), out, status)
        h = ctypes.c_void_p(None)
        st = _lib.lib().m2s_grid_plan_create(handles, len(grids), _vp(first), _vp(size), _vp(count),
                                             int(sign_method), ctypes.c_void_p(out.data_ptr()),
                                             ctypes.c_void_p(status.data_ptr()), None, ctypes.byref(h))
        _check(st, "grid_plan_create")
        self._h = h

    def run(self, stream=None):
        _check(_lib.lib().m2s_grid_plan_run(self._h, None if stream is None else ctypes.c_void_p(stream)),
               "grid_plan_run")

    def autotune(self, stream=None):
        """Picks the fastest cooperative grid size for this plan; returns it."""
        b = ctypes.c_uint32(0)
        _check(_lib.lib().m2s_grid_plan_autotune(self._h, None if stream is None else ctypes.c_void_p(stream),
                                                 ctypes.byref(b)), "grid_plan_autotune")
        return int(b.value)

    @property
    def cells(self):
        return int(_lib.lib().m2s_grid_plan_cells(self._h))

    @property
    def device_bytes(self):
        return int(_lib.lib().m2s_grid_plan_device_bytes(self._h))

    @property
    def blocks(self):
        return int(_lib.lib().m2s_grid_plan_blocks(self._h))

    @property
    def waves(self):
        return int(_lib.lib().m2s_grid_plan_waves(self._h))

    def close(self):
        if self._h and self._h.value:
            _lib.lib().m2s_grid_plan_free(self._h)
            self._h = ctypes.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def set_grid_tuning(blocks_per_sm: int = 0, cells_per_block: int = 1024, wave_cells: int = 1 << 27,
                    solo_max: int = 64):
    """Process-wide grid propagation knobs (speed only): cooperative blocks per
    SM, cells per cooperative block, the most cells a batch job holds, and the
    largest relax round run on one block (0: none)."""
    _lib.lib().m2s_set_grid_tuning(int(blocks_per_sm), int(cells_per_block), int(wave_cells), int(solo_max))


def clear_grid_autotune():
    _lib.lib().m2s_clear_grid_autotune()


# ---- results for the viewer -----------------------------------------------------

def sort_cells_by_distance(distances):
    """mesh_to_sdf_client/src/sdf.rs:63-71 on the GPU: (order, (min, max)) —
    the cell indices stably sorted by f32::total_cmp of the distances (u32) and
    the distances' extremes (the viewer's iso limits)."""
    d = np.ascontiguousarray(distances, F32).reshape(-1)
    order = np.empty(len(d), np.uint32)
    mm = np.zeros(2, F32)
    if len(d):
        _check(_lib.lib().m2s_sort_cells_by_distance(_vp(d), len(d), _vp(order), _vp(mm), None),
               "sort_cells_by_distance")
    return order, (float(mm[0]), float(mm[1]))


def sort_cells_by_distance_device(distances, order, minmax=None, stream=None):
    """The same on device tensors (float32 in, uint32/int32 order out, optional 2-float minmax)."""
    _check(_lib.lib().m2s_sort_cells_by_distance_device(
        ctypes.c_void_p(distances.data_ptr()), distances.numel(), ctypes.c_void_p(order.data_ptr()),
        None if minmax is None else ctypes.c_void_p(minmax.data_ptr()),
        None if stream is None else ctypes.c_void_p(stream)), "sort_cells_by_distance_device")


# ---- mesh check ------------------------------------------------------------------

def _rust_debug_f32(x) -> str:
    """`{:?}` of an f32 as Rust prints it: shortest round-trip digits, decimal
    with at least one fractional digit for 1e-4 <= |x| < 1e16 (and 0),
    exponential otherwise."""
    x = np.float32(x)
    if np.isnan(x):
        return "NaN"
    if np.isinf(x):
        return "inf" if x > 0 else "-inf"
    a = np.abs(x)  # compared in f32, as Rust does
    if a == 0 or np.float32(1e-4) <= a < np.float32(1e16):
        return np.format_float_positional(x, unique=True, trim="0")
    mant, exp = np.format_float_scientific(x, unique=True, trim="-").split("e")
    return f"{mant}e{int(exp)}"


def check_mesh_triangle_list(vertices, faces):
    """generate/mesh_check.rs:24-81 on the GPU: None when the mesh is
    watertight with no duplicate vertices or faces (the crate's Ok(())),
    otherwise the crate's error message (its Err(String))."""
    v = np.ascontiguousarray(np.asarray(vertices, F32).reshape(-1, 3))
    f = np.ascontiguousarray(np.asarray(faces).reshape(-1).astype(np.uint32))
    result = ctypes.c_int(0)
    detail = np.zeros(2, np.uint64)
    _check(_lib.lib().m2s_check_mesh_triangle_list(_vp(v) if len(v) else None, len(v), _vp(f) if len(f) else None,
                                                   len(f), ctypes.byref(result), _vp(detail), None),
           "check_mesh_triangle_list")
    k, a, b = result.value, int(detail[0]), int(detail[1])
    if k == 0:
        return None
    if k == 1:
        return "Faces must be a multiple of 3"
    if k == 2:
        x, y, z = (_rust_debug_f32(c) for c in v[a])
        return f"Duplicate vertex found at ({x}, {y}, {z})"
    if k == 3:
        return f"Duplicate face found: [{f[3 * a]}, {f[3 * a + 1]}, {f[3 * a + 2]}]"
    if k == 4:
        return f"Duplicate edge {a} -> {b} - do you have an inverted normal?"
    return (f"Mesh is not waterproof - edge {a} -> {b} does not have a corresponding edge {b} -> {a}")


# ---- serving loop (no counterpart in the crate) -----------------------------

SERVER_STATS = ("uploads", "point_requests", "grid_requests", "failed", "grid_batches", "grid_requests_batched",
                "largest_batch", "reserved_bytes", "peak_reserved_bytes", "resident_meshes", "queued", "evictions")


def _host_ptr(a):
    """Pointer of a C-contiguous numpy array or CPU torch tensor (pinned or not)."""
    if hasattr(a, "data_ptr"):
        if a.is_cuda or not a.is_contiguous():
            raise ValueError("server buffers are contiguous host memory")
        return ctypes.c_void_p(a.data_ptr())
    if not a.flags["C_CONTIGUOUS"]:
        raise ValueError("server buffers are contiguous host memory")
    return ctypes.c_void_p(a.ctypes.data)


class Server:
    """Resident meshes, device-memory admission and batched requests on one GPU
    (m2s_server_*).  submit_* return a ticket at once; the buffers passed stay
    referenced here until wait() returns for that ticket.  Results equal the
    single-request calls: query_sdf for points, SdfAccelerationMesh.grid_device
    for grids."""

    def __init__(self, hbm_budget_bytes: int, point_streams: int = 4):
        h = ctypes.c_void_p(None)
        _check(_lib.lib().m2s_server_create(int(hbm_budget_bytes), int(point_streams), ctypes.byref(h)),
               "server_create")
        self._h = h
        self._keep = {}

    def submit_upload(self, vertices, indices: Topology, acceleration_method: AccelerationMethod = None):
        """Returns (mesh_id, ticket)."""
        am = acceleration_method or AccelerationMethod.default()
        v = _points(vertices)
        idx, ni, bits, topo = indices._ffi()
        mid, t = ctypes.c_uint32(0), ctypes.c_uint64(0)
        _check(_lib.lib().m2s_server_submit_upload(self._h, _vp(v), len(v), _vp(idx), ni, bits, topo, am.kind,
                                                   int(am.sign), ctypes.byref(mid), ctypes.byref(t)),
               "server_submit_upload")
        return int(mid.value), int(t.value)

    def submit_points(self, mesh_id: int, queries, out):
        """queries: (n,3) float32 host array; out: n float32 host array."""
        t = ctypes.c_uint64(0)
        n = int(queries.shape[0])
        _check(_lib.lib().m2s_server_submit_points(self._h, int(mesh_id), _host_ptr(queries), n, _host_ptr(out),
                                                   ctypes.byref(t)), "server_submit_points")
        self._keep[t.value] = (queries, out)
        return int(t.value)

    def submit_grid(self, mesh_id: int, grid: Grid, sign_method: SignMethod, out):
        """out: grid.get_total_cell_count() float32 host array."""
        first = np.ascontiguousarray(grid.first_cell, F32)
        size = np.ascontiguousarray(grid.cell_size, F32)
        count = np.ascontiguousarray(np.array(grid.cell_count, np.uint64))
        t = ctypes.c_uint64(0)
        _check(_lib.lib().m2s_server_submit_grid(self._h, int(mesh_id), _vp(first), _vp(size), _vp(count),
                                                 int(sign_method), _host_ptr(out), ctypes.byref(t)),
               "server_submit_grid")
        self._keep[t.value] = (out,)
        return int(t.value)

    def wait(self, ticket: int, timeout_s: float = -1.0):
        """(status, latency_s) of a ticket; status 0 is success."""
        st, lat = ctypes.c_int(0), ctypes.c_double(0.0)
        _check(_lib.lib().m2s_server_wait(self._h, int(ticket), float(timeout_s), ctypes.byref(st),
                                          ctypes.byref(lat)), "server_wait")
        self._keep.pop(int(ticket), None)
        return int(st.value), float(lat.value)

    def remove_mesh(self, mesh_id: int):
        _check(_lib.lib().m2s_server_remove_mesh(self._h, int(mesh_id)), "server_remove_mesh")

    def stats(self):
        a = np.zeros(len(SERVER_STATS), np.uint64)
        _check(_lib.lib().m2s_server_stats(self._h, _vp(a)), "server_stats")
        return dict(zip(SERVER_STATS, (int(x) for x in a)))

    def close(self):
        if self._h and self._h.value:
            _lib.lib().m2s_server_free(self._h)
            self._h = ctypes.c_void_p(None)
            self._keep.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def radix_sort_pairs_device(keys, values, key_bits=32, stream=None):
    """Stable LSD radix sort of device uint32 (int32 tensors reinterpreted) key/value pairs, in place."""
    st = _lib.lib().m2s_radix_sort_pairs_device(ctypes.c_void_p(keys.data_ptr()), ctypes.c_void_p(values.data_ptr()),
                                                keys.numel(), int(key_bits),
                                                None if stream is None else ctypes.c_void_p(stream))
    _check(st, "radix_sort_pairs_device")
