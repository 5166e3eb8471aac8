"""CPU oracle for mesh_to_sdf_b200 — TEST INFRASTRUCTURE, never part of the product.

A C++ restatement of the Rust crate ``mesh_to_sdf`` (``m2s_oracle.cpp``), wrapped
with ctypes.  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline
leg of ``bench.py`` may import this module; the shipped library never does, and
it has no CPU fallback that could route through here.

Status codes are the numbers of ``include/m2s.h``.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_SO = os.path.join(_HERE, "liboracle.so")
_lock = threading.Lock()
_lib = None

ACCEL = {"none": 0, "bvh": 1, "rtree": 2, "rtree_bvh": 3}
SIGN = {"raycast": 0, "normal": 1}


def build(force: bool = False) -> str:
    """Compile liboracle.so in place with the Makefile beside this file."""
    args = ["make", "-C", _HERE, "-s"] + (["-B"] if force else [])
    subprocess.check_call(args)
    return _SO


def lib():
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(_SO):
                build()
            L = ctypes.CDLL(_SO)
            P = ctypes.c_void_p
            U64 = ctypes.c_uint64
            I = ctypes.c_int
            F = ctypes.c_float
            L.orc_point_triangle_distance.restype = F
            L.orc_point_triangle_distance2.restype = F
            L.orc_point_triangle_signed_distance.restype = F
            L.orc_compare_distances.argtypes = [F, F]
            L.orc_compare_distances.restype = I
            L.orc_ray_triangle_intersection_aligned.restype = I
            L.orc_expand_topology.argtypes = [U64, P, U64, I, I, P, P]
            L.orc_generate_sdf.argtypes = [P, U64, P, U64, I, I, P, U64, I, I, P, P, I]
            L.orc_query_vector_to_closest_point.argtypes = [P, U64, P, U64, I, I, P, U64, P, P, P, I]
            L.orc_generate_grid_sdf.argtypes = [P, U64, P, U64, I, I, P, P, P, I, P, P, I, P]
            L.orc_generate_sdf_f64.argtypes = [P, U64, P, U64, I, I, P, U64, P, P, I]
            L.orc_grid_snap_point.restype = I
            L.orc_check_mesh_triangle_list.argtypes = [P, U64, P, U64, P, P]
            _lib = L
    return _lib


def _f3(x):
    a = np.ascontiguousarray(np.asarray(x, dtype=np.float32).reshape(-1))
    return a


def _ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


class OracleError(RuntimeError):
    def __init__(self, status: int, what: str):
        super().__init__(f"{what}: oracle status {status}")
        self.status = status


def _mesh(vertices, indices, strip):
    v = np.ascontiguousarray(np.asarray(vertices, dtype=np.float32).reshape(-1, 3))
    if indices is None:
        return v, None, 0, 0, 1 if strip else 0
    idx = np.asarray(indices)
    if idx.dtype == np.uint16:
        bits = 16
    else:
        idx = idx.astype(np.uint32)
        bits = 32
    idx = np.ascontiguousarray(idx.reshape(-1))
    return v, idx, len(idx), bits, 1 if strip else 0


def _sign_code(sign):
    return SIGN[sign] if isinstance(sign, str) else int(sign)


def _accel_code(accel):
    return ACCEL[accel] if isinstance(accel, str) else int(accel)


# ---------------------------------------------------------------- geometry
def _pts(*xs):
    """float32[3] copies of the arguments; the caller keeps the list alive for the call."""
    return [_f3(x) for x in xs]


def closest_point_triangle(p, a, b, c):
    out = np.zeros(3, np.float32)
    arrs = _pts(p, a, b, c)
    lib().orc_closest_point_triangle(*[_ptr(x) for x in arrs], _ptr(out))
    return out


def point_triangle_distance(p, a, b, c) -> float:
    arrs = _pts(p, a, b, c)
    return lib().orc_point_triangle_distance(*[_ptr(x) for x in arrs])


def point_triangle_distance2(p, a, b, c) -> float:
    arrs = _pts(p, a, b, c)
    return lib().orc_point_triangle_distance2(*[_ptr(x) for x in arrs])


def point_triangle_signed_distance(p, a, b, c) -> float:
    arrs = _pts(p, a, b, c)
    return lib().orc_point_triangle_signed_distance(*[_ptr(x) for x in arrs])


def ray_triangle_intersection_aligned(o, a, b, c, axis: int):
    t = np.zeros(1, np.float32)
    arrs = _pts(o, a, b, c)
    hit = lib().orc_ray_triangle_intersection_aligned(*[_ptr(x) for x in arrs], int(axis), _ptr(t))
    return float(t[0]) if hit else None


def triangle_bounding_box(a, b, c):
    mn = np.zeros(3, np.float32)
    mx = np.zeros(3, np.float32)
    arrs = _pts(a, b, c)
    lib().orc_triangle_bounding_box(*[_ptr(x) for x in arrs], _ptr(mn), _ptr(mx))
    return mn, mx


def compare_distances(a: float, b: float) -> int:
    """-1 / 0 / 1, or 2 where the reference panics on NaN."""
    return lib().orc_compare_distances(float(a), float(b))


def expand_topology(n_vertices, indices=None, strip=False):
    idx = None
    bits = 0
    ni = 0
    if indices is not None:
        idx = np.asarray(indices)
        bits = 16 if idx.dtype == np.uint16 else 32
        idx = np.ascontiguousarray(idx.astype(np.uint16 if bits == 16 else np.uint32).reshape(-1))
        ni = len(idx)
    n = ctypes.c_uint64(0)
    st = lib().orc_expand_topology(n_vertices, _ptr(idx), ni, bits, 1 if strip else 0, None, ctypes.byref(n))
    if st:
        return st, None
    out = np.zeros((n.value, 3), np.uint32)
    lib().orc_expand_topology(n_vertices, _ptr(idx), ni, bits, 1 if strip else 0, _ptr(out), ctypes.byref(n))
    return 0, out


# ---------------------------------------------------------------- entry points
def generate_sdf(vertices, indices, queries, accel, sign="raycast", strip=False, n_threads=0, check=True):
    v, idx, ni, bits, topo = _mesh(vertices, indices, strip)
    q = np.ascontiguousarray(np.asarray(queries, dtype=np.float32).reshape(-1, 3))
    out = np.zeros(len(q), np.float32)
    n = ctypes.c_uint64(0)
    st = lib().orc_generate_sdf(_ptr(v), len(v), _ptr(idx), ni, bits, topo, _ptr(q), len(q),
                                _accel_code(accel), _sign_code(sign), _ptr(out), ctypes.byref(n), int(n_threads))
    if check and st:
        raise OracleError(st, "generate_sdf")
    return (out[: n.value] if not st else None) if check else (st, out[: n.value])


def query_vector_to_closest_point(vertices, indices, queries, strip=False, n_threads=0):
    v, idx, ni, bits, topo = _mesh(vertices, indices, strip)
    q = np.ascontiguousarray(np.asarray(queries, dtype=np.float32).reshape(-1, 3))
    vec = np.zeros((len(q), 3), np.float32)
    inside = np.zeros(len(q), np.uint8)
    n = ctypes.c_uint64(0)
    st = lib().orc_query_vector_to_closest_point(_ptr(v), len(v), _ptr(idx), ni, bits, topo, _ptr(q), len(q),
                                                 _ptr(vec), _ptr(inside), ctypes.byref(n), int(n_threads))
    if st:
        raise OracleError(st, "query_vector_to_closest_point")
    return vec, inside.astype(bool)


def generate_grid_sdf(vertices, indices, first_cell, cell_size, cell_count, sign="raycast", strip=False,
                      n_threads=1, check=True, stats=None):
    v, idx, ni, bits, topo = _mesh(vertices, indices, strip)
    f = _f3(first_cell)
    s = _f3(cell_size)
    c = np.ascontiguousarray(np.asarray(cell_count, dtype=np.uint64).reshape(3))
    N = int(c[0]) * int(c[1]) * int(c[2])
    out = np.zeros(N, np.float32)
    n = ctypes.c_uint64(0)
    st_arr = np.zeros(4, np.uint64)
    st = lib().orc_generate_grid_sdf(_ptr(v), len(v), _ptr(idx), ni, bits, topo, _ptr(f), _ptr(s), _ptr(c),
                                     _sign_code(sign), _ptr(out), ctypes.byref(n), int(n_threads), _ptr(st_arr))
    if stats is not None:
        stats[:] = [int(x) for x in st_arr]
    if check:
        if st:
            raise OracleError(st, "generate_grid_sdf")
        return out[: n.value]
    return st, out[: n.value]


def generate_sdf_f64(vertices, indices, queries, strip=False, n_threads=0):
    """(unsigned distance in float64, 3-ray inside vote evaluated in float64)."""
    v, idx, ni, bits, topo = _mesh(vertices, indices, strip)
    q = np.ascontiguousarray(np.asarray(queries, dtype=np.float32).reshape(-1, 3))
    d = np.zeros(len(q), np.float64)
    inside = np.zeros(len(q), np.uint8)
    st = lib().orc_generate_sdf_f64(_ptr(v), len(v), _ptr(idx), ni, bits, topo, _ptr(q), len(q), _ptr(d),
                                    _ptr(inside), int(n_threads))
    if st:
        raise OracleError(st, "generate_sdf_f64")
    return d, inside.astype(bool)


def grid_from_bounding_box(bbox_min, bbox_max, cell_count):
    first = np.zeros(3, np.float32)
    size = np.zeros(3, np.float32)
    mn, mx = _pts(bbox_min, bbox_max)
    c = np.ascontiguousarray(np.asarray(cell_count, dtype=np.uint64).reshape(3))
    lib().orc_grid_from_bounding_box(_ptr(mn), _ptr(mx), _ptr(c), _ptr(first), _ptr(size))
    return first, size


def grid_cell_center(first_cell, cell_size, cell):
    out = np.zeros(3, np.float32)
    f, s = _pts(first_cell, cell_size)
    c = np.ascontiguousarray(np.asarray(cell, dtype=np.uint64).reshape(3))
    lib().orc_grid_cell_center(_ptr(f), _ptr(s), _ptr(c), _ptr(out))
    return out


def grid_snap_point(first_cell, cell_size, cell_count, p):
    cell = np.zeros(3, np.uint64)
    f, s, pp = _pts(first_cell, cell_size, p)
    c = np.ascontiguousarray(np.asarray(cell_count, dtype=np.uint64).reshape(3))
    inside = lib().orc_grid_snap_point(_ptr(f), _ptr(s), _ptr(c), _ptr(pp), _ptr(cell))
    return bool(inside), [int(x) for x in cell]


def check_mesh_triangle_list(vertices, faces):
    """(kind, (a, b)) of generate/mesh_check.rs:24-81 — see m2s_oracle.h for the kinds."""
    v = np.ascontiguousarray(np.asarray(vertices, np.float32).reshape(-1, 3))
    f = np.ascontiguousarray(np.asarray(faces, np.uint32).reshape(-1))
    kind = ctypes.c_int(0)
    detail = np.zeros(2, np.uint64)
    lib().orc_check_mesh_triangle_list(_ptr(v), len(v), _ptr(f), len(f), ctypes.byref(kind), _ptr(detail))
    return kind.value, (int(detail[0]), int(detail[1]))
