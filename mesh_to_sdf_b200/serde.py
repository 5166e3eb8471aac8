"""serde.rs: saving and loading signed distance fields in the crate's format V1.

The bytes are produced and parsed by the library (m2s_serialize_* /
m2s_deserialize), so a file written here reads back in the crate with
`read_from_file`, and the crate's files read here.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import Union

import numpy as np

from . import Grid, _lib

F32 = np.float32


class SerdeError(RuntimeError):
    """serde.rs:41-52: serialization, deserialization or I/O failed."""


@dataclass
class SerializeGeneric:
    """serde.rs:83-90: query points and their distances (from generate_sdf)."""
    query_points: np.ndarray
    distances: np.ndarray


@dataclass
class SerializeGrid:
    """serde.rs:92-99: a grid and its distances (from generate_grid_sdf)."""
    grid: Grid
    distances: np.ndarray


DeserializeGeneric = SerializeGeneric  # serde.rs:125-132
DeserializeGrid = SerializeGrid        # serde.rs:134-141
SerializeSdf = Union[SerializeGeneric, SerializeGrid]


def _vp(a):
    return ctypes.c_void_p(a.ctypes.data)


def serialize(sdf: SerializeSdf) -> bytes:
    """serde.rs:154-160: the V1 bytes of `sdf`."""
    L = _lib.lib()
    d = np.ascontiguousarray(sdf.distances, F32).reshape(-1)
    n = ctypes.c_uint64(0)
    if isinstance(sdf, SerializeGeneric):
        q = np.ascontiguousarray(sdf.query_points, F32).reshape(-1, 3)
        args = lambda out, cap: L.m2s_serialize_generic(_vp(q), len(q), _vp(d), len(d), out, cap, ctypes.byref(n))
    elif isinstance(sdf, SerializeGrid):
        first = np.ascontiguousarray(sdf.grid.first_cell, F32)
        size = np.ascontiguousarray(sdf.grid.cell_size, F32)
        count = np.ascontiguousarray(np.array(sdf.grid.cell_count, np.uint64))
        args = lambda out, cap: L.m2s_serialize_grid(_vp(first), _vp(size), _vp(count), _vp(d), len(d), out, cap,
                                                     ctypes.byref(n))
    else:
        raise TypeError("SerializeGeneric or SerializeGrid expected")
    if args(None, 0) != 0:
        raise SerdeError("serialization failed")
    buf = np.empty(n.value, np.uint8)
    if args(_vp(buf), len(buf)) != 0:
        raise SerdeError("serialization failed")
    return buf.tobytes()


def deserialize(data: bytes):
    """serde.rs:163-171: a DeserializeGeneric or DeserializeGrid."""
    L = _lib.lib()
    raw = np.frombuffer(data, np.uint8)
    kind, npts, nd = ctypes.c_int(0), ctypes.c_uint64(0), ctypes.c_uint64(0)
    src = _vp(raw) if len(raw) else None
    if L.m2s_deserialize(src, len(raw), ctypes.byref(kind), ctypes.byref(npts), ctypes.byref(nd), None, None, None,
                         None, None) != 0:
        raise SerdeError("deserialization failed")
    q = np.empty((npts.value, 3), F32)
    d = np.empty(nd.value, F32)
    first, size = np.zeros(3, F32), np.zeros(3, F32)
    count = np.zeros(3, np.uint64)
    L.m2s_deserialize(src, len(raw), ctypes.byref(kind), ctypes.byref(npts), ctypes.byref(nd), _vp(q), _vp(d),
                      _vp(first), _vp(size), _vp(count))
    if kind.value == 0:
        return DeserializeGeneric(q, d)
    return DeserializeGrid(Grid(first, size, [int(c) for c in count]), d)


def save_to_file(sdf: SerializeSdf, path) -> None:
    """serde.rs:187-193."""
    try:
        with open(path, "wb") as f:
            f.write(serialize(sdf))
    except OSError as e:
        raise SerdeError(str(e)) from e


def read_from_file(path):
    """serde.rs:214-219."""
    try:
        with open(path, "rb") as f:
            data = f.read()
    except OSError as e:
        raise SerdeError(str(e)) from e
    return deserialize(data)
