"""serde.rs format V1, on the CPU (the codec is host code in the library).

Pinned by the crate's own fixtures (serde.rs:298-369: the same data must give
the same bytes, and the bytes must read back to the same data):
  * always, by their length and SHA-256 (tests/golden/serde_fixture_digests.json,
    written by tests/golden/make_serde_digests.py from the crate's files), so
    the library's bytes are checked against the crate's on any machine;
  * when M2S_REFERENCE_DIR names a checkout of the reference, also against the
    fixture files themselves (read in place; the test fails if the variable is
    set and the files are missing).
And by an independent msgpack encoder (the `msgpack` package) for the cases
the fixtures do not reach: long arrays (16- and 32-bit lengths), cell counts
in every integer width, non-finite floats, structs written as maps and 64-bit
floats.
"""
import hashlib
import json
import os

import msgpack
import numpy as np
import pytest

import mesh_to_sdf_b200 as m2s
from mesh_to_sdf_b200 import serde

DIGESTS = json.load(open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden",
                                      "serde_fixture_digests.json")))


def _check_digest(name, data):
    want = DIGESTS[name]
    assert len(data) == want["bytes"], (name, len(data))
    assert hashlib.sha256(data).hexdigest() == want["sha256"], name


def _fixture(name):
    """The crate's fixture bytes from M2S_REFERENCE_DIR, or None when the
    variable is unset (the digest check stands alone then)."""
    root = os.environ.get("M2S_REFERENCE_DIR")
    if not root:
        return None
    path = os.path.join(root, "mesh_to_sdf", "tests", name)
    assert os.path.exists(path), f"M2S_REFERENCE_DIR is set but {path} is missing"
    with open(path, "rb") as f:
        data = f.read()
    _check_digest(name, data)
    return data


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def test_generic_fixture_bytes():
    # serde.rs:298-330: queries (1,2,3), (6,5,4); distances 1, 3
    q = np.array([[1, 2, 3], [6, 5, 4]], np.float32)
    d = np.array([1, 3], np.float32)
    data = serde.serialize(serde.SerializeGeneric(q, d))
    _check_digest("sdf_generic_v1.bin", data)
    fixture = _fixture("sdf_generic_v1.bin")
    assert fixture is None or fixture == data
    back = serde.deserialize(data)
    assert isinstance(back, serde.DeserializeGeneric)
    assert np.array_equal(back.query_points, q) and np.array_equal(back.distances, d)


def test_grid_fixture_bytes():
    # serde.rs:333-366: Grid::new([1,2,3],[4,5,6],[7,8,9]), distances 0..504
    grid = m2s.Grid.new([1, 2, 3], [4, 5, 6], [7, 8, 9])
    d = np.arange(grid.get_total_cell_count(), dtype=np.float32)
    data = serde.serialize(serde.SerializeGrid(grid, d))
    _check_digest("sdf_grid_v1.bin", data)
    fixture = _fixture("sdf_grid_v1.bin")
    assert fixture is None or fixture == data
    back = serde.deserialize(data)
    assert isinstance(back, serde.DeserializeGrid)
    assert back.grid.cell_count == (7, 8, 9)
    assert np.array_equal(back.grid.first_cell, grid.first_cell) and np.array_equal(back.grid.cell_size, grid.cell_size)
    assert np.array_equal(back.distances, d)


def _pack(obj):
    return msgpack.packb(obj, use_single_float=True)


@pytest.mark.parametrize("n", [0, 1, 15, 16, 65535, 65536])
def test_generic_matches_msgpack(n):
    rng = np.random.default_rng(n)
    q = rng.normal(size=(n, 3)).astype(np.float32)
    d = rng.normal(size=n).astype(np.float32)
    if n:
        d[0] = np.inf
        q[-1, 1] = -0.0
    ref = _pack({"V1": {"Generic": [q.tolist(), d.tolist()]}})
    got = serde.serialize(serde.SerializeGeneric(q, d))
    assert got == ref
    back = serde.deserialize(got)
    assert np.array_equal(_bits(back.query_points), _bits(q)) and np.array_equal(_bits(back.distances), _bits(d))


@pytest.mark.parametrize("counts", [(1, 1, 1), (127, 1, 2), (128, 255, 1), (256, 1, 3), (65535, 1, 1),
                                    (65536, 1, 1), (1, 1 << 32, 1), (3, 4, 5)])
def test_grid_counts_every_width(counts):
    grid = m2s.Grid.new([0.5, -1.25, 3.0], [0.1, -0.2, 1e-3], counts)
    n = min(int(np.prod(counts, dtype=np.uint64)), 70000)
    d = np.linspace(-2, 2, n, dtype=np.float32)
    d[n // 2] = np.nan
    ref = _pack({"V1": {"Grid": [[grid.first_cell.tolist(), grid.cell_size.tolist(), list(counts)], d.tolist()]}})
    got = serde.serialize(serde.SerializeGrid(grid, d))
    assert got == ref
    back = serde.deserialize(got)
    assert back.grid.cell_count == tuple(counts)
    assert np.array_equal(_bits(back.distances), _bits(d))


def test_reader_accepts_maps_and_doubles():
    # a struct written with field names and f64 / integer numbers, as rmp-serde's reader accepts
    data = msgpack.packb({"V1": {"Grid": {"grid": {"first_cell": [1.0, 2, 3.5], "cell_size": {"x": 1, "y": 2.5, "z": 3},
                                                   "cell_count": [2, 1, 1]},
                                          "distances": [0.25, -1]}}}, use_single_float=False)
    back = serde.deserialize(data)
    assert back.grid.cell_count == (2, 1, 1)
    assert back.grid.first_cell.tolist() == [1.0, 2.0, 3.5] and back.grid.cell_size.tolist() == [1.0, 2.5, 3.0]
    assert back.distances.tolist() == [0.25, -1.0]


@pytest.mark.parametrize("data", [b"", b"\x80", _pack({"V2": {"Generic": [[], []]}}),
                                  _pack({"V1": {"Mesh": [[], []]}}), _pack({"V1": {"Generic": [[[1.0, 2.0]], []]}}),
                                  _pack({"V1": {"Generic": [[], [1.0]]}})[:-2],
                                  _pack({"V1": {"Generic": [[], []]}}) + b"\x00",
                                  _pack({"V1": {"Grid": [[[0, 0, 0], [1, 1, 1], [1, -1, 1]], []]}})])
def test_malformed_data_is_refused(data):
    with pytest.raises(serde.SerdeError):
        serde.deserialize(data)


def test_file_round_trip(tmp_path):
    # serde.rs:269-295
    q = np.array([[1, 2, 3], [6, 5, 4]], np.float32)
    d = np.array([1, 3], np.float32)
    path = tmp_path / "sdf.bin"
    serde.save_to_file(serde.SerializeGeneric(q, d), path)
    back = serde.read_from_file(path)
    assert np.array_equal(back.query_points, q) and np.array_equal(back.distances, d)
    with pytest.raises(serde.SerdeError):
        serde.read_from_file(tmp_path / "missing.bin")
