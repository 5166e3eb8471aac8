"""CPU-only checks of the C ABI boundary: the library loads, exports every
symbol include/m2s.h declares, and validates arguments like the crate does
before any device work.  No compute call reaches a GPU here."""
import ctypes
import os
import re

import numpy as np
import pytest

import mesh_to_sdf_b200 as m2s
from mesh_to_sdf_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "m2s.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(m2s_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = _lib.lib()
    names = declared_symbols()
    assert len(names) >= 15
    for name in names:
        assert hasattr(L, name), name
    # and the Python binding covers all of them
    assert set(names) == set(_lib.SIGNATURES)


def test_status_strings():
    L = _lib.lib()
    assert L.m2s_status_string(0) == b"ok"
    assert b"non-finite" in L.m2s_status_string(2)
    assert L.m2s_version() >= 100


TETRA_V = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, -1]], np.float32)
TETRA_IDX = np.array([0, 1, 2, 0, 2, 3, 0, 3, 1, 1, 3, 2], np.uint32)


def test_host_validation_matches_crate_panics():
    # lib.rs:374-376 (non-finite query) and lib.rs:203 (list length % 3) are
    # decided on the host before any device is touched.
    with pytest.raises(m2s.M2SError) as e:
        m2s.generate_sdf(TETRA_V, m2s.Topology.TriangleList(TETRA_IDX), [[0, 0, np.nan]],
                         m2s.AccelerationMethod.bvh(m2s.SignMethod.Raycast))
    assert e.value.status == 2
    with pytest.raises(m2s.M2SError) as e:
        m2s.generate_sdf(TETRA_V, m2s.Topology.TriangleList(np.append(TETRA_IDX, 0)), [[0.2, 0.2, 0.05]],
                         m2s.AccelerationMethod.bvh(m2s.SignMethod.Raycast))
    assert e.value.status == 3
    with pytest.raises(m2s.M2SError) as e:  # lib.rs:207 (no indices, vertex count % 3)
        m2s.generate_sdf(TETRA_V, m2s.Topology.TriangleList(None), [[0.2, 0.2, 0.05]])
    assert e.value.status == 3


@pytest.mark.skipif(os.path.exists("/dev/nvidia0"), reason="checks the no-device path")
def test_no_device_fails_loudly():
    assert not m2s.device_available()
    with pytest.raises(m2s.M2SError) as e:
        m2s.generate_sdf(TETRA_V, m2s.Topology.TriangleList(TETRA_IDX), [[0.2, 0.2, 0.05]])
    assert e.value.status == 10
    grid = m2s.Grid.from_bounding_box([0, 0, 0], [1, 1, 1], [4, 4, 4])
    with pytest.raises(m2s.M2SError) as e:
        m2s.generate_grid_sdf(TETRA_V, m2s.Topology.TriangleList(TETRA_IDX), grid)
    assert e.value.status == 10


def test_grid_helpers_match_oracle(orc):
    # grid.rs:179-297 through the Python mirror, against the oracle's restatement.
    rng = np.random.default_rng(5)
    for _ in range(50):
        lo = rng.uniform(-3, 1, 3).astype(np.float32)
        hi = (lo + rng.uniform(0.1, 4, 3)).astype(np.float32)
        n = [int(x) for x in rng.integers(1, 40, 3)]
        g = m2s.Grid.from_bounding_box(lo, hi, n)
        f, s = orc.grid_from_bounding_box(lo, hi, n)
        assert np.array_equal(g.first_cell.view(np.uint32), f.view(np.uint32))
        assert np.array_equal(g.cell_size.view(np.uint32), s.view(np.uint32))
        cell = [int(rng.integers(0, k)) for k in n]
        assert np.array_equal(g.get_cell_center(cell), orc.grid_cell_center(f, s, cell))
        p = rng.uniform(-4, 6, 3).astype(np.float32)
        snap = g.snap_point_to_grid(p)
        inside, c = orc.grid_snap_point(f, s, n, p)
        assert snap.inside == inside and list(snap.cell) == c
        i = g.get_cell_idx(cell)
        assert g.get_cell_integer_coordinates(i) == cell
    centers = g.cell_centers()
    assert np.array_equal(centers[g.get_cell_idx([1, 2, 0])], g.get_cell_center([1, 2, 0]))


def test_grid_known_answers():
    # grid.rs:190-211
    g = m2s.Grid.new([0.0, 1.0, 2.0], [1.0, 2.0, 3.0], [10, 20, 30])
    assert g.get_last_cell().tolist() == [10.0, 41.0, 92.0]
    g = m2s.Grid.from_bounding_box([-1.0, 0.0, 1.0], [0.0, 2.0, 5.0], [2, 2, 2])
    assert g.first_cell.tolist() == [-0.75, 0.5, 2.0] and g.cell_size.tolist() == [0.5, 1.0, 2.0]
    mn, mx = g.get_bounding_box()
    assert mn.tolist() == [-1.0, 0.0, 1.0] and mx.tolist() == [0.0, 2.0, 5.0]
    g = m2s.Grid.from_bounding_box([0, 0, 0], [1, 1, 1], [2, 3, 4])
    assert [g.get_cell_idx(c) for c in ([0, 0, 1], [0, 1, 0], [1, 0, 0], [1, 1, 1])] == [1, 4, 12, 17]


def test_acceleration_method_list():
    # lib.rs:289-296
    names = [repr(m) for m in m2s.ALL_SDF_ACCELERATION_METHODS]
    assert names == ["AccelerationMethod.None(Raycast)", "AccelerationMethod.None(Normal)",
                     "AccelerationMethod.Bvh(Raycast)", "AccelerationMethod.Bvh(Normal)", "AccelerationMethod.Rtree",
                     "AccelerationMethod.RtreeBvh"]
