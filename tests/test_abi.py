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


def test_rust_crate_binds_every_declared_symbol():
    # rust/mesh_to_sdf_cuda/src/ffi.rs (the drop-in crate's raw bindings; no
    # Rust toolchain on this image) declares exactly the header's functions
    import re

    ffi = open(os.path.join(ROOT, "rust", "mesh_to_sdf_cuda", "src", "ffi.rs")).read()
    bound = set(re.findall(r"pub fn (m2s_\w+)\(", ffi))
    assert bound == set(declared_symbols()), (set(declared_symbols()) - bound, bound - set(declared_symbols()))


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


def test_header_compiles_and_links_from_cpp(tmp_path):
    # a C++ caller of include/m2s.h, linked against the library: the boundary
    # as a non-Python host sees it (no device work: status strings, argument
    # checks and, without a GPU, the no-device status)
    import shutil
    import subprocess

    gxx = shutil.which("g++")
    if not gxx:
        pytest.skip("no g++")
    lib_path = _lib.lib()._name
    src = tmp_path / "caller.cpp"
    src.write_text(r'''
#include <cstdio>
#include <cstring>
#include "m2s.h"
int main() {
  if (std::strcmp(m2s_status_string(M2S_OK), "ok") != 0) return 1;
  const float v[12] = {0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, -1};
  const uint32_t idx[4] = {0, 1, 2, 0};  // not a multiple of 3: the crate panics (lib.rs:203)
  const float q[3] = {0.2f, 0.2f, 0.05f};
  float out[1];
  uint64_t n = 0;
  int st = m2s_generate_sdf(v, 4, idx, 4, M2S_INDEX_U32, M2S_TOPOLOGY_TRIANGLE_LIST, q, 1, M2S_ACCEL_BVH,
                            M2S_SIGN_RAYCAST, out, &n, nullptr);
  std::printf("%d %s\n", st, m2s_status_string(st));
  return st == M2S_ERR_INDEX_COUNT ? 0 : 2;
}
''')
    exe = tmp_path / "caller"
    r = subprocess.run([gxx, "-std=c++17", "-I", os.path.join(ROOT, "include"), str(src), lib_path, "-o", str(exe),
                        f"-Wl,-rpath,{os.path.dirname(lib_path)}"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, (r.stdout, r.stderr)
