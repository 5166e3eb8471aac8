"""The reference's own mesh-asset tests, run on the oracle (CPU).

The reference checks its generators on two glTF meshes it ships,
`assets/suzanne.glb` (1966 vertices, 968 triangles) and `assets/ferris3d.glb`
(13 skinned parts).  The meshes are not copied into this repository: when
M2S_REFERENCE_DIR names a checkout of the reference they are read in place by
`tests/glb.py` (and must then exist, with the SHA-256 below); otherwise these
tests are skipped.  Each test names the reference test it ports, with the same
query points, grids and tolerances:

  generate/generic/default.rs:115-150   test_generate
  generate/generic/bvh.rs:190-236       test_generate_bvh
  generate/generic/bvh.rs:239-296       test_generate_bvh_big
  generate/generic/bvh.rs:299-355       test_generate_bvh_normal
  generate/generic/rtree.rs:166-210     test_generate_rtree
  generate/generic/rtree.rs:213-280     test_generate_rtree_big
  generate/generic/rtree_bvh.rs:287-335 test_generate_rtree_bvh
  generate/generic/rtree_bvh.rs:338-380 test_query_vector_to_closest_point_sign_distance
  generate/generic/rtree_bvh.rs:422-475 test_generate_rtree_bvh_big
  generate/grid.rs:728-818              test_grid_continuity
  generate/grid.rs:820-853              test_grid_raycast

The reference's "same check but for the acceleration structure" halves compare
its build/query split with the one-shot call; the oracle has only the one-shot
call, and the library's split is checked against it by the GPU tests.  The
ferris tests run on every part of the mesh, not only `models[0]`, so they do
not depend on the order in which the loader lists the parts.
"""
import hashlib
import os

import numpy as np
import pytest

import glb

SHA256 = {
    "suzanne.glb": "4ee42831d577ab1bcd5a5a6ee669bd1280a8b3d8c39543a1fecf5e12100956a8",
    "ferris3d.glb": "e74ceee228a0846278abced052ad644807c919229d0ba67a110a40f5313f73a1",
}

POINTS5 = np.array([[0.01, 0.01, 0.5], [1.0, 1.0, 1.0], [0.1, 0.2, 0.2], [1.1, 2.2, 5.2], [-0.1, 0.2, -0.2]],
                   np.float32)

_cache = {}


def _models(name):
    root = os.environ.get("M2S_REFERENCE_DIR")
    if not root:
        pytest.skip("M2S_REFERENCE_DIR is unset: the reference's meshes are read in place")
    if name not in _cache:
        path = os.path.join(root, "mesh_to_sdf", "assets", name)
        assert os.path.exists(path), f"M2S_REFERENCE_DIR is set but {path} is missing"
        with open(path, "rb") as f:
            assert hashlib.sha256(f.read()).hexdigest() == SHA256[name], path
        _cache[name] = glb.models(path)
    return _cache[name]


@pytest.fixture(scope="module")
def suzanne():
    (mesh,) = _models("suzanne.glb")
    return mesh


def _grid(orc, vertices, cells, extend=0.0, max_scale=1.0):
    lo, hi = vertices.min(0), vertices.max(0)
    if extend:
        e = np.float32(extend) * (hi - lo)
        lo, hi = lo - e, hi + e
    hi = hi * np.float32(max_scale)
    first, size = orc.grid_from_bounding_box(lo, hi, [cells] * 3)
    return first, size


def _centres(orc, first, size, cells):
    """Cell centres in the reference's loop order (x outer, z inner), which
    is also its grid's storage order."""
    return np.array([orc.grid_cell_center(first, size, [x, y, z])
                     for x in range(cells) for y in range(cells) for z in range(cells)], np.float32)


def test_assets_read_as_the_reference_describes_them(orc):
    (v, i), = _models("suzanne.glb")
    assert v.shape == (1966, 3) and i.shape == (2904,) and i.max() == 1965
    parts = _models("ferris3d.glb")
    assert len(parts) == 13
    for v, i in parts:
        assert len(i) % 3 == 0 and i.max() < len(v)


def test_generate_default(orc, suzanne):
    v, i = suzanne
    q = np.array([[0, 0, 0], [1, 1, 1], [0.1, 0.2, 0.2]], np.float32)
    sdf = orc.generate_sdf(v, i, q, "none", "normal")
    # the reference's baseline from its own run and pysdf, within 0.1
    assert np.all(np.abs(sdf - np.array([-0.42, 0.69, -0.46], np.float32)) < 0.1), sdf


def test_generate_bvh(orc, suzanne):
    v, i = suzanne
    bvh = orc.generate_sdf(v, i, POINTS5, "bvh", "raycast")
    none = orc.generate_sdf(v, i, POINTS5, "none", "raycast")
    assert np.all(np.abs(bvh - none) < 0.01), (bvh, none)


@pytest.mark.parametrize("accel,sign,cells", [("bvh", "raycast", 32), ("bvh", "normal", 16),
                                              ("rtree_bvh", "raycast", 32)])
def test_generate_big_against_grid(orc, suzanne, accel, sign, cells):
    # bvh.rs test_generate_bvh_big / test_generate_bvh_normal, rtree_bvh.rs
    # test_generate_rtree_bvh_big: every cell centre within 0.01 of the grid
    v, i = suzanne
    first, size = _grid(orc, v, cells)
    q = _centres(orc, first, size, cells)
    sdf = orc.generate_sdf(v, i, q, accel, sign)
    grid = orc.generate_grid_sdf(v, i, first, size, [cells] * 3, sign)
    bad = np.flatnonzero(~(np.abs(sdf - grid) < 0.01))
    assert len(bad) == 0, [(int(k), float(sdf[k]), float(grid[k])) for k in bad[:8]]


def test_generate_rtree(orc, suzanne):
    v, i = suzanne
    rtree = orc.generate_sdf(v, i, POINTS5, "rtree")
    bvh = orc.generate_sdf(v, i, POINTS5, "bvh", "normal")
    assert np.all(np.abs(rtree - bvh) < 0.01), (rtree, bvh)


def test_generate_rtree_big(orc, suzanne):
    v, i = suzanne
    first, size = _grid(orc, v, 32)
    q = _centres(orc, first, size, 32)
    sdf = orc.generate_sdf(v, i, q, "rtree")
    grid = orc.generate_grid_sdf(v, i, first, size, [32] * 3, "normal")
    assert np.all(np.abs(np.abs(sdf) - np.abs(grid)) < 0.01)
    # the rtree signs by its one closest triangle, the grid by a refined
    # subset: fewer than 1% of the signs may differ
    fails = int(np.count_nonzero(np.abs(sdf - grid) > 0.01))
    assert fails / len(sdf) < 0.01, fails


def test_generate_rtree_bvh(orc, suzanne):
    v, i = suzanne
    rb = orc.generate_sdf(v, i, POINTS5, "rtree_bvh")
    bvh = orc.generate_sdf(v, i, POINTS5, "bvh", "raycast")
    assert np.all(np.abs(rb - bvh) < 0.01), (rb, bvh)


def test_query_vector_to_closest_point_sign_distance(orc, suzanne):
    v, i = suzanne
    q = POINTS5[:3]
    vec, inside = orc.query_vector_to_closest_point(v, i, q)
    sdf = orc.generate_sdf(v, i, q, "rtree_bvh")
    assert np.all(np.abs(np.linalg.norm(vec, axis=1) - np.abs(sdf)) < 0.001), (vec, sdf)
    assert np.array_equal(inside, sdf < 0), (inside, sdf)


def _ferris_grids(orc, **kw):
    for part, (v, i) in enumerate(_models("ferris3d.glb")):
        first, size = _grid(orc, v, 32, **kw)
        yield part, v, i, first, size, orc.generate_grid_sdf(v, i, first, size, [32] * 3, "raycast")


def test_grid_continuity(orc):
    # grid.rs test_grid_continuity: the bounding box grown by 20% per side;
    # neighbours' unsigned distances differ by at most the cell size, and a
    # sign change only happens where both distances are within a cell size.
    # The sign half holds on the closed parts; two parts (the eyes and the
    # tongue) are open surfaces with edges that have no reverse edge, no
    # inside, and Raycast signs that change far from them.  The closed parts
    # include both candidates for `models[0]` (the arm and the head).
    closed = 0
    for part, v, i, first, size, sdf in _ferris_grids(orc, extend=0.2):
        is_closed = orc.check_mesh_triangle_list(v, i)[0] != 5
        closed += is_closed
        d = sdf.reshape(32, 32, 32)[:-1, :-1, :-1]
        for axis in range(3):
            n = np.roll(sdf.reshape(32, 32, 32), -1, axis)[:-1, :-1, :-1]
            s = size[axis]
            unsigned = np.abs(np.abs(d) - np.abs(n)) <= s
            assert np.all(unsigned), (part, axis, int(np.count_nonzero(~unsigned)))
            if is_closed:
                flips = np.sign(d * n) < 0
                signed = ~flips | ((np.abs(d) <= s) & (np.abs(n) <= s))
                assert np.all(signed), (part, axis, int(np.count_nonzero(~signed)))
    assert closed == 11


def test_grid_raycast(orc):
    # grid.rs test_grid_raycast: bbox_max halved, so the mesh pokes out of
    # the grid and the rays leave it early; the call must simply succeed
    for part, v, i, first, size, sdf in _ferris_grids(orc, max_scale=0.5):
        assert sdf.shape == (32 ** 3,) and not np.all(np.isnan(sdf)), part
