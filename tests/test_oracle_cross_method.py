"""The reference's cross-method checks, on the oracle and this repository's
seeded closed meshes, so that they run on any machine (the same checks on
the reference's own meshes are in tests/test_reference_assets.py, which needs
a checkout).  Tolerances are the reference tests':

  generate/generic/bvh.rs:190-355      Bvh vs None at 5 points; Bvh(Raycast) vs the
                                       grid on 32^3 cell centres; Bvh(Normal) on 16^3
  generate/generic/rtree.rs:166-280    Rtree vs Bvh(Normal); on 32^3 |d| within 0.01
                                       and fewer than 1 % of the signs differ
  generate/generic/rtree_bvh.rs:287-475  RtreeBvh vs Bvh(Raycast); vector lengths
                                       vs |sdf|; RtreeBvh vs the grid on 32^3
  generate/grid.rs:728-818             neighbouring cells: |d| within a cell size,
                                       a sign change only within a cell size
CPU only."""
import numpy as np
import pytest

from mesh_to_sdf_b200 import synth

POINTS5 = np.array([[0.01, 0.01, 0.5], [1.0, 1.0, 1.0], [0.1, 0.2, 0.2], [1.1, 2.2, 5.2], [-0.1, 0.2, -0.2]],
                   np.float32)
MESHES = {"icosphere_s3": lambda: synth.icosphere(3), "star_s3": lambda: synth.star(3, seed=4),
          "star_s4": lambda: synth.star(4, seed=9)}


def _grid(orc, v, cells, extend=0.0):
    lo, hi = v.min(0), v.max(0)
    if extend:
        e = np.float32(extend) * (hi - lo)
        lo, hi = lo - e, hi + e
    return orc.grid_from_bounding_box(lo, hi, [cells] * 3)


def _centres(orc, first, size, cells):
    return np.array([orc.grid_cell_center(first, size, [x, y, z])
                     for x in range(cells) for y in range(cells) for z in range(cells)], np.float32)


@pytest.mark.parametrize("mesh", list(MESHES))
def test_point_methods_agree(orc, mesh):
    v, i = MESHES[mesh]()
    none = orc.generate_sdf(v, i, POINTS5, "none", "raycast")
    bvh = orc.generate_sdf(v, i, POINTS5, "bvh", "raycast")
    assert np.all(np.abs(bvh - none) < 0.01), (bvh, none)
    rtree = orc.generate_sdf(v, i, POINTS5, "rtree")
    bvh_n = orc.generate_sdf(v, i, POINTS5, "bvh", "normal")
    assert np.all(np.abs(rtree - bvh_n) < 0.01), (rtree, bvh_n)
    rb = orc.generate_sdf(v, i, POINTS5, "rtree_bvh")
    assert np.all(np.abs(rb - bvh) < 0.01), (rb, bvh)
    vec, inside = orc.query_vector_to_closest_point(v, i, POINTS5)
    assert np.all(np.abs(np.linalg.norm(vec, axis=1) - np.abs(rb)) < 0.001)
    assert np.array_equal(inside, rb < 0)


@pytest.mark.parametrize("mesh", list(MESHES))
@pytest.mark.parametrize("accel,sign,cells", [("bvh", "raycast", 32), ("bvh", "normal", 16),
                                              ("rtree_bvh", "raycast", 32)])
def test_points_agree_with_grid(orc, mesh, accel, sign, cells):
    v, i = MESHES[mesh]()
    first, size = _grid(orc, v, cells)
    q = _centres(orc, first, size, cells)
    sdf = orc.generate_sdf(v, i, q, accel, sign)
    grid = orc.generate_grid_sdf(v, i, first, size, [cells] * 3, sign)
    bad = np.flatnonzero(~(np.abs(sdf - grid) < 0.01))
    assert len(bad) == 0, [(int(k), float(sdf[k]), float(grid[k])) for k in bad[:8]]


@pytest.mark.parametrize("mesh", list(MESHES))
def test_rtree_against_normal_grid(orc, mesh):
    v, i = MESHES[mesh]()
    first, size = _grid(orc, v, 32)
    q = _centres(orc, first, size, 32)
    sdf = orc.generate_sdf(v, i, q, "rtree")
    grid = orc.generate_grid_sdf(v, i, first, size, [32] * 3, "normal")
    assert np.all(np.abs(np.abs(sdf) - np.abs(grid)) < 0.01)
    assert np.count_nonzero(np.abs(sdf - grid) > 0.01) / len(sdf) < 0.01


@pytest.mark.parametrize("mesh", list(MESHES))
def test_grid_continuity(orc, mesh):
    v, i = MESHES[mesh]()
    first, size = _grid(orc, v, 32, extend=0.2)
    sdf = orc.generate_grid_sdf(v, i, first, size, [32] * 3, "raycast").reshape(32, 32, 32)
    d = sdf[:-1, :-1, :-1]
    for axis in range(3):
        n = np.roll(sdf, -1, axis)[:-1, :-1, :-1]
        s = size[axis]
        assert np.all(np.abs(np.abs(d) - np.abs(n)) <= s), axis
        flips = np.sign(d * n) < 0
        assert np.all(~flips | ((np.abs(d) <= s) & (np.abs(n) <= s))), axis
