"""The FP64 audit (m2s_set_fp64_audit): f32 ray tests and Voronoi-region
choices whose compared quantity lies within a forward-error bound are
re-decided in FP64 on the device and counted; results never change.

Cases built so the counts are known:
  * a ray that passes within rounding of a triangle's edge, where f32 and
    FP64 disagree: the reference's w0 = (o - t1)_z (t2 - t1)_y - (o - t1)_y
    (t2 - t1)_z (geo.rs:196) rounds to exactly 0 in f32 (no crossing), while
    FP64 gives +6.5e-9 (a crossing).  The vertices were found by a seeded
    search that emulates the f32 arithmetic in numpy (every operation rounded,
    no fused multiply-add) and is repeated below as a check;
  * a cube whose faces and edges lie exactly on the ray origins of a grid:
    the edge functions are exactly zero there, so the tests are flagged, and
    FP64 agrees with f32.
"""
import numpy as np
import pytest

import mesh_to_sdf_b200 as m2s
from mesh_to_sdf_b200 import synth

pytestmark = pytest.mark.gpu

T = m2s.Topology
A = m2s.AccelerationMethod
S = m2s.SignMethod

TRI = np.array([[1.0, -0.54958564, -0.1977969], [1.0, -0.8046243, -0.18827872], [1.0, -0.01904873, -0.35725582]],
               np.float32)
ORIGIN = np.array([[0.0, -0.21571323, -0.31495333]], np.float32)


@pytest.fixture(scope="module", autouse=True)
def _device():
    if not m2s.device_available():
        pytest.fail("no sm_100 device: the GPU suite must run on a B200")
    yield
    m2s.set_fp64_audit(False)


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def test_case_disagrees_in_numpy():
    # the f32 edge functions of the +X test, each operation rounded to f32
    f = np.float32
    t0, t1, t2 = TRI
    o = ORIGIN[0]

    def w32(a, b):
        p, e = (o - a).astype(f), (b - a).astype(f)
        return f(f(p[2] * e[1]) - f(p[1] * e[2]))

    def w64(a, b):
        p, e = o.astype(np.float64) - a, b.astype(np.float64) - a
        return p[2] * e[1] - p[1] * e[2]

    assert w32(t1, t2) == 0.0 and w64(t1, t2) > 0.0
    assert w32(t2, t0) > 0 and w32(t0, t1) > 0 and w64(t2, t0) > 0 and w64(t0, t1) > 0


def test_point_ray_decision_fp64_disagrees():
    idx = np.array([0, 1, 2], np.uint32)
    for am in (A.rtree_bvh(), A.bvh(S.Raycast)):
        m2s.set_fp64_audit(False)
        plain = m2s.generate_sdf(TRI, T.TriangleList(idx), ORIGIN, am)
        m2s.set_fp64_audit(True)
        audited = m2s.generate_sdf(TRI, T.TriangleList(idx), ORIGIN, am)
        a = m2s.last_query_audit()
        m2s.set_fp64_audit(False)
        assert np.array_equal(bits(plain), bits(audited)), repr(am)
        assert a["ray_tests"] >= 1 and a["ray_ambiguous"] >= 1 and a["ray_fp64_disagrees"] == 1, a
        assert a["regions"] == 1, a


def test_grid_on_cube_edges_flags_exact_zeros():
    # unit cube [-0.5, 0.5]^3, 12 outward triangles; grid centres every 0.25 from -1
    v = np.array([[x, y, z] for x in (-0.5, 0.5) for y in (-0.5, 0.5) for z in (-0.5, 0.5)], np.float32)
    quads = [(0, 1, 3, 2), (4, 6, 7, 5), (0, 4, 5, 1), (2, 3, 7, 6), (0, 2, 6, 4), (1, 5, 7, 3)]
    idx = np.array([k for a, b, c, d in quads for k in (a, b, c, a, c, d)], np.uint32)
    grid = m2s.Grid.new([-1.0, -1.0, -1.0], [0.25, 0.25, 0.25], [9, 9, 9])
    for sign in (S.Raycast, S.Normal):
        m2s.set_fp64_audit(False)
        plain = m2s.generate_grid_sdf(v, T.TriangleList(idx), grid, sign)
        m2s.set_fp64_audit(True)
        audited = m2s.generate_grid_sdf(v, T.TriangleList(idx), grid, sign)
        a = m2s.last_grid_audit()
        m2s.set_fp64_audit(False)
        assert np.array_equal(bits(plain), bits(audited)), sign
        assert a["regions"] == grid.get_total_cell_count(), a
        if sign == S.Raycast:
            assert a["ray_tests"] > 0 and a["ray_ambiguous"] > 0, a
            assert a["ray_fp64_disagrees"] == 0 and a["vote_flips"] == 0, a  # exact zeros: FP64 agrees
        else:
            assert a["ray_tests"] == 0, a


def test_audit_changes_no_result_on_the_star():
    v, idx = synth.star(4, seed=31)
    lo, hi = synth.padded_bbox(v)
    grid = m2s.Grid.from_bounding_box(lo, hi, [48, 52, 44])
    q = synth.mixed_points(v, idx, 20_000, seed=32)
    for sign in (S.Raycast, S.Normal):
        m2s.set_fp64_audit(False)
        g0 = m2s.generate_grid_sdf(v, T.TriangleList(idx), grid, sign)
        m2s.set_fp64_audit(True)
        g1 = m2s.generate_grid_sdf(v, T.TriangleList(idx), grid, sign)
        a = m2s.last_grid_audit()
        m2s.set_fp64_audit(False)
        assert np.array_equal(bits(g0), bits(g1)), sign
        assert a["regions"] > 0 and a["region_fp64_disagrees"] <= a["region_ambiguous"], a
    for am in (A.rtree_bvh(), A.bvh(S.Raycast), A.rtree(), A.bvh(S.Normal)):
        m2s.set_fp64_audit(False)
        p0 = m2s.generate_sdf(v, T.TriangleList(idx), q, am)
        m2s.set_fp64_audit(True)
        p1 = m2s.generate_sdf(v, T.TriangleList(idx), q, am)
        a = m2s.last_query_audit()
        m2s.set_fp64_audit(False)
        assert np.array_equal(bits(p0), bits(p1)), repr(am)
        assert a["regions"] == len(q), (repr(am), a)
        assert a["ray_fp64_disagrees"] <= a["ray_ambiguous"] and a["region_fp64_disagrees"] <= a["region_ambiguous"]
