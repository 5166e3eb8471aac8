"""Pins the CPU oracle to the reference crate's own known-answer tests.

Every case below is a test of the Rust crate `mesh_to_sdf` restated against the
oracle (file:line citations are to `mesh_to_sdf/src/`).  These run on the CPU
only and must pass before any GPU parity claim that uses the oracle.
"""
import math

import numpy as np
import pytest

F32 = np.float32

# lib.rs:491-492
TETRA_IDX = np.array([0, 1, 2, 0, 2, 3, 0, 3, 1, 1, 3, 2], np.uint32)
TETRA_V = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, -1]], np.float32)

ALL_METHODS = [("none", "raycast"), ("none", "normal"), ("bvh", "raycast"), ("bvh", "normal"),
               ("rtree", "normal"), ("rtree_bvh", "raycast")]


def f32(x):
    return float(np.float32(x))


def test_mesh_waterproof(orc):
    # lib.rs:494-524 (one-sided check `sdf - expected < 1e-5`, kept as written)
    s2 = f32(math.sqrt(0.5))
    pfive = f32(f32(0.5 / f32(math.hypot(s2, 1.0))) * s2)
    cases = [
        ([0.0, 0.0, 0.0], 0.0), ([0.5, 0.0, 0.0], 0.0), ([0.2, 0.2, 0.0], 0.0), ([0.2, 0.2, 0.05], 0.05),
        ([0.2, 0.2, -0.05], -0.05), ([1.0, 1.0, 0.05], f32(math.sqrt(f32(0.05 * 0.05 + 0.5 * 0.5 + 0.5 * 0.5)))),
        ([1.0, 1.0, -0.05], f32(math.sqrt(f32(0.05 * 0.05 + 0.5 * 0.5 + 0.5 * 0.5)))),
        ([1.0, 1.0, 0.0], f32(math.hypot(0.5, 0.5))), ([0.0, 0.0, -1.05], 0.05), ([0.0, 0.0, -0.95], 0.0),
        ([0.5, 0.5, -0.5], pfive), ([0.5 - 1e-6, 0.5, -0.5], pfive), ([0.5, 0.5 - 1e-6, -0.5], pfive),
        ([0.5, 0.5, -0.5 - 1e-6], pfive),
    ]
    for accel, sign in ALL_METHODS:
        for q, expected in cases:
            sdf = orc.generate_sdf(TETRA_V, TETRA_IDX, [q], accel, sign)
            assert len(sdf) == 1
            assert sdf[0] - expected < 1e-5, (accel, sign, q, sdf[0], expected)


def test_mesh_not_waterproof_using_bvh_raycast(orc):
    # lib.rs:526-540
    idx = TETRA_IDX[:-3]
    sdf = orc.generate_sdf(TETRA_V, idx, [[1.0, 1.0, -0.05]], "bvh", "raycast")
    assert sdf[0] == np.sqrt(np.float32(0.05 * 0.05 + 0.5 * 0.5 + 0.5 * 0.5), dtype=np.float32)


def test_mesh_reversed_normal_using_bvh_raycast(orc):
    # lib.rs:542-555
    idx = TETRA_IDX.copy()
    idx[0], idx[1], idx[2] = TETRA_IDX[2], TETRA_IDX[1], TETRA_IDX[0]
    sdf = orc.generate_sdf(TETRA_V, idx, [[0.2, 0.2, 0.05]], "bvh", "raycast")
    assert sdf[0] == np.float32(0.05)


def test_panics_become_status_codes(orc):
    # lib.rs:557-585: bad index, index count not a multiple of 3, NaN query.
    idx = TETRA_IDX.copy()
    idx[0] = 100
    st, _ = orc.generate_sdf(TETRA_V, idx, [[0.2, 0.2, 0.05]], "bvh", "raycast", check=False)
    assert st == 4
    idx = np.append(TETRA_IDX, 0).astype(np.uint32)
    st, _ = orc.generate_sdf(TETRA_V, idx, [[0.2, 0.2, 0.05]], "bvh", "raycast", check=False)
    assert st == 3
    st, _ = orc.generate_sdf(TETRA_V, TETRA_IDX, [[0.0, 0.0, float("nan")]], "bvh", "raycast", check=False)
    assert st == 2


CUBE_V = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 0], [1, 0, 1], [0, 1, 1], [1, 1, 1]],
                  np.float32)
CUBE_IDX = np.array([0, 2, 4, 0, 4, 1, 3, 5, 7, 3, 7, 6, 0, 1, 5, 0, 5, 3, 2, 6, 7, 2, 7, 4, 0, 3, 6, 0, 6, 2,
                     1, 4, 7, 1, 7, 5], np.uint32)


def test_all_acceleration_methods_on_cube(orc):
    # lib.rs:587-683 (Normal methods only, as in the reference)
    inner = [[0.2, 0.2, 0.2], [0.8, 0.2, 0.2], [0.2, 0.8, 0.2], [0.2, 0.2, 0.8], [0.8, 0.8, 0.2],
             [0.8, 0.2, 0.8], [0.2, 0.8, 0.8], [0.8, 0.8, 0.8]]
    outer = [[-0.2, -0.2, -0.2], [1.2, -0.2, -0.2], [-0.2, 1.2, -0.2], [-0.2, -0.2, 1.2], [1.2, 1.2, -0.2],
             [1.2, -0.2, 1.2], [-0.2, 1.2, 1.2], [1.2, 1.2, 1.2]]
    for accel, sign in [("none", "normal"), ("bvh", "normal"), ("rtree", "normal")]:
        sdf = orc.generate_sdf(CUBE_V, CUBE_IDX, inner, accel, sign)
        assert np.all(np.abs(sdf - np.float32(-0.2)) < 1e-6), (accel, sdf)
        sdf = orc.generate_sdf(CUBE_V, CUBE_IDX, outer, accel, sign)
        assert np.all(np.abs(sdf - np.float32(math.sqrt(0.2 * 0.2 * 3))) < 1e-6), (accel, sdf)


def test_query_vector_known_points(orc):
    # rtree_bvh.rs:383-419
    cases = [([0.0, 0.0, 0.0], [0.0, 0.0, 0.0], False), ([0.0, 0.5, 0.0], [0.0, 0.0, 0.0], False),
             ([0.2, 0.2, 0.0], [0.0, 0.0, 0.0], False), ([-0.1, -0.1, 0.2], [0.1, 0.1, -0.2], False),
             ([0.1, -0.1, 0.2], [0.0, 0.1, -0.2], False), ([0.2, 0.2, 0.2], [0.0, 0.0, -0.2], False),
             ([0.2, 0.2, -0.1], [0.0, 0.0, 0.1], True)]
    for p, vec, inside in cases:
        v, ins = orc.query_vector_to_closest_point(TETRA_V, TETRA_IDX, [p])
        assert np.linalg.norm(v[0].astype(np.float64) - np.array(vec)) < 1e-6, (p, v[0])
        if np.linalg.norm(v[0]) > 1e-6:
            assert bool(ins[0]) == inside, p


def test_doc_examples(orc):
    # lib.rs:10-31, lib.rs:342-362, lib.rs:440-461
    v = [[0.5, 1.5, 0.5], [1.0, 2.0, 3.0], [1.0, 3.0, 7.0]]
    assert list(orc.generate_sdf(v, np.array([0, 1, 2], np.uint32), [[0.5, 0.5, 0.5]], "rtree_bvh")) == [1.0]
    v = [[0.0, 1.0, 0.0], [1.0, 2.0, 3.0], [1.0, 3.0, 4.0]]
    assert list(orc.generate_sdf(v, np.array([0, 1, 2], np.uint32), [[0.0, 0.0, 0.0]], "rtree_bvh")) == [1.0]
    # generate/grid.rs:204-231
    v = [[0.5, 1.5, 0.5], [1.0, 2.0, 3.0], [1.0, 3.0, 4.0]]
    first, size = orc.grid_from_bounding_box([0, 0, 0], [10, 10, 10], [10, 10, 10])
    sdf = orc.generate_grid_sdf(v, np.array([0, 1, 2], np.uint32), first, size, [10, 10, 10], "raycast")
    assert sdf[0] == 1.0


def test_generate_grid_equals_none_raycast(orc):
    # generate/grid.rs:693-724: grid Raycast == None(Raycast), bit for bit.
    v = np.array([[0, 1, 0], [1, 2, 3], [1, 3, 4], [2, 0, 0]], np.float32)
    idx = np.array([0, 1, 2, 1, 2, 3], np.uint32)
    first, size = orc.grid_from_bounding_box([0, 0, 0], [5, 5, 5], [5, 5, 5])
    q = [orc.grid_cell_center(first, size, [x, y, z]) for x in range(5) for y in range(5) for z in range(5)]
    sdf = orc.generate_sdf(v, idx, q, "none", "raycast")
    for nt in (1, 4):
        grid = orc.generate_grid_sdf(v, idx, first, size, [5, 5, 5], "raycast", n_threads=nt)
        assert np.array_equal(sdf.view(np.uint32), grid.view(np.uint32))


def _approx_eq_default(a, b):
    # float_cmp::assert_approx_eq! default margin: epsilon = f32::EPSILON, ulps = 4
    a = np.float32(a)
    b = np.float32(b)
    if a == b or abs(a - b) <= np.finfo(np.float32).eps:
        return True
    ai = int(np.array(a).view(np.int32))
    bi = int(np.array(b).view(np.int32))
    return abs(ai - bi) <= 4


def test_topology_encodings(orc):
    # generate/grid.rs:844-901
    first, size = orc.grid_from_bounding_box([0, 0, 0], [5, 5, 5], [25, 25, 25])
    v0, v1, v2, v3 = [0.0, 1.0, 0.0], [1.0, 2.0, 3.0], [1.0, 3.0, 4.0], [2.0, 0.0, 0.0]
    a = orc.generate_grid_sdf([v0, v1, v2, v3], np.array([0, 1, 2, 1, 2, 3, 2, 3, 0], np.uint32), first, size,
                              [25] * 3, "normal")
    b = orc.generate_grid_sdf([v0, v1, v2, v1, v2, v3, v2, v3, v0], None, first, size, [25] * 3, "normal")
    c = orc.generate_grid_sdf([v0, v1, v2, v3], np.array([0, 1, 2, 3, 0], np.uint32), first, size, [25] * 3,
                              "normal", strip=True)
    d = orc.generate_grid_sdf([v0, v1, v2, v3, v0], None, first, size, [25] * 3, "normal", strip=True)
    for other in (b, c, d):
        assert all(_approx_eq_default(x, y) for x, y in zip(a, other))


def test_topology_expansion(orc):
    # lib.rs:161-170 doc: list 0..6 -> (012)(345); strip -> (012)(123)(234)(345)
    st, t = orc.expand_topology(6, None, strip=False)
    assert st == 0 and t.tolist() == [[0, 1, 2], [3, 4, 5]]
    st, t = orc.expand_topology(6, None, strip=True)
    assert st == 0 and t.tolist() == [[0, 1, 2], [1, 2, 3], [2, 3, 4], [3, 4, 5]]
    st, t = orc.expand_topology(4, np.array([0, 1, 2, 3, 0], np.uint16), strip=True)
    assert st == 0 and t.tolist() == [[0, 1, 2], [1, 2, 3], [2, 3, 0]]
    st, _ = orc.expand_topology(7, None, strip=False)
    assert st == 3
    st, t = orc.expand_topology(2, None, strip=True)
    assert st == 0 and len(t) == 0


def test_grid_helpers(orc):
    # grid.rs:200-297
    first, size = orc.grid_from_bounding_box([-1.0, 0.0, 1.0], [0.0, 2.0, 5.0], [2, 2, 2])
    assert first.tolist() == [-0.75, 0.5, 2.0] and size.tolist() == [0.5, 1.0, 2.0]
    first, size = orc.grid_from_bounding_box([0, 0, 0], [1, 1, 1], [2, 2, 2])
    assert orc.grid_snap_point(first, size, [2, 2, 2], [0.4, 0.8, 0.1]) == (True, [0, 1, 0])
    assert orc.grid_snap_point(first, size, [2, 2, 2], [-0.5, 0.8, 0.8]) == (False, [0, 1, 1])
    assert orc.grid_snap_point(first, size, [2, 2, 2], [0.8, 0.8, 0.8]) == (True, [1, 1, 1])
    assert orc.grid_snap_point(first, size, [2, 2, 2], [0.8, 1.5, 0.8]) == (False, [1, 1, 1])
    exp = {(0, 0, 0): [0.25] * 3, (0, 0, 1): [0.25, 0.25, 0.75], (1, 1, 0): [0.75, 0.75, 0.25],
           (1, 1, 1): [0.75] * 3}
    for cell, c in exp.items():
        assert orc.grid_cell_center(first, size, cell).tolist() == c


def test_closest_point_segment_kat(orc):
    # geo.rs:311-323 through the degenerate-triangle path (a == b -> segment a..c)
    a, b = [0.0, 0.0, 0.0], [1.0, 0.0, 0.0]
    assert orc.closest_point_triangle([0.3, 1.0, 0.0], a, a, b).tolist() == [np.float32(0.3), 0.0, 0.0]
    assert orc.closest_point_triangle([10.3, 1.0, 10.0], a, a, b).tolist() == [1.0, 0.0, 0.0]


def test_ray_kat(orc):
    # geo.rs:289-309, the directions that an aligned ray can express
    a, b, c = [0.0, 1.0, 0.0], [1.0, 0.0, 0.0], [0.0, 0.0, 1.0]
    o = [0.2, 0.2, 0.2]
    for axis in range(3):
        assert orc.ray_triangle_intersection_aligned(o, a, b, c, axis) is not None
    # from the far side, every +axis ray points away from the triangle
    assert all(orc.ray_triangle_intersection_aligned([0.5, 0.5, 0.5], a, b, c, ax) is None for ax in range(3))


def _baseline_distance(x0, x1, x2, x3):
    # geo.rs:329-393 (SDFGen-style baseline) in float32, default Point arithmetic
    f = np.float32
    x0, x1, x2, x3 = (np.asarray(v, f) for v in (x0, x1, x2, x3))

    def dot(u, v):
        return f(f(f(u[0] * v[0]) + f(u[1] * v[1])) + f(u[2] * v[2]))

    def dist(u, v):
        d = (u - v).astype(f)
        return f(np.sqrt(dot(d, d)))

    def seg(x0, x1, x2):
        dx = (x2 - x1).astype(f)
        m2 = dot(dx, dx)
        s = f(dot(dx, (x2 - x0).astype(f)) / m2)
        s = f(min(max(s, f(0)), f(1)))
        return dist(x0, (x1 * s + x2 * f(f(1) - s)).astype(f))

    x03, x13, x23 = x0 - x3, x1 - x3, x2 - x3
    m13, m23, d = dot(x13, x13), dot(x23, x23), dot(x13, x23)
    invdet = f(f(1) / max(f(m13 * m23 - d * d), f(1e-30)))
    a, b = dot(x13, x03), dot(x23, x03)
    w23 = f(invdet * f(m23 * a - d * b))
    w31 = f(invdet * f(m13 * b - d * a))
    w12 = f(f(f(1) - w23) - w31)
    if w23 >= 0 and w31 >= 0 and w12 >= 0:
        return dist(x0, ((x1 * w23).astype(f) + (x2 * w31).astype(f) + (x3 * w12).astype(f)).astype(f))
    if w23 > 0:
        return min(seg(x0, x1, x2), seg(x0, x1, x3))
    if w31 > 0:
        return min(seg(x0, x1, x2), seg(x0, x2, x3))
    return min(seg(x0, x1, x3), seg(x0, x2, x3))


def _approx(a, b, ulps, eps):
    a, b = np.float32(a), np.float32(b)
    if a == b or abs(float(a) - float(b)) <= eps:
        return True
    return abs(int(np.array(a).view(np.int32)) - int(np.array(b).view(np.int32))) <= ulps


def test_closest_point_property_and_regressions(orc):
    # geo.rs:225-256 property (1000 cases in [-10, 10]) plus the two saved
    # shrunk cases of proptest-regressions/geo.txt:7-8.
    rng = np.random.default_rng(1234)
    cases = [([0.0, -8.055119, 1.1846914], [0.0, 0.0, 0.0], [0.0, 0.0, 8.367966], [-7.806354, 9.330519, 0.0]),
             ([0.0, -5.8359632, 4.405388], [0.0, 0.9572999, 9.758267], [6.9999175, -4.739112, 7.5462694],
              [0.0, -9.673183, 0.52112055])]
    cases += [tuple(rng.uniform(-10, 10, (4, 3)).astype(np.float32)) for _ in range(1000)]
    for p, a, b, c in cases:
        close = lambda u, v: any(_approx(u[i], v[i], 5, 1e-3) for i in range(3))
        if close(a, b) or close(a, c) or close(b, c):
            continue
        d = orc.point_triangle_distance(p, a, b, c)
        assert not math.isnan(d)
        assert _approx(d, _baseline_distance(p, a, b, c), 5, 1e-3), (p, a, b, c)


def _generic_ray(o, dirv, v0, v1, v2):
    # geo.rs:397-455 in float32
    f = np.float32
    o, dirv, v0, v1, v2 = (np.asarray(x, f) for x in (o, dirv, v0, v1, v2))

    def dot(u, v):
        return f(f(f(u[0] * v[0]) + f(u[1] * v[1])) + f(u[2] * v[2]))

    def cross(u, v):
        return np.array([f(u[1] * v[2] - u[2] * v[1]), f(u[2] * v[0] - u[0] * v[2]), f(u[0] * v[1] - u[1] * v[0])], f)

    n = cross(v1 - v0, v2 - v0)
    nd = dot(n, dirv)
    if abs(nd) < f(0.00001):
        return None
    d = f(-dot(n, v0))
    t = f(-f(dot(n, o) + d) / nd)
    if t < 0:
        return None
    p = (o + (dirv * t).astype(f)).astype(f)
    for e0, e1 in ((v0, v1), (v1, v2), (v2, v0)):
        if dot(n, cross((e1 - e0).astype(f), (p - e0).astype(f))) < 0:
            return None
    return t


def test_ray_property(orc):
    # geo.rs:258-287: aligned test agrees with the generic test on all three axes.
    rng = np.random.default_rng(99)
    mismatch = 0
    for _ in range(1000):
        p, a, b, c = rng.uniform(-10, 10, (4, 3)).astype(np.float32)
        for axis in range(3):
            d = [0.0, 0.0, 0.0]
            d[axis] = 1.0
            g = _generic_ray(p, d, a, b, c)
            h = orc.ray_triangle_intersection_aligned(p, a, b, c, axis)
            if (g is None) != (h is None):
                mismatch += 1
            elif g is not None:
                assert _approx(g, h, 5, 1e-3)
    assert mismatch == 0


def test_compare_distances(orc):
    # lib.rs:315-332
    assert orc.compare_distances(1.0, 2.0) == -1
    assert orc.compare_distances(-1.0, 1.0) == 1  # tie: positive wins
    assert orc.compare_distances(1.0, -1.0) == -1
    assert orc.compare_distances(1.0, 1.0 + 5e-7) == -1  # tie, same sign: plain magnitude order
    assert orc.compare_distances(-1.0, 1.0 + 5e-7) == 1
    assert orc.compare_distances(-0.0, 0.0) == 1
    assert orc.compare_distances(float("nan"), 1.0) == 2
