"""The plane bound that lets the Raycast brute force skip closest points.

`k_brute` (AccelerationMethod::None, Raycast sign) skips a triangle's
closest-point evaluation when its plane bound

    |h| (1 - 2^-13) - 2^-11 (|p|max + |triangle|max),   h = p's distance to the plane,

already exceeds the query's best distance (so the triangle cannot be strictly
nearer), for proper triangles whose angle at
`a` has sin^2 >= 1/200 and whose coordinates stay below 2^30.  That is exact
only if the reference's own f32 distance is never below the bound, whatever
Voronoi region its rounding picks.  These tests check that claim against the
oracle's f32 restatement of geo.rs on adversarial pairs: triangles near the
admission threshold, tiny triangles far from the point, large coordinates,
points close to the plane but far to its side, and points in every region.
CPU only.
"""
import numpy as np
import pytest

import oracle

F = np.float32


def admitted_bound(p, a, b, c):
    """(admitted, bound) as the kernel forms them (float32 normal and
    shape test; the bound itself in float64)."""
    ab, ac = (b - a).astype(F), (c - a).astype(F)
    n = np.array([ab[1] * ac[2] - ab[2] * ac[1], ab[2] * ac[0] - ab[0] * ac[2], ab[0] * ac[1] - ab[1] * ac[0]], F)
    nn2 = F(np.dot(n, n))
    lab2, lac2 = F(np.dot(ab, ab)), F(np.dot(ac, ac))
    vmax = float(np.max(np.abs(np.stack([a, b, c]))))
    proper = not (np.array_equal(a, b) or np.array_equal(b, c) or np.array_equal(a, c))
    ok = proper and vmax < 2.0 ** 30 and nn2 > 0 and F(200.0) * nn2 >= lab2 * lac2
    if not ok:
        return False, -np.inf
    u = n.astype(np.float64) / np.sqrt(float(nn2))
    h = abs(float(np.dot(u, p.astype(np.float64) - a.astype(np.float64))))
    pm = float(np.max(np.abs(p)))
    return True, h * (1 - 2.0 ** -13) - 2.0 ** -11 * (vmax + pm)


def reference_distances(a, b, c, pts):
    v = np.stack([a, b, c]).astype(F)
    return np.abs(oracle.generate_sdf(v, np.array([0, 1, 2], np.uint32), pts.astype(F), "none", "raycast"))


def triangles(rng, n, scale, offset, sin_min=0.07):
    """Random triangles with the angle at `a` above asin(sin_min)."""
    out = []
    while len(out) < n:
        a = rng.normal(size=3) * offset
        e1 = rng.normal(size=3)
        e1 /= np.linalg.norm(e1)
        e2 = rng.normal(size=3)
        e2 -= e1 * np.dot(e1, e2)
        e2 /= np.linalg.norm(e2)
        ang = rng.uniform(np.arcsin(sin_min), np.pi - np.arcsin(sin_min))
        l1, l2 = scale * rng.uniform(0.2, 1.0), scale * rng.uniform(0.2, 1.0)
        b = a + l1 * e1
        c = a + l2 * (np.cos(ang) * e1 + np.sin(ang) * e2)
        out.append(tuple(x.astype(F) for x in (a, b, c)))
    return out


def points_around(rng, a, b, c, dists):
    """Points in every region at the given distances: off the face, beyond each
    edge and vertex, and in the plane far to the side."""
    a64, b64, c64 = (x.astype(np.float64) for x in (a, b, c))
    n = np.cross(b64 - a64, c64 - a64)
    n /= np.linalg.norm(n)
    cen = (a64 + b64 + c64) / 3
    pts = []
    for d in dists:
        for _ in range(4):
            w = rng.dirichlet([1, 1, 1]) * rng.uniform(-0.5, 1.5, 3)
            base = w[0] * a64 + w[1] * b64 + w[2] * c64
            side = rng.normal(size=3)
            side -= n * np.dot(n, side)
            side /= np.linalg.norm(side)
            pts.append(base + n * d * rng.choice([-1, 1]))            # off the plane
            pts.append(cen + side * d + n * d * rng.uniform(-1e-3, 1e-3))  # in the plane, to the side
            pts.append(base + rng.normal(size=3) * d)                 # anywhere
    return np.array(pts)


# (scale, offset, least admitted pairs): where the edges are near the f32 spacing
# of the coordinates (1e-6 at 100, 1e-2 at 1e6) most triangles round to
# degenerate or thin ones, which the shape test rejects
@pytest.mark.parametrize("scale,offset,least", [(1.0, 0.0, 1000), (1.0, 1e3, 1000), (1e-3, 1.0, 1000),
                                                (1e-6, 1.0, 1000), (1e-6, 1e2, 50), (1e3, 1e5, 1000),
                                                (1e-2, 1e6, 50), (1.0, 1e7, 1000)])
def test_reference_distance_never_below_plane_bound(scale, offset, least):
    rng = np.random.default_rng(int(scale * 1e6) % 1000 + int(offset) % 997)
    dists = [scale * f for f in (1e-6, 1e-3, 0.1, 1.0, 10.0, 1e3, 1e5)]
    checked = positive = 0
    for a, b, c in triangles(rng, 40, scale, offset):
        if not np.any(np.cross(b.astype(np.float64) - a, c.astype(np.float64) - a)):
            continue  # rounded to a degenerate triangle: never admitted
        pts = points_around(rng, a, b, c, dists)
        pts = pts[np.all(np.abs(pts) < 2.0 ** 29, axis=1)].astype(F)
        ref = reference_distances(a, b, c, pts)
        for p, d in zip(pts, ref):
            ok, lb = admitted_bound(p, a, b, c)
            if not ok:
                continue
            checked += 1
            positive += lb > 0
            assert d >= lb, (a, b, c, p, d, lb)
    assert checked >= least and positive >= least // 5, (checked, positive)


def test_admission_rejects_slivers_and_degenerate():
    a = np.array([0, 0, 0], F)
    b = np.array([1, 0, 0], F)
    assert not admitted_bound(np.zeros(3, F), a, b, np.array([2, 1e-3, 0], F))[0]  # sin A ~ 5e-4
    assert not admitted_bound(np.zeros(3, F), a, b, b)[0]
    assert not admitted_bound(np.zeros(3, F), a, a, a)[0]
    assert admitted_bound(np.zeros(3, F), a, b, np.array([0, 1, 0], F))[0]
    big = np.array([2.0 ** 31, 0, 0], F)
    assert not admitted_bound(np.zeros(3, F), a + big, b + big, np.array([0, 1, 0], F) + big)[0]
