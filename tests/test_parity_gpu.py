"""GPU parity: the CUDA path (through the C ABI) against the CPU oracle.

Bars, as stated per test:
  * point queries: bit-exact (every method; Rtree and Bvh(Normal) use the
    oracle's pinned tie order, lowest triangle index first);
  * grids: signs exact cell for cell (Raycast); distances are values of real
    triangles (never below the exact nearest distance) and differ from the
    single-heap reference only in a small fraction of cells — the reference's
    own propagation is order-dependent (its 8-thread run differs from its
    1-thread run), and the tests bound the GPU by that envelope.
"""
import numpy as np
import pytest

import mesh_to_sdf_b200 as m2s
from mesh_to_sdf_b200 import synth

pytestmark = pytest.mark.gpu

T = m2s.Topology
A = m2s.AccelerationMethod
S = m2s.SignMethod

ORC_ACCEL = {A.NONE: "none", A.BVH: "bvh", A.RTREE: "rtree", A.RTREE_BVH: "rtree_bvh"}

TETRA_V = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, -1]], np.float32)
TETRA_IDX = np.array([0, 1, 2, 0, 2, 3, 0, 3, 1, 1, 3, 2], np.uint32)


@pytest.fixture(scope="module", autouse=True)
def _device():
    if not m2s.device_available():
        pytest.fail("no sm_100 device: the GPU suite must run on a B200")


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def assert_bit_equal(gpu, ref, what):
    gpu, ref = np.asarray(gpu, np.float32), np.asarray(ref, np.float32)
    assert gpu.shape == ref.shape, what
    bad = np.nonzero(bits(gpu) != bits(ref))[0]
    assert len(bad) == 0, f"{what}: {len(bad)} of {len(gpu)} differ, e.g. idx {bad[:5]} gpu {gpu[bad[:5]]} ref {ref[bad[:5]]}"


def orc_sdf(orc, v, idx, q, am, strip=False):
    return orc.generate_sdf(v, idx, q, ORC_ACCEL[am.kind], int(am.sign), strip=strip)


# ----------------------------------------------------------------- known answers
def test_waterproof_tetra_all_methods(orc):
    # lib.rs:494-524 points, every method, bit-exact against the oracle
    q = np.array([[0, 0, 0], [0.5, 0, 0], [0.2, 0.2, 0], [0.2, 0.2, 0.05], [0.2, 0.2, -0.05], [1, 1, 0.05],
                  [1, 1, -0.05], [1, 1, 0], [0, 0, -1.05], [0, 0, -0.95], [0.5, 0.5, -0.5], [0.5 - 1e-6, 0.5, -0.5],
                  [0.5, 0.5 - 1e-6, -0.5], [0.5, 0.5, -0.5 - 1e-6]], np.float32)
    for am in m2s.ALL_SDF_ACCELERATION_METHODS:
        gpu = m2s.generate_sdf(TETRA_V, T.TriangleList(TETRA_IDX), q, am)
        assert_bit_equal(gpu, orc_sdf(orc, TETRA_V, TETRA_IDX, q, am), repr(am))


def test_hole_and_reversed_normal(orc):
    # lib.rs:526-555
    sdf = m2s.generate_sdf(TETRA_V, T.TriangleList(TETRA_IDX[:-3]), [[1.0, 1.0, -0.05]], A.bvh(S.Raycast))
    assert sdf[0] == np.sqrt(np.float32(0.05 * 0.05 + 0.5 * 0.5 + 0.5 * 0.5), dtype=np.float32)
    idx = TETRA_IDX.copy()
    idx[0], idx[2] = TETRA_IDX[2], TETRA_IDX[0]
    assert m2s.generate_sdf(TETRA_V, T.TriangleList(idx), [[0.2, 0.2, 0.05]], A.bvh(S.Raycast))[0] == np.float32(0.05)


def test_doc_examples():
    # lib.rs:10-31, 342-362, 440-461; generate/grid.rs:204-231
    v = [[0.5, 1.5, 0.5], [1.0, 2.0, 3.0], [1.0, 3.0, 7.0]]
    idx = np.array([0, 1, 2], np.uint32)
    assert m2s.generate_sdf(v, T.TriangleList(idx), [[0.5, 0.5, 0.5]], A.rtree_bvh()).tolist() == [1.0]
    v = [[0.0, 1.0, 0.0], [1.0, 2.0, 3.0], [1.0, 3.0, 4.0]]
    assert m2s.generate_sdf(v, T.TriangleList(idx), [[0.0, 0.0, 0.0]], A.rtree_bvh()).tolist() == [1.0]
    acc = m2s.build_sdf_acceleration(v, T.TriangleList(idx), A.rtree_bvh())
    assert m2s.query_sdf(acc, [[0.0, 0.0, 0.0]]).tolist() == [1.0]
    v = [[0.5, 1.5, 0.5], [1.0, 2.0, 3.0], [1.0, 3.0, 4.0]]
    grid = m2s.Grid.from_bounding_box([0, 0, 0], [10, 10, 10], [10, 10, 10])
    assert m2s.generate_grid_sdf(v, T.TriangleList(idx), grid, S.Raycast)[0] == 1.0


def test_cube_normal_methods():
    # lib.rs:587-683
    cv = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [1, 1, 0], [1, 0, 1], [0, 1, 1], [1, 1, 1]], np.float32)
    ci = np.array([0, 2, 4, 0, 4, 1, 3, 5, 7, 3, 7, 6, 0, 1, 5, 0, 5, 3, 2, 6, 7, 2, 7, 4, 0, 3, 6, 0, 6, 2, 1, 4, 7,
                   1, 7, 5], np.uint32)
    inner = np.array([[a, b, c] for a in (0.2, 0.8) for b in (0.2, 0.8) for c in (0.2, 0.8)], np.float32)
    outer = np.array([[a, b, c] for a in (-0.2, 1.2) for b in (-0.2, 1.2) for c in (-0.2, 1.2)], np.float32)
    for am in (A.none(S.Normal), A.bvh(S.Normal), A.rtree()):
        assert np.all(np.abs(m2s.generate_sdf(cv, T.TriangleList(ci), inner, am) + 0.2) < 1e-6), am
        assert np.all(np.abs(m2s.generate_sdf(cv, T.TriangleList(ci), outer, am) - np.sqrt(0.12)) < 1e-6), am


def test_vector_known_points(orc):
    # rtree_bvh.rs:383-419
    acc = m2s.build_sdf_acceleration(TETRA_V, T.TriangleList(TETRA_IDX), A.rtree_bvh())
    pts = np.array([[0, 0, 0], [0, 0.5, 0], [0.2, 0.2, 0], [-0.1, -0.1, 0.2], [0.1, -0.1, 0.2], [0.2, 0.2, 0.2],
                    [0.2, 0.2, -0.1]], np.float32)
    exp = np.array([[0, 0, 0], [0, 0, 0], [0, 0, 0], [0.1, 0.1, -0.2], [0, 0.1, -0.2], [0, 0, -0.2], [0, 0, 0.1]])
    vec, inside = m2s.query_vector_to_closest_point_rtree_bvh(acc, pts)
    assert np.all(np.linalg.norm(vec - exp, axis=1) < 1e-6)
    assert inside[-1] and not inside[3:6].any()
    ov, oi = orc.query_vector_to_closest_point(TETRA_V, TETRA_IDX, pts)
    assert_bit_equal(vec.reshape(-1), ov.reshape(-1), "vector")
    assert np.array_equal(inside, oi)


# ----------------------------------------------------------------- methods vs oracle
MESHES = {
    "icosphere_s3": lambda: (*synth.icosphere(3), False),
    "star_s4": lambda: (*synth.star(4, seed=3), False),
    "terrain_40_strip": lambda: (*synth.terrain(40, seed=1), True),
}


@pytest.mark.parametrize("mesh", list(MESHES))
def test_every_method_bit_exact(orc, mesh):
    v, idx, strip = MESHES[mesh]()
    q = synth.mixed_points(v, idx if not strip else None, 3000, seed=11) if not strip else \
        synth.uniform_points(3000, *synth.padded_bbox(v), seed=11)
    topo = T.TriangleStrip(idx) if strip else T.TriangleList(idx)
    for am in m2s.ALL_SDF_ACCELERATION_METHODS:
        gpu = m2s.generate_sdf(v, topo, q, am)
        assert_bit_equal(gpu, orc_sdf(orc, v, idx, q, am, strip=strip), f"{mesh} {am!r}")


def _tie_fan(n_rim, seed):
    # A fan around the origin whose triangles all share vertex 0, half of them
    # wound the other way, plus exact duplicates with the opposite winding:
    # a point above the hub is equally far (the shared vertex) from many
    # triangles of both signs, and nearly so from its jittered neighbours, so
    # compare_distances' ties and sign rule decide the fold at every step.
    rng = np.random.default_rng(seed)
    ang = np.sort(rng.uniform(0, 2 * np.pi, n_rim))
    rim = np.stack([np.cos(ang), np.sin(ang), rng.normal(0, 1e-3, n_rim)], 1) * rng.uniform(0.9, 1.1, (n_rim, 1))
    v = np.vstack([[[0, 0, 0]], rim]).astype(np.float32)
    tris = []
    for k in range(n_rim):
        t = [0, 1 + k, 1 + (k + 1) % n_rim]
        tris.append(t if rng.random() < 0.5 else t[::-1])
        if rng.random() < 0.3:
            tris.append(tris[-1][::-1])
    idx = np.array(tris, np.uint32).reshape(-1)
    hub = np.concatenate([rng.normal(0, 1e-6, (600, 2)), rng.choice([-1, 1], (600, 1)) *
                          rng.uniform(1e-5, 0.3, (600, 1))], 1)
    q = np.vstack([hub, rng.uniform(-1.2, 1.2, (400, 3))]).astype(np.float32)
    return v, idx, q


@pytest.mark.parametrize("n_rim", [70, 333])
def test_none_normal_fold_ties(orc, n_rim):
    # default.rs:63-70: the compare_distances fold in triangle order, on both
    # brute-force kernels (a warp per query below 2^17 queries, a thread per
    # query from there); one tile and ragged groups of 32 (n_rim 70), several
    # tiles (n_rim 333)
    v, idx, q = _tie_fan(n_rim, seed=n_rim)
    ref = orc.generate_sdf(v, idx, q, "none", int(S.Normal))
    assert_bit_equal(m2s.generate_sdf(v, T.TriangleList(idx), q, A.none(S.Normal)), ref, "warp per query")
    big = np.tile(q, ((1 << 17) // len(q) + 1, 1))
    gpu = m2s.generate_sdf(v, T.TriangleList(idx), big, A.none(S.Normal))
    assert_bit_equal(gpu, np.tile(ref, (1 << 17) // len(q) + 1), "thread per query")


def test_topology_encodings(orc):
    # generate/grid.rs:844-901 and lib.rs:193-215: u16, u32, no-index list, strips
    v, idx = synth.icosphere(2)
    q = synth.uniform_points(500, [-1.3] * 3, [1.3] * 3, seed=2)
    ref = orc.generate_sdf(v, idx, q, "bvh", "raycast")
    flat = v[idx.astype(np.int64)]
    for topo in (T.TriangleList(idx), T.TriangleList(idx.astype(np.uint16))):
        assert_bit_equal(m2s.generate_sdf(v, topo, q, A.bvh(S.Raycast)), ref, "list")
    assert_bit_equal(m2s.generate_sdf(flat, T.TriangleList(None), q, A.bvh(S.Raycast)), ref, "list none")
    tv, ti = synth.terrain(24, seed=4)
    tq = synth.uniform_points(400, *synth.padded_bbox(tv), seed=5)
    ref = orc.generate_sdf(tv, ti, tq, "rtree", "normal", strip=True)
    assert_bit_equal(m2s.generate_sdf(tv, T.TriangleStrip(ti.astype(np.uint32)), tq, A.rtree()), ref, "strip")
    sv = tv[ti.astype(np.int64)]
    assert_bit_equal(m2s.generate_sdf(sv, T.TriangleStrip(None), tq, A.rtree()), ref, "strip none")


def test_build_query_equals_generate():
    # default.rs:131-150, bvh.rs:216-232, rtree.rs:191-206, rtree_bvh.rs:314-331
    v, idx = synth.star(3, seed=7)
    q = synth.mixed_points(v, idx, 2000, seed=8)
    for am in m2s.ALL_SDF_ACCELERATION_METHODS:
        acc = m2s.build_sdf_acceleration(v, T.TriangleList(idx), am)
        assert_bit_equal(m2s.query_sdf(acc, q), m2s.generate_sdf(v, T.TriangleList(idx), q, am), repr(am))


def test_vector_query_matches_oracle(orc):
    v, idx = synth.star(4, seed=1)
    q = synth.mixed_points(v, idx, 3000, seed=3)
    acc = m2s.build_sdf_acceleration(v, T.TriangleList(idx), A.rtree_bvh())
    vec, inside = m2s.query_vector_to_closest_point_rtree_bvh(acc, q)
    ov, oi = orc.query_vector_to_closest_point(v, idx, q)
    assert_bit_equal(vec.reshape(-1), ov.reshape(-1), "vectors")
    assert np.array_equal(inside, oi)
    sdf = m2s.query_sdf(acc, q)  # rtree_bvh.rs:337-380
    assert np.all(np.abs(np.linalg.norm(vec, axis=1) - np.abs(sdf)) < 1e-3)
    assert np.array_equal(inside, sdf < 0)


def test_large_batch_morton_order(orc):
    # from 2^17 queries the per-thread search runs in Morton order (Bvh(Normal)
    # from 4096); results stay in input order, and an unsorted 20k batch agrees
    v, idx = synth.star(5, seed=2)
    q = synth.mixed_points(v, idx, (1 << 17) + 500, seed=4)
    for n in (20000, len(q)):
        for am in (A.bvh(S.Raycast), A.rtree(), A.rtree_bvh(), A.bvh(S.Normal)):
            assert_bit_equal(m2s.generate_sdf(v, T.TriangleList(idx), q[:n], am), orc_sdf(orc, v, idx, q[:n], am),
                             f"{am!r} {n}")


def test_packet_search_bit_exact(orc):
    # Morton-ordered batches search a warp at a time (always for Bvh(Normal),
    # from 2^19 queries for the others): the same bits as the oracle, with a
    # ragged last warp; the hard pass still takes over-budget lanes
    v, idx = synth.star(3, seed=5)
    q = synth.mixed_points(v, idx, (1 << 19) + 777, seed=9)
    topo = T.TriangleList(idx)
    for am in (A.bvh(S.Raycast), A.rtree(), A.rtree_bvh(), A.bvh(S.Normal)):
        assert_bit_equal(m2s.generate_sdf(v, topo, q, am), orc_sdf(orc, v, idx, q, am), repr(am))
    assert_bit_equal(m2s.generate_sdf(v, topo, q[:5000], A.bvh(S.Normal)),
                     orc_sdf(orc, v, idx, q[:5000], A.bvh(S.Normal)), "Bvh(Normal) 5000")
    acc = m2s.build_sdf_acceleration(v, topo, A.rtree_bvh())
    vec, inside = m2s.query_vector_to_closest_point_rtree_bvh(acc, q)
    ov, oi = orc.query_vector_to_closest_point(v, idx, q)
    assert_bit_equal(vec.reshape(-1), ov.reshape(-1), "vectors")
    assert np.array_equal(inside, oi)
    tv, ti = synth.terrain(40, seed=2)  # a strip of long flat triangles, uniform points
    tq = synth.uniform_points((1 << 19) + 33, *synth.padded_bbox(tv), seed=3)
    for am in (A.rtree(), A.bvh(S.Normal), A.bvh(S.Raycast)):
        assert_bit_equal(m2s.generate_sdf(tv, T.TriangleStrip(ti), tq, am),
                         orc_sdf(orc, tv, ti, tq, am, strip=True), "terrain " + repr(am))
    L = m2s._lib.lib()
    saved = L.m2s_query_budget()
    try:  # a small budget sends many lanes of each warp to the hard pass
        L.m2s_set_query_budget(64)
        assert_bit_equal(m2s.generate_sdf(v, topo, q, A.rtree()), orc_sdf(orc, v, idx, q, A.rtree()), "budget 64")
    finally:
        L.m2s_set_query_budget(saved)


def test_brute_force_morton_order(orc):
    # None visits batches of 2^28 (query, triangle) pairs or more in Morton
    # order (Raycast: chunked over triangles too; Normal here on one warp per
    # query); results stay in input order, bit-exact
    v, idx = synth.star(5, seed=6)
    q = synth.mixed_points(v, idx, 13200, seed=12)
    assert len(q) * (len(idx) // 3) >= 1 << 28
    v4, i4 = synth.star(4, seed=7)  # Normal on the thread kernel, sorted: 2^17+ queries, 2^28+ pairs
    q4 = synth.mixed_points(v4, i4, (1 << 17) + 100, seed=13)
    assert_bit_equal(m2s.generate_sdf(v4, T.TriangleList(i4), q4, A.none(S.Normal)),
                     orc_sdf(orc, v4, i4, q4, A.none(S.Normal)), "Normal, thread kernel")
    for am in (A.none(S.Raycast), A.none(S.Normal)):
        assert_bit_equal(m2s.generate_sdf(v, T.TriangleList(idx), q, am), orc_sdf(orc, v, idx, q, am), repr(am))


def _plane_bound_soup(seed):
    """Triangles that stress the Raycast brute force's plane bound: tiny
    well-shaped ones (edges 1e-4 .. 1e-6) scattered far from the queries,
    slivers on either side of the bound's shape threshold (sin^2 of the angle
    at a near 1/200), and ordinary ones, around offsets 0, 1e3 and 1e5."""
    rng = np.random.default_rng(seed)
    tris = []
    for off in (0.0, 1e3, 1e5):
        for scale, sin_a, n in ((1e-4, 0.5, 300), (1e-6, 0.5, 300), (0.05, 0.069, 300), (0.05, 0.072, 300),
                                (0.05, 0.6, 600)):
            a = rng.normal(size=(n, 3)) * (0.5 + off * 1e-3) + off
            e1 = rng.normal(size=(n, 3))
            e1 /= np.linalg.norm(e1, axis=1, keepdims=True)
            e2 = rng.normal(size=(n, 3))
            e2 -= e1 * np.sum(e1 * e2, axis=1, keepdims=True)
            e2 /= np.linalg.norm(e2, axis=1, keepdims=True)
            ang = np.arcsin(sin_a)
            b = a + scale * e1
            c = a + scale * (np.cos(ang) * e1 + np.sin(ang) * e2)
            tris.append(np.stack([a, b, c], 1))
    v = np.concatenate(tris).reshape(-1, 3).astype(np.float32)
    return v, np.arange(len(v), dtype=np.uint32)


@pytest.mark.parametrize("seed", [21, 22])
def test_none_raycast_plane_bound_adversarial(orc, seed):
    # the brute force skips a triangle's closest point when its plane is
    # already farther than the best distance; on a soup built to break that
    # bound the results must still equal the reference's bit for bit, in the
    # Morton-ordered chunked kernel and in the single-chunk one
    v, idx = _plane_bound_soup(seed)
    rng = np.random.default_rng(seed + 100)
    q = np.concatenate([rng.normal(size=(20000, 3)) * 0.7,
                        rng.normal(size=(10000, 3)) * 0.7 + 1e3,
                        rng.normal(size=(10000, 3)) * 50.0 + 1e5,
                        v[rng.integers(0, len(v), 10000)] + rng.normal(size=(10000, 3)) * 1e-5]).astype(np.float32)
    assert len(q) * (len(idx) // 3) >= 1 << 28  # Morton order, triangle chunks
    am = A.none(S.Raycast)
    ref = orc_sdf(orc, v, idx, q, am)
    assert_bit_equal(m2s.generate_sdf(v, T.TriangleList(idx), q, am), ref, "chunked")
    assert_bit_equal(m2s.generate_sdf(v, T.TriangleList(idx), q[:1500], am), ref[:1500], "one chunk")


def test_query_counting_changes_no_result():
    # profiling runs the counting kernel instantiations: same bits, sane counts
    v, idx = synth.star(4, seed=5)
    q = synth.mixed_points(v, idx, 6000, seed=6)
    for am in (A.bvh(S.Raycast), A.bvh(S.Normal), A.rtree(), A.rtree_bvh()):
        acc = m2s.build_sdf_acceleration(v, T.TriangleList(idx), am)
        plain = m2s.query_sdf(acc, q)
        m2s.set_profiling(True)
        try:
            counted = m2s.query_sdf(acc, q)
            st = m2s.last_query_stats()
        finally:
            m2s.set_profiling(False)
        assert_bit_equal(counted, plain, repr(am))
        assert st["queries"] == len(q), repr(am)
        assert st["search_node_fetches"] >= len(q) and st["search_triangle_tests"] >= len(q), (repr(am), st)
        if am.kind == A.RTREE:
            assert st["sign_node_fetches"] == 0 and st["sign_triangle_tests"] == 0, st
        else:
            assert st["sign_node_fetches"] >= len(q), (repr(am), st)


def test_query_autotune_keeps_results():
    import torch

    v, idx = synth.star(4, seed=12)
    q = synth.mixed_points(v, idx, 20000, seed=13)
    L = m2s._lib.lib()
    saved = L.m2s_query_budget()
    try:
        for am in (A.bvh(S.Raycast), A.rtree(), A.rtree_bvh()):
            acc = m2s.build_sdf_acceleration(v, T.TriangleList(idx), am)
            ref = m2s.query_sdf(acc, q)
            budget, ms = acc.autotune_queries(torch.from_numpy(q).cuda())
            assert budget in acc.QUERY_BUDGETS and L.m2s_query_budget() == budget
            assert all(t > 0 for t in ms.values()), ms
            assert min(ms, key=ms.get) == budget
            for b in (0, 256, 4096):  # the budget moves work between passes, never results
                L.m2s_set_query_budget(b)
                assert_bit_equal(m2s.query_sdf(acc, q), ref, f"{am!r} budget {b}")
    finally:
        L.m2s_set_query_budget(saved)


@pytest.mark.parametrize("n", [700, 9000, 100_000, 150_000, 300_000])
def test_bvh_normal_band_fold_paths(orc, n):
    # Bvh(Normal) folds the tie band of the nearest distance in triangle
    # order: on one warp per query for small batches (700), on one thread per
    # query otherwise, and, below 2^18 queries (9,000; 100,000 and 150,000
    # with the packet search), when a thread's search or fold exceeds the node
    # budget, on one warp in the second pass; from 2^18 (300,000) in one pass.  Every path and every budget (budget 0:
    # one pass, no hand-off) gives the oracle's bits.  The points include many
    # deep inside the star, whose band traversals are long.
    v, idx = synth.star(5, seed=31)
    q = synth.mixed_points(v, idx, n, seed=32, frac_uniform=0.9)
    ref = orc_sdf(orc, v, idx, q, A.bvh(S.Normal))
    acc = m2s.build_sdf_acceleration(v, T.TriangleList(idx), A.bvh(S.Normal))
    L = m2s._lib.lib()
    saved = L.m2s_query_budget()
    try:
        for b in (0, 16, 256, 4096):
            L.m2s_set_query_budget(b)
            assert_bit_equal(m2s.query_sdf(acc, q), ref, f"n {n} budget {b}")
    finally:
        L.m2s_set_query_budget(saved)
        acc.close()


@pytest.mark.parametrize("n", [1000, 12_000])
def test_equidistant_centre_points_warp_stack_fallback(orc, n):
    # Points at and near the centre of a fine icosphere (20,480 triangles) are
    # nearly equidistant from every triangle: an exact search tests most of
    # them, its warp-wide frontier outgrows the warp kernels' 512-entry
    # stacks, and lane 0 finishes the search (or band fold) alone.  1,000
    # points run one warp per query from the start; 12,000 reach the warp
    # pass after the thread pass's node budget.  Every method gives the
    # oracle's bits (the exact centre's axis rays pass through shared edges:
    # the reference's parity rule, followed bit for bit, calls it outside).
    v, idx = synth.icosphere(5)
    rng = np.random.default_rng(41)
    q = np.vstack([np.zeros((1, 3)), rng.normal(0, 1e-3, (63, 3)),
                   rng.uniform(-1.2, 1.2, (n - 64, 3))]).astype(np.float32)
    for am in (A.rtree(), A.rtree_bvh(), A.bvh(S.Raycast), A.bvh(S.Normal)):
        gpu = m2s.generate_sdf(v, T.TriangleList(idx), q, am)
        assert_bit_equal(gpu, orc_sdf(orc, v, idx, q, am), f"n {n} {am!r}")


def test_fp64_error_report(orc):
    # error report: distance error against an FP64 brute force
    v, idx = synth.star(4, seed=9)
    q = synth.mixed_points(v, idx, 4000, seed=10)
    gpu = m2s.generate_sdf(v, T.TriangleList(idx), q, A.rtree_bvh())
    d64, inside64 = orc.generate_sdf_f64(v, idx, q)
    lo, hi = synth.bbox(v)
    diag = float(np.linalg.norm(hi.astype(np.float64) - lo))
    err = np.abs(np.abs(gpu.astype(np.float64)) - d64)
    assert err.max() <= 1e-6 * diag, (err.max(), diag)
    assert np.mean((gpu < 0) != inside64) < 1e-3


# ----------------------------------------------------------------- errors / edge cases
def test_error_statuses():
    bad = TETRA_IDX.copy()
    bad[0] = 100
    with pytest.raises(m2s.M2SError) as e:  # lib.rs:557-566
        m2s.generate_sdf(TETRA_V, T.TriangleList(bad), [[0.2, 0.2, 0.05]], A.bvh(S.Raycast))
    assert e.value.status == 4
    empty = np.zeros(0, np.uint32)
    q = [[0.1, 0.2, 0.3], [1, 1, 1]]
    out = m2s.generate_sdf(TETRA_V, T.TriangleList(empty), q, A.none(S.Raycast))
    assert out.tolist() == [np.finfo(np.float32).max] * 2  # default.rs:56
    for n in (2, 1 << 17):  # Normal folds from f32::MAX too, on both brute-force kernels
        qn = np.tile(np.asarray(q, np.float32), (n // 2, 1))
        assert np.all(m2s.generate_sdf(TETRA_V, T.TriangleList(empty), qn, A.none(S.Normal)) == np.finfo(np.float32).max)
    assert len(m2s.generate_sdf(TETRA_V, T.TriangleList(empty), q, A.rtree_bvh())) == 0  # rtree_bvh.rs:96-97
    assert m2s.build_sdf_acceleration(TETRA_V, T.TriangleList(empty), A.rtree_bvh()) is None
    with pytest.raises(m2s.M2SError) as e:  # rtree.rs:148
        m2s.generate_sdf(TETRA_V, T.TriangleList(empty), q, A.rtree())
    assert e.value.status == 6
    # a single triangle (the LBVH root is a leaf)
    one = m2s.generate_sdf(TETRA_V, T.TriangleList(TETRA_IDX[:3]), q, A.bvh(S.Raycast))
    assert np.all(one > 0)
    # degenerate triangles fall back to segments (geo.rs:73-88)
    deg = np.array([0, 0, 1, 1, 2, 2, 3, 3, 3], np.uint32)
    qq = synth.uniform_points(200, [-1, -1, -2], [2, 2, 1], seed=1)
    for am in m2s.ALL_SDF_ACCELERATION_METHODS:
        m2s.generate_sdf(TETRA_V, T.TriangleList(deg), qq, am)


def test_degenerate_mesh_matches_oracle(orc):
    deg = np.array([0, 0, 1, 1, 2, 2, 3, 3, 3, 0, 1, 2], np.uint32)
    qq = synth.uniform_points(300, [-1, -1, -2], [2, 2, 1], seed=1)
    for am in m2s.ALL_SDF_ACCELERATION_METHODS:
        assert_bit_equal(m2s.generate_sdf(TETRA_V, T.TriangleList(deg), qq, am),
                         orc_sdf(orc, TETRA_V, deg, qq, am), repr(am))


def test_radix_sort_bit_exact_against_stable_sort():
    import torch

    rng = np.random.default_rng(0)
    for n, kb in ((1, 30), (1000, 30), (70001, 30), (1 << 20, 32), (300000, 8)):
        keys = rng.integers(0, 1 << min(kb, 31), n, dtype=np.uint64).astype(np.uint32)
        keys[: n // 3] = keys[n // 2] if n > 2 else keys[: n // 3]  # many duplicates
        vals = np.arange(n, dtype=np.uint32)
        k = torch.from_numpy(keys.view(np.int32)).cuda()
        v = torch.from_numpy(vals.view(np.int32)).cuda()
        m2s.radix_sort_pairs_device(k, v, kb)
        torch.cuda.synchronize()
        order = np.argsort(keys, kind="stable")
        assert np.array_equal(k.cpu().numpy().view(np.uint32), keys[order])
        assert np.array_equal(v.cpu().numpy().view(np.uint32), vals[order])


# ----------------------------------------------------------------- grids
def test_grid_equals_none_raycast():
    # generate/grid.rs:693-724: bit for bit
    v = np.array([[0, 1, 0], [1, 2, 3], [1, 3, 4], [2, 0, 0]], np.float32)
    idx = np.array([0, 1, 2, 1, 2, 3], np.uint32)
    grid = m2s.Grid.from_bounding_box([0, 0, 0], [5, 5, 5], [5, 5, 5])
    gsdf = m2s.generate_grid_sdf(v, T.TriangleList(idx), grid, S.Raycast)
    psdf = m2s.generate_sdf(v, T.TriangleList(idx), grid.cell_centers(), A.none(S.Raycast))
    assert_bit_equal(gsdf, psdf, "grid vs None(Raycast)")


def grid_report(orc, v, idx, grid, sign, strip=False):
    topo = T.TriangleStrip(idx) if strip else T.TriangleList(idx)
    gpu = m2s.generate_grid_sdf(v, topo, grid, sign)
    args = (v, idx, grid.first_cell, grid.cell_size, grid.cell_count, int(sign))
    ref1 = orc.generate_grid_sdf(*args, strip=strip, n_threads=1)
    ref8 = orc.generate_grid_sdf(*args, strip=strip, n_threads=8)
    centers = grid.cell_centers()
    nn = np.abs(orc.generate_sdf(v, idx, centers, "rtree_bvh" if not strip else "rtree", strip=strip))
    return gpu, ref1, ref8, nn


def check_grid(gpu, ref1, ref8, nn, cell, sign, label):
    n = len(gpu)
    a, r = np.abs(gpu), np.abs(ref1)
    # every GPU value is the distance of a real triangle
    assert np.all(a >= nn), label
    # the GPU stays within a cell diagonal of the exact nearest distance
    assert np.all(a - nn <= cell), label
    diff_gpu = np.mean(bits(a) != bits(r))
    diff_ref8 = np.mean(bits(np.abs(ref8)) != bits(r))
    # the reference's own 8-thread heap differs from its 1-thread heap; the GPU
    # schedule must stay within twice that drift (or 2 % of the cells)
    assert diff_gpu <= max(2.0 * diff_ref8, 0.02), (label, diff_gpu, diff_ref8)
    if sign == S.Raycast:
        assert np.array_equal(np.signbit(gpu), np.signbit(ref1)), label
    return diff_gpu, diff_ref8


def test_grid_icosphere_c1_shape(orc):
    # the small grid config: icosphere s3, 32^3 over [-1.2, 1.2]^3, Raycast
    v, idx = synth.icosphere(3)
    grid = m2s.Grid.from_bounding_box([-1.2] * 3, [1.2] * 3, [32, 32, 32])
    gpu, ref1, ref8, nn = grid_report(orc, v, idx, grid, S.Raycast)
    check_grid(gpu, ref1, ref8, nn, float(np.linalg.norm(grid.cell_size)), S.Raycast, "c1")


def test_grid_star(orc):
    v, idx = synth.star(5, seed=0)
    lo, hi = synth.padded_bbox(v)
    grid = m2s.Grid.from_bounding_box(lo, hi, [48, 40, 56])
    gpu, ref1, ref8, nn = grid_report(orc, v, idx, grid, S.Raycast)
    check_grid(gpu, ref1, ref8, nn, float(np.linalg.norm(grid.cell_size)), S.Raycast, "star")
    again = m2s.generate_grid_sdf(v, T.TriangleList(idx), grid, S.Raycast)
    assert_bit_equal(again, gpu, "grid determinism")


def test_grid_terrain_normal(orc):
    v, idx = synth.terrain(48, seed=2)
    lo, hi = synth.padded_bbox(v)
    grid = m2s.Grid.from_bounding_box(lo, hi, [36, 36, 12])
    gpu, ref1, ref8, nn = grid_report(orc, v, idx, grid, S.Normal, strip=True)
    check_grid(gpu, ref1, ref8, nn, float(np.linalg.norm(grid.cell_size)), S.Normal, "terrain")
    same_mag = bits(np.abs(gpu)) == bits(np.abs(ref1))
    flips = np.mean(np.signbit(gpu[same_mag]) != np.signbit(ref1[same_mag]))
    assert flips < 0.01, flips


def test_grid_out_of_bounds_rays(orc):
    # generate/grid.rs:808-840: the grid covers only part of the mesh
    v, idx = synth.star(4, seed=5)
    lo, hi = synth.bbox(v)
    grid = m2s.Grid.from_bounding_box(lo, hi * np.float32(0.5), [32, 32, 32])
    gpu, ref1, ref8, nn = grid_report(orc, v, idx, grid, S.Raycast)
    check_grid(gpu, ref1, ref8, nn, float(np.linalg.norm(grid.cell_size)), S.Raycast, "oob")


def test_grid_continuity():
    # generate/grid.rs:729-804 on a watertight star, bbox grown by 20 %
    v, idx = synth.star(4, seed=6)
    lo, hi = synth.padded_bbox(v, 0.2)
    grid = m2s.Grid.from_bounding_box(lo, hi, [32, 32, 32])
    sdf = m2s.generate_grid_sdf(v, T.TriangleList(idx), grid, S.Raycast).reshape(32, 32, 32)
    size = grid.cell_size
    for axis in range(3):
        a = np.take(sdf, range(31), axis=axis)
        b = np.take(sdf, range(1, 32), axis=axis)
        assert np.all(np.abs(np.abs(a) - np.abs(b)) <= size[axis] * 1.0001)
        flip = np.sign(a) * np.sign(b) < 0
        assert np.all(np.abs(a[flip]) <= size[axis]) and np.all(np.abs(b[flip]) <= size[axis])


def test_grid_negative_and_anisotropic_sizes(orc):
    v, idx = synth.icosphere(2)
    grid = m2s.Grid.new([1.1, -1.1, 1.0], [-0.1, 0.1, -0.25], [22, 23, 9])
    gpu, ref1, ref8, nn = grid_report(orc, v, idx, grid, S.Raycast)
    assert np.array_equal(np.signbit(gpu), np.signbit(ref1))
    assert np.all(np.abs(gpu) >= nn)


def test_grid_tiny_and_flat_shapes(orc):
    # one cell, lines and planes of cells, a grid with a zero extent
    v, idx = synth.icosphere(2)
    for count in ([1, 1, 1], [1, 1, 40], [40, 1, 1], [1, 37, 1], [2, 2, 2], [33, 29, 1]):
        grid = m2s.Grid.from_bounding_box([-1.3] * 3, [1.3] * 3, count)
        for sign in (S.Raycast, S.Normal):
            gpu, ref1, ref8, nn = grid_report(orc, v, idx, grid, sign)
            label = f"{count} {sign!r}"
            check_grid(gpu, ref1, ref8, nn, float(np.linalg.norm(grid.cell_size)), sign, label)
    # a zero cell count with triangles: the crate's seeding clamp (`clamp(0, n - 1)`,
    # generate/grid.rs:400-426) panics; the ABI refuses the grid instead
    empty = m2s.Grid.new([-1.3] * 3, [0.1] * 3, [0, 8, 8])
    with pytest.raises(m2s.M2SError):
        m2s.generate_grid_sdf(v, T.TriangleList(idx), empty, S.Raycast)


def test_grid_coarse_mesh_far_states(orc):
    # a coarse sphere in a fine grid: seeds lie many buckets from the surface and
    # wait in the far list; the result keeps the same envelope as the others
    v, idx = synth.icosphere(1)
    grid = m2s.Grid.from_bounding_box([-1.3] * 3, [1.3] * 3, [40, 40, 40])
    gpu, ref1, ref8, nn = grid_report(orc, v, idx, grid, S.Raycast)
    assert m2s.last_grid_stats()["far_phases"] > 0
    check_grid(gpu, ref1, ref8, nn, float(np.linalg.norm(grid.cell_size)), S.Raycast, "coarse")


def test_grid_solo_rounds_do_not_change_results():
    # small rounds relaxed by one block give the same bits as every block
    # relaxing every round (terrain: thousands of tiny rounds; a coarse sphere)
    cases = [(synth.terrain(64, seed=4), True, S.Normal), (synth.icosphere(1), False, S.Raycast)]
    try:
        for (v, idx), strip, sign in cases:
            lo, hi = synth.padded_bbox(v)
            grid = m2s.Grid.from_bounding_box(lo, hi, [40, 44, 36])
            topo = T.TriangleStrip(idx) if strip else T.TriangleList(idx)
            outs, solo_rounds = [], []
            for solo in (0, 64, 4096):
                m2s.set_grid_tuning(solo_max=solo)
                outs.append(m2s.generate_grid_sdf(v, topo, grid, sign))
                solo_rounds.append(m2s.last_grid_stats()["solo_rounds"])
            assert np.array_equal(bits(outs[0]), bits(outs[1])) and np.array_equal(bits(outs[0]), bits(outs[2]))
            assert solo_rounds[0] == 0 and solo_rounds[1] > 0, solo_rounds
    finally:
        m2s.set_grid_tuning()
