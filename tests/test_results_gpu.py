"""GPU tests of the result-side rows: the viewer's distance-ordered cell list
(mesh_to_sdf_client/src/sdf.rs:63-71) and the watertightness check
(generate/mesh_check.rs:24-81), through the C ABI.

Bars: the cell order is bit-identical to a stable sort by f32::total_cmp
(NumPy's stable argsort of the total-order keys) and the iso limits are the
exact extremes; the check gives the oracle's verdict and the oracle's first
reported failure (kind and operands) on the crate's own five cases and on
perturbed meshes, and the known answer on a large closed mesh with one face
removed (the oracle's edge loop is quadratic).
"""
import numpy as np
import pytest

import mesh_to_sdf_b200 as m2s
from mesh_to_sdf_b200 import synth

pytestmark = pytest.mark.gpu

T = m2s.Topology
S = m2s.SignMethod

TETRA_V = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, -1]], np.float32)  # mesh_check.rs:89-90
TETRA_F = np.array([0, 1, 2, 0, 2, 3, 0, 3, 1, 1, 3, 2], np.uint32)


@pytest.fixture(scope="module", autouse=True)
def _device():
    if not m2s.device_available():
        pytest.fail("no sm_100 device: the GPU suite must run on a B200")


def total_order(d):
    b = np.ascontiguousarray(d, np.float32).view(np.uint32)
    return np.where(b & 0x80000000, ~b, b | 0x80000000).astype(np.uint32)


def reference_order(d):
    return np.argsort(total_order(d), kind="stable").astype(np.uint32)


def test_cell_order_small_with_ties_and_signed_zeros():
    rng = np.random.default_rng(3)
    d = rng.choice(np.array([-1.5, -0.0, 0.0, 0.25, 2.0, np.inf, -np.inf, 1e-30], np.float32), 5000)
    order, (lo, hi) = m2s.sort_cells_by_distance(d)
    assert np.array_equal(order, reference_order(d))
    assert lo == -np.inf and hi == np.inf


def test_cell_order_of_a_grid():
    v, idx = synth.star(4, seed=9)
    lo, hi = synth.padded_bbox(v)
    grid = m2s.Grid.from_bounding_box(lo, hi, [64, 80, 48])
    d = m2s.generate_grid_sdf(v, T.TriangleList(idx), grid, S.Raycast)
    order, (mn, mx) = m2s.sort_cells_by_distance(d)
    assert np.array_equal(order, reference_order(d))
    assert mn == d.min() and mx == d.max()
    import torch

    dd = torch.from_numpy(d).cuda()
    o = torch.empty(len(d), dtype=torch.int32, device="cuda")
    mm = torch.empty(2, dtype=torch.float32, device="cuda")
    m2s.sort_cells_by_distance_device(dd, o, mm)
    torch.cuda.synchronize()
    assert np.array_equal(o.cpu().numpy().view(np.uint32), order)
    assert mm.cpu().numpy().tolist() == [mn, mx]


def _both(orc, v, f):
    got = m2s.check_mesh_triangle_list(v, f)
    kind, (a, b) = orc.check_mesh_triangle_list(v, f)
    return got, kind, a, b


def _expected_message(v, f, kind, a, b):
    f = np.asarray(f, np.uint32)
    if kind == 0:
        return None
    if kind == 1:
        return "Faces must be a multiple of 3"
    if kind == 2:
        x, y, z = (m2s._rust_debug_f32(c) for c in np.asarray(v, np.float32)[a])
        return f"Duplicate vertex found at ({x}, {y}, {z})"
    if kind == 3:
        return f"Duplicate face found: [{f[3 * a]}, {f[3 * a + 1]}, {f[3 * a + 2]}]"
    if kind == 4:
        return f"Duplicate edge {a} -> {b} - do you have an inverted normal?"
    return f"Mesh is not waterproof - edge {a} -> {b} does not have a corresponding edge {b} -> {a}"


def test_check_crate_cases(orc):
    # mesh_check.rs:92-171, the crate's five tests
    reversed_ = TETRA_F.copy()
    reversed_[0], reversed_[2] = TETRA_F[2], TETRA_F[0]
    cases = [
        (TETRA_V, TETRA_F, 0),
        (np.vstack([TETRA_V, TETRA_V[-1:]]), TETRA_F, 2),
        (TETRA_V, np.concatenate([TETRA_F, TETRA_F[-3:]]), 3),
        (TETRA_V, TETRA_F[:-3], 5),
        (TETRA_V, reversed_, 4),
    ]
    for v, f, want in cases:
        got, kind, a, b = _both(orc, v, f)
        assert kind == want
        assert got == _expected_message(v, f, kind, a, b)
    assert m2s.check_mesh_triangle_list(TETRA_V, TETRA_F[:-1]) == "Faces must be a multiple of 3"
    assert m2s.check_mesh_triangle_list(np.vstack([TETRA_V, TETRA_V[-1:]]), TETRA_F) == \
        "Duplicate vertex found at (0.0, 0.0, -1.0)"


def test_check_matches_oracle_on_perturbed_meshes(orc):
    rng = np.random.default_rng(17)
    base_v, base_f = synth.icosphere(3)  # 1280 faces
    base_v = base_v.copy()
    for trial in range(40):
        v, f = base_v.copy(), base_f.copy().reshape(-1, 3)
        op = trial % 8
        if op == 1:  # drop faces
            f = np.delete(f, rng.choice(len(f), int(rng.integers(1, 4)), replace=False), axis=0)
        elif op == 2:  # flip faces
            k = rng.choice(len(f), int(rng.integers(1, 3)), replace=False)
            f[k] = f[k][:, ::-1]
        elif op == 3:  # repeat a face
            f = np.vstack([f, f[int(rng.integers(len(f)))]])
        elif op == 4:  # repeat a vertex (unused copy), NaNs, signed zeros
            extra = v[int(rng.integers(len(v)))].copy()
            if trial % 16 == 4:
                v[5] = [np.nan, 1, 2]
                extra = np.array([np.float32("nan") * -1, 1, 2], np.float32)  # another NaN payload and sign
            v = np.vstack([v, extra])
        elif op == 5:  # -0.0 and 0.0 are different vertices for the crate
            v = np.vstack([v, [0.0, 0.0, 7.0], [-0.0, 0.0, 7.0]]).astype(np.float32)
        elif op == 6:  # degenerate faces with repeated indices (self-loop edges)
            f = np.vstack([f, [3, 3, 4]])
        elif op == 7:  # shuffle the face order of a broken mesh
            f = np.delete(f, [0, 7], axis=0)
            f = f[rng.permutation(len(f))]
        got, kind, a, b = _both(orc, v, f.reshape(-1))
        assert got == _expected_message(v, f.reshape(-1), kind, a, b), (trial, op, got, kind, a, b)


def test_check_large_closed_mesh_and_known_failure():
    v, f = synth.icosphere(6)  # 81,920 faces
    assert m2s.check_mesh_triangle_list(v, f) is None
    F = f.reshape(-1, 3)
    gone = 12345
    g = np.delete(F, gone, axis=0).reshape(-1)
    # The removed face's three edges lose their reverses: each remaining edge
    # b -> a of the pair fails, and the crate reports the one popped first,
    # the one at the highest position.
    a0, a1, a2 = (int(x) for x in F[gone])
    orphans = {(a1, a0), (a2, a1), (a0, a2)}
    E = g.reshape(-1, 3)
    pos = {}
    for p in range(len(E) * 3):
        fi, k = divmod(p, 3)
        e = (int(E[fi, k]), int(E[fi, (k + 1) % 3]))
        if e in orphans:
            pos[e] = p
    a, b = max(pos, key=pos.get)
    assert m2s.check_mesh_triangle_list(v, g) == \
        f"Mesh is not waterproof - edge {a} -> {b} does not have a corresponding edge {b} -> {a}"
