"""The grid propagation's proposal filter changes no bit.

The filtered kernel variant (m2s_set_grid_bound_filter; off by default)
drops a neighbour proposal unevaluated when the triangle's distance bound (its plane and edge lines, with a slack far above f32 rounding)
proves that it cannot beat the cell's value.  These tests run every grid with
the filter on and off and require identical bits, on shapes chosen to stress
the bound: smooth closed meshes, an open terrain strip with zero-area
connector windows, slivers and needles, a coarse mesh whose states reach far
from the surface, grids one or two cells thick (the plain kernel's row units
of three z-neighbours all meet a boundary there), a grid far from the
origin, and the batched kernel.
"""
import numpy as np
import pytest

import mesh_to_sdf_b200 as m2s
from mesh_to_sdf_b200 import synth

pytestmark = pytest.mark.gpu

T = m2s.Topology
S = m2s.SignMethod


@pytest.fixture(scope="module", autouse=True)
def _device():
    if not m2s.device_available():
        pytest.fail("no sm_100 device: the GPU suite must run on a B200")
    yield
    m2s.set_grid_bound_filter(False)


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def slivers(n, seed):
    """A triangle soup around the unit sphere: a third ordinary, a third
    slivers (the third vertex within 1e-5 of the opposite edge's line), a third
    needles (one edge 1e-5 long)."""
    rng = np.random.default_rng(seed)
    c = rng.normal(size=(n, 3))
    c /= np.linalg.norm(c, axis=1, keepdims=True)
    d1 = rng.normal(size=(n, 3)) * 0.05
    d2 = rng.normal(size=(n, 3)) * 0.05
    a, b = c + d1, c - d1
    third = c + d2
    k = np.arange(n) % 3
    mid = (a + b) / 2
    third[k == 1] = mid[k == 1] + rng.normal(size=(int((k == 1).sum()), 3)) * 1e-5
    third[k == 2] = b[k == 2] + rng.normal(size=(int((k == 2).sum()), 3)) * 1e-5
    v = np.stack([a, b, third], 1).reshape(-1, 3).astype(np.float32)
    return v, np.arange(len(v), dtype=np.uint32)


def run_both(v, topo, grid, sign):
    out = []
    stats = []
    for on in (True, False):
        m2s.set_grid_bound_filter(on)
        out.append(m2s.generate_grid_sdf(v, topo, grid, sign))
        stats.append(m2s.last_grid_stats())
    m2s.set_grid_bound_filter(False)
    return out, stats


CASES = {
    "star_s4_raycast": (lambda: synth.star(4, seed=1), False, [72, 80, 64], S.Raycast),
    "star_s4_normal": (lambda: synth.star(4, seed=1), False, [72, 80, 64], S.Normal),
    "icosphere_s1_coarse": (lambda: synth.icosphere(1), False, [56, 56, 56], S.Raycast),
    "terrain_strip_normal": (lambda: synth.terrain(96, seed=3), True, [64, 64, 40], S.Normal),
    "terrain_strip_raycast": (lambda: synth.terrain(96, seed=3), True, [64, 64, 40], S.Raycast),
    "slivers_raycast": (lambda: slivers(3000, 7), False, [60, 60, 60], S.Raycast),
    "slivers_normal": (lambda: slivers(3000, 7), False, [60, 60, 60], S.Normal),
    # one and two cells along z: every row unit of the plain kernel's big
    # rounds meets the grid's z boundary
    "star_s4_flat_z1": (lambda: synth.star(4, seed=4), False, [420, 400, 1], S.Raycast),
    "star_s4_flat_z2": (lambda: synth.star(4, seed=4), False, [300, 320, 2], S.Raycast),
    "star_s4_thin_x": (lambda: synth.star(4, seed=4), False, [2, 300, 320], S.Raycast),
}


@pytest.mark.parametrize("case", list(CASES))
def test_filter_changes_no_bit(case):
    make, strip, count, sign = CASES[case]
    v, idx = make()
    topo = T.TriangleStrip(idx) if strip else T.TriangleList(idx)
    lo, hi = synth.padded_bbox(v)
    grid = m2s.Grid.from_bounding_box(lo, hi, count)
    (on, off), (s_on, s_off) = run_both(v, topo, grid, sign)
    bad = np.nonzero(bits(on) != bits(off))[0]
    assert len(bad) == 0, f"{case}: {len(bad)} cells differ, e.g. {bad[:5]} on {on[bad[:5]]} off {off[bad[:5]]}"
    # the same proposals are made either way; the filter only drops some unevaluated
    assert s_on["neighbour_evals"] == s_off["neighbour_evals"] and s_off["dropped_bound"] == 0
    if min(count) > 2:
        assert s_on["dropped_bound"] > 0, s_on


def test_filter_far_from_origin():
    # coordinates near 1000: the slack scales with the coordinates' magnitude
    v, idx = synth.star(3, seed=2)
    v = (v * np.float32(0.7) + np.float32(1000.0)).astype(np.float32)
    lo, hi = synth.padded_bbox(v)
    grid = m2s.Grid.from_bounding_box(lo, hi, [48, 48, 48])
    for sign in (S.Raycast, S.Normal):
        (on, off), _ = run_both(v, T.TriangleList(idx), grid, sign)
        assert np.array_equal(bits(on), bits(off)), sign


def test_filter_batched_kernel():
    # the batched (many grids) propagation kernel, both signs
    items = synth.batch_meshes(6, seed=3, subdivs=(2, 3, 4), edges=(32, 48, 64))
    meshes = [m2s.build_sdf_acceleration(v, T.TriangleList(i), m2s.AccelerationMethod.none()) for v, i, *_ in items]
    grids = [m2s.Grid.from_bounding_box(lo, hi, [e, e, e]) for _, _, lo, hi, e in items]
    import torch

    n = int(m2s.grid_offsets(grids)[-1])
    try:
        for sign in (S.Raycast, S.Normal):
            outs = []
            for on in (True, False):
                m2s.set_grid_bound_filter(on)
                out = torch.empty(n, dtype=torch.float32, device="cuda")
                m2s.grid_sdf_batch_device(meshes, grids, sign, out)
                torch.cuda.synchronize()
                outs.append(out.cpu().numpy())
            assert np.array_equal(bits(outs[0]), bits(outs[1])), sign
    finally:
        m2s.set_grid_bound_filter(False)
        for m in meshes:
            m.close()
