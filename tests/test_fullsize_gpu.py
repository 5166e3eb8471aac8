"""Full-size properties of the grid path, at the bench's configuration (star
icosphere s6, 81,920 triangles, 256^3 Raycast over the 10 %-padded box) and
the terrain configuration (512 x 512 fBm strip, 384 x 384 x 128 Normal).

The oracle's single heap needs minutes at these sizes, so the bars are the
properties that hold at any size:
  * two runs give the same bits, and so does the batched job (MULTI kernels);
  * every cell holds the distance of a real triangle: |value| is never below
    the exact nearest distance at the cell centre (the GPU's exact nearest
    search, bit-exact against the oracle in test_parity_gpu.py) and within one
    cell diagonal above it (grid.rs:495-558 relaxes the 3x3x3 block);
  * Raycast: every sign equals the restatement's on all host threads (signs
    come from ray parities, independent of the propagation order) and values
    differ from it in under 7.5 % of cells (measured: 6.03 %; the reference's
    own 1- vs 8-thread drift is 1-15 % on the test meshes,
    generate/grid.rs:318-339);
  * Normal (terrain): values differ from the restatement's in under 1 % of
    cells, and every sign difference is accounted for: the two sides hold
    different triangles there (the same triangle gives the same signed value),
    either at exactly the same distance, or within compare_distances' tie
    band (lib.rs:315-332), or — where the propagation order let a different
    triangle win — at most a cell diagonal apart, in a bounded number of cells;
  * the proposal filter (m2s_set_grid_bound_filter) changes no bit.
"""
import os

import numpy as np
import pytest

import mesh_to_sdf_b200 as m2s
from mesh_to_sdf_b200 import synth

pytestmark = pytest.mark.gpu

T = m2s.Topology
A = m2s.AccelerationMethod
S = m2s.SignMethod


@pytest.fixture(scope="module", autouse=True)
def _device():
    if not m2s.device_available():
        pytest.fail("no sm_100 device: the GPU suite must run on a B200")


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def run_grid(v, topo, grid, sign):
    import torch

    mesh = m2s.build_sdf_acceleration(v, topo, A.none(sign))
    out = torch.empty(grid.get_total_cell_count(), dtype=torch.float32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    mesh.grid_device(grid, sign, out, status)
    first = out.cpu().numpy()
    mesh.grid_device(grid, sign, out, status)
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    again = out.cpu().numpy()
    assert np.array_equal(bits(first), bits(again)), "two runs differ"
    return first


def exact_nearest(v, topo, grid, method):
    import torch

    acc = m2s.build_sdf_acceleration(v, topo, method)
    c = torch.from_numpy(grid.cell_centers()).cuda()
    out = torch.empty(len(c), dtype=torch.float32, device="cuda")
    acc.query_device(c, out)
    torch.cuda.synchronize()
    return np.abs(out.cpu().numpy())


def check_real_triangle(d, nn, grid, label):
    a = np.abs(d)
    cell = float(np.linalg.norm(grid.cell_size.astype(np.float64)))
    assert np.all(a >= nn), (label, int(np.sum(a < nn)))
    assert np.all(a.astype(np.float64) - nn <= cell), (label, float(np.max(a.astype(np.float64) - nn)))


def test_bench_grid_full_size(orc):
    v, idx = synth.star(6, seed=0)
    lo, hi = synth.padded_bbox(v, 0.1)
    grid = m2s.Grid.from_bounding_box(lo, hi, [256, 256, 256])
    topo = T.TriangleList(idx)
    d = run_grid(v, topo, grid, S.Raycast)
    check_real_triangle(d, exact_nearest(v, topo, grid, A.rtree_bvh()), grid, "star s6 256^3")
    ref = orc.generate_grid_sdf(v, idx, grid.first_cell, grid.cell_size, grid.cell_count, "raycast",
                                n_threads=os.cpu_count() or 1)
    assert np.array_equal(np.signbit(d), np.signbit(ref))
    assert np.mean(bits(np.abs(d)) != bits(np.abs(ref))) < 0.075
    m2s.set_grid_bound_filter(True)
    try:
        filtered = run_grid(v, topo, grid, S.Raycast)
    finally:
        m2s.set_grid_bound_filter(False)
    assert np.array_equal(bits(filtered), bits(d)), "the proposal filter changed the bench grid"
    # the batched job gives the same bits: with one wave for both grids the
    # 256^3 grid runs through the MULTI kernels beside a small one
    import torch

    small = m2s.Grid.from_bounding_box(lo, hi, [8, 8, 8])
    out = torch.empty(len(d) + small.get_total_cell_count(), dtype=torch.float32, device="cuda")
    meshes = [m2s.build_sdf_acceleration(v, topo, A.none(S.Raycast)) for _ in range(2)]
    m2s.set_grid_tuning(wave_cells=1 << 26)
    try:
        m2s.grid_sdf_batch_device(meshes, [grid, small], S.Raycast, out)
        torch.cuda.synchronize()
    finally:
        m2s.set_grid_tuning()
    assert np.array_equal(bits(out[: len(d)].cpu().numpy()), bits(d))


def approx_eq_band(a, b):
    """float-cmp's approx_eq!(f32, a, b, ulps = 2, epsilon = 1e-6) on
    non-negative magnitudes (lib.rs:321): within 1e-6, or at most 2 ulps apart."""
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    ulps = np.abs(bits(a).astype(np.int64) - bits(b).astype(np.int64))
    return (np.abs(a.astype(np.float64) - b.astype(np.float64)) <= np.float32(1e-6)) | (ulps <= 2)


def sign_breakdown(gpu, ref, cell_diag):
    """Cells whose Normal sign differs, by cause (see the module docstring)."""
    flip = np.signbit(gpu) != np.signbit(ref)
    ga, ra = np.abs(gpu[flip]), np.abs(ref[flip])
    same = bits(ga) == bits(ra)
    band = ~same & approx_eq_band(ga, ra)
    order = ~same & ~band
    gap = np.abs(ga[order].astype(np.float64) - ra[order]) / cell_diag
    return {"sign_differs": int(flip.sum()), "same_distance": int(same.sum()), "tie_band": int(band.sum()),
            "order": int(order.sum()), "order_max_gap_cell_diagonals": float(gap.max()) if len(gap) else 0.0}


def test_terrain_grid_full_size(orc):
    v, idx = synth.terrain(512, seed=0)
    lo, hi = synth.padded_bbox(v, 0.1)
    grid = m2s.Grid.from_bounding_box(lo, hi, [384, 384, 128])
    topo = T.TriangleStrip(idx)
    d = run_grid(v, topo, grid, S.Normal)
    check_real_triangle(d, exact_nearest(v, topo, grid, A.rtree()), grid, "terrain 384x384x128")
    ref = orc.generate_grid_sdf(v, idx, grid.first_cell, grid.cell_size, grid.cell_count, "normal", strip=True,
                                n_threads=os.cpu_count() or 1)
    differ = float(np.mean(bits(np.abs(d)) != bits(np.abs(ref))))
    cell = float(np.linalg.norm(grid.cell_size.astype(np.float64)))
    br = sign_breakdown(d, ref, cell)
    print("terrain vs restatement:", {"value_differs_frac": differ, **br})
    # measured on B200 against the restatement on 16 host threads: values
    # 0.77 %, signs 90,539 (0.48 %: 34,275 at the same distance, 8,464 in the
    # tie band, 47,800 by order, at most 0.039 cell diagonals apart); the
    # restatement's own multi-thread run varies from run to run, so the bars
    # keep some room
    assert differ < 0.012, differ
    # a different winning triangle at a distinct distance stays close (both
    # are propagated values of real triangles) and is rare
    assert br["order_max_gap_cell_diagonals"] <= 0.25, br
    assert br["order"] <= 0.004 * len(d), br
    assert br["sign_differs"] <= 0.007 * len(d), br
