"""GPU tests of batched grids: m2s_grid_sdf_batch_device, grid plans (CUDA
graphs) and the grid autotuner, through the C ABI.

Bar: every grid of a batch is bit-identical to the same (mesh, grid) computed
alone by m2s_grid_sdf_device — a mesh's result may not depend on the other
meshes in the batch — for both signs, with a plan replayed several times and
after the autotuner changed its launch shape.  The single-grid path itself is
held to the oracle by the grid tests of test_parity_gpu.py.
"""
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


def _torch():
    import torch

    return torch


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _workload(sign, seed=3):
    """Small batch: displaced spheres of several sizes and grids, an
    anisotropic grid, and a coarse sphere in a fine grid (states far beyond the
    first bucket window)."""
    items = synth.batch_meshes(10, seed=seed, subdivs=(1, 2, 3, 4), edges=(8, 16, 24, 40))
    meshes, grids = [], []
    for v, idx, lo, hi, e in items:
        meshes.append(m2s.build_sdf_acceleration(v, T.TriangleList(idx), A.none(sign)))
        grids.append(m2s.Grid.from_bounding_box(lo, hi, [e, e, e]))
    v, idx = synth.icosphere(2)
    meshes.append(m2s.build_sdf_acceleration(v, T.TriangleList(idx), A.none(sign)))
    grids.append(m2s.Grid.new([1.1, -1.1, 1.0], [-0.1, 0.1, -0.25], [22, 23, 9]))
    v, idx = synth.icosphere(1)
    meshes.append(m2s.build_sdf_acceleration(v, T.TriangleList(idx), A.none(sign)))
    grids.append(m2s.Grid.from_bounding_box([-1.3] * 3, [1.3] * 3, [48, 48, 48]))
    return meshes, grids


def _single(mesh, grid, sign):
    torch = _torch()
    out = torch.full((grid.get_total_cell_count(),), float("nan"), dtype=torch.float32, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    mesh.grid_device(grid, sign, out, st)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    return out.cpu().numpy(), m2s.last_grid_stats()


def _batch(meshes, grids, sign):
    torch = _torch()
    off = m2s.grid_offsets(grids)
    out = torch.full((int(off[-1]),), float("nan"), dtype=torch.float32, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    m2s.grid_sdf_batch_device(meshes, grids, sign, out, st)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    return out.cpu().numpy(), off, m2s.last_grid_stats()


@pytest.mark.parametrize("sign", [S.Raycast, S.Normal])
def test_batch_equals_single_grids(sign):
    meshes, grids = _workload(sign)
    got, off, bstats = _batch(meshes, grids, sign)
    rounds = []
    far = 0
    for k, (mesh, grid) in enumerate(zip(meshes, grids)):
        alone, stats = _single(mesh, grid, sign)
        part = got[off[k]:off[k + 1]]
        bad = np.nonzero(bits(part) != bits(alone))[0]
        assert len(bad) == 0, (k, len(bad), part[bad[:4]], alone[bad[:4]])
        rounds.append(stats["rounds"])
        far += stats["far_phases"]
    # the batch relaxes a bucket of every grid in the same round
    assert bstats["rounds"] < sum(rounds), (bstats["rounds"], rounds)
    assert far > 0, "the coarse sphere should send states to the far list"


def test_plan_replays_and_autotune_keep_results():
    torch = _torch()
    sign = S.Raycast
    meshes, grids = _workload(sign, seed=5)
    ref, off, _ = _batch(meshes, grids, sign)
    out = torch.full((int(off[-1]),), float("nan"), dtype=torch.float32, device="cuda")
    st = torch.zeros(1, dtype=torch.int32, device="cuda")
    m2s.set_grid_tuning(wave_cells=30000)  # several waves in one graph
    plan = m2s.GridPlan(meshes, grids, sign, out, st)
    m2s.set_grid_tuning()
    try:
        assert plan.waves > 1
        assert plan.cells == int(off[-1])
        assert plan.device_bytes > 0
        for _ in range(3):
            out.fill_(float("nan"))
            plan.run()
            torch.cuda.synchronize()
            assert np.array_equal(bits(out.cpu().numpy()), bits(ref))
        chosen = plan.autotune()
        assert chosen == plan.blocks and chosen >= 1
        out.fill_(float("nan"))
        plan.run()
        torch.cuda.synchronize()
        assert np.array_equal(bits(out.cpu().numpy()), bits(ref))
        assert int(st.item()) == 0
    finally:
        plan.close()
        m2s.clear_grid_autotune()


def test_launch_shape_never_changes_results():
    sign = S.Raycast
    meshes, grids = _workload(sign, seed=7)
    ref, _, _ = _batch(meshes, grids, sign)
    try:
        # wave size 1 cell: every grid in a job of its own; 1 << 30: the whole batch in one job;
        # blocks per SM, cells per block, wave size, solo rounds (0: every round on every block)
        for bps, cpb, wave, solo in [(1, 2048, 4 << 20, 64), (0, 64, 1, 0), (2, 1 << 20, 1 << 30, 1000),
                                     (0, 2048, 20000, 0), (0, 2048, 1 << 30, 0), (0, 2048, 1 << 30, 10)]:
            m2s.set_grid_tuning(bps, cpb, wave, solo)
            got, _, _ = _batch(meshes, grids, sign)
            assert np.array_equal(bits(got), bits(ref)), (bps, cpb, wave, solo)
    finally:
        m2s.set_grid_tuning()


def test_batch_with_empty_mesh():
    sign = S.Raycast
    v, idx = synth.star(3, seed=1)
    full = m2s.build_sdf_acceleration(v, T.TriangleList(idx), A.none(sign))
    empty = m2s.build_sdf_acceleration(np.zeros((0, 3), np.float32), T.TriangleList(np.zeros(0, np.uint32)),
                                       A.none(sign))
    assert empty is not None and empty.triangle_count == 0
    lo, hi = synth.padded_bbox(v)
    grids = [m2s.Grid.from_bounding_box(lo, hi, [20, 20, 20]), m2s.Grid.from_bounding_box(lo, hi, [8, 9, 10])]
    got, off, _ = _batch([full, empty], grids, sign)
    alone, _ = _single(full, grids[0], sign)
    assert np.array_equal(bits(got[:off[1]]), bits(alone))
    empty_alone, _ = _single(empty, grids[1], sign)
    assert np.array_equal(bits(got[off[1]:]), bits(empty_alone))
    assert np.all(got[off[1]:] == np.finfo(np.float32).max)


def test_batch_rejects_bad_grids():
    torch = _torch()
    v, idx = synth.icosphere(1)
    mesh = m2s.build_sdf_acceleration(v, T.TriangleList(idx), A.none(S.Raycast))
    out = torch.empty(64, dtype=torch.float32, device="cuda")
    bad = m2s.Grid.new([0, 0, 0], [0.1, 0.1, 0.1], [4, 0, 4])
    with pytest.raises(m2s.M2SError) as e:
        m2s.grid_sdf_batch_device([mesh, mesh], [m2s.Grid.new([0, 0, 0], [0.1] * 3, [4, 4, 4]), bad], S.Raycast, out)
    assert e.value.status == 1


def test_many_small_rounds_at_full_occupancy_are_deterministic():
    # coarse spheres in fine grids chain many small rounds (solo runs of block
    # 0 while every other block waits); with as many blocks as fit, results
    # must not depend on the launch shape or on solo runs
    items = synth.batch_meshes(40, seed=21, subdivs=(1, 2, 3), edges=(24, 48, 64, 80))
    sign = S.Raycast
    meshes = [m2s.build_sdf_acceleration(v, T.TriangleList(i), A.none(sign)) for v, i, *_ in items]
    grids = [m2s.Grid.from_bounding_box(lo, hi, [e, e, e]) for _, _, lo, hi, e in items]
    ref = None
    try:
        for bps, cpb, wave, solo in [(0, 2048, 4 << 20, 0), (0, 1, 4 << 20, 64), (0, 1, 1 << 30, 64),
                                     (3, 1, 1 << 20, 227), (0, 64, 4 << 20, 8), (1, 1, 4 << 20, 64)]:
            m2s.set_grid_tuning(bps, cpb, wave, solo)
            got, _, stats = _batch(meshes, grids, sign)
            if ref is None:
                ref = got
            assert np.array_equal(bits(got), bits(ref)), (bps, cpb, wave, solo)
    finally:
        m2s.set_grid_tuning()


def test_grid_barrier_wait_is_bounded():
    # the propagation's grid barrier gives up after its time limit instead of
    # waiting for blocks that never arrive (here: one block fewer than it
    # expects), and the context stays usable
    import time

    L = m2s._lib.lib()
    out = np.zeros(2, np.uint32)
    assert L.m2s_test_grid_barrier(8, 8, out.ctypes.data) == 0
    assert out.tolist() == [8, 0]
    t0 = time.perf_counter()
    assert L.m2s_test_grid_barrier(3, 4, out.ctypes.data) == 0
    waited = time.perf_counter() - t0
    assert out.tolist() == [0, 3]
    assert 1.5 < waited < 30.0, waited
    v, idx = synth.icosphere(2)
    grid = m2s.Grid.from_bounding_box([-1.2] * 3, [1.2] * 3, [24, 24, 24])
    a = m2s.generate_grid_sdf(v, T.TriangleList(idx), grid, S.Raycast)
    b = m2s.generate_grid_sdf(v, T.TriangleList(idx), grid, S.Raycast)
    assert np.array_equal(bits(a), bits(b))
