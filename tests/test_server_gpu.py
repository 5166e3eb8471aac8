"""GPU tests of the serving loop (m2s_server_*), through the C ABI.

Bars:
  * every result of a mixed stream (uploads, point and grid requests on
    several meshes and methods, submitted without waiting) is bit-identical to
    the single-request call: query_sdf on a mesh built with the same method,
    grid_device for grids;
  * admission: a request larger than the whole budget is refused at
    submission; requests that fit one at a time but not together all complete,
    and the reserved bytes never exceed the budget;
  * an upload that does not fit evicts an idle mesh, least recently used first;
  * grid requests that queue up beyond one wave (more than 4M cells) are
    split over several waves, and every grid still equals its single-grid
    call bit for bit;
  * continuous batching: a grid request submitted while a large grid's wave
    runs is taken by the other lane at once and completes first, its wave
    overlapping the large one on the device, bit-identical to its single call.
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


def bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def test_mixed_stream_equals_single_calls():
    rng = np.random.default_rng(11)
    items = synth.batch_meshes(4, seed=13, subdivs=(2, 3, 4), edges=(12, 20, 28))
    methods = [A.rtree_bvh(), A.bvh(S.Raycast), A.rtree(), A.none(S.Normal)]
    srv = m2s.Server(8 << 30, point_streams=3)
    try:
        ids, ups = [], []
        for (v, idx, *_), am in zip(items, methods):
            mid, t = srv.submit_upload(v, T.TriangleList(idx), am)
            ids.append(mid)
            ups.append(t)
        jobs = []
        for k in range(24):  # submitted before any upload is waited for
            j = int(rng.integers(len(items)))
            v, idx, lo, hi, e = items[j]
            if k % 3 == 2:
                grid = m2s.Grid.from_bounding_box(lo, hi, [e, e + 1, e + 2])
                sign = S(int(rng.integers(2)))
                out = np.full(grid.get_total_cell_count(), np.nan, np.float32)
                jobs.append(("grid", j, (grid, sign), out, srv.submit_grid(ids[j], grid, sign, out)))
            else:
                q = synth.uniform_points(int(rng.integers(50, 6000)), lo, hi, seed=100 + k)
                out = np.full(len(q), np.nan, np.float32)
                jobs.append(("points", j, q, out, srv.submit_points(ids[j], q, out)))
        for t in ups:
            assert srv.wait(t)[0] == 0
        direct = [m2s.build_sdf_acceleration(v, T.TriangleList(idx), am) for (v, idx, *_), am in zip(items, methods)]
        grid_mesh = [m2s.build_sdf_acceleration(v, T.TriangleList(idx), A.none()) for v, idx, *_ in items]
        import torch

        for kind, j, arg, out, t in jobs:
            status, latency = srv.wait(t)
            assert status == 0 and latency > 0
            if kind == "points":
                ref = m2s.query_sdf(direct[j], arg)
            else:
                grid, sign = arg
                d = torch.empty(grid.get_total_cell_count(), dtype=torch.float32, device="cuda")
                grid_mesh[j].grid_device(grid, sign, d)
                ref = d.cpu().numpy()
            assert np.array_equal(bits(out), bits(ref)), (kind, j)
        st = srv.stats()
        assert st["uploads"] == 4 and st["point_requests"] == 16 and st["grid_requests"] == 8
        assert st["failed"] == 0 and st["grid_batches"] >= 1 and st["queued"] == 0
    finally:
        srv.close()


def test_budget_admission():
    v, idx = synth.star(3, seed=2)
    lo, hi = synth.padded_bbox(v)
    budget = 96 << 20
    srv = m2s.Server(budget)
    try:
        mid, t = srv.submit_upload(v, T.TriangleList(idx), A.rtree_bvh())
        assert srv.wait(t)[0] == 0
        big = m2s.Grid.from_bounding_box(lo, hi, [256, 256, 256])  # its workspace alone exceeds the budget
        with pytest.raises(m2s.M2SError) as e:
            srv.submit_grid(mid, big, S.Raycast, np.empty(big.get_total_cell_count(), np.float32))
        assert e.value.status == 8
        # each fits alone, not all at once: admission runs them as memory frees
        grid = m2s.Grid.from_bounding_box(lo, hi, [64, 64, 64])
        q = synth.uniform_points(400_000, lo, hi, seed=3)
        outs, tickets = [], []
        for k in range(6):
            if k % 2:
                o = np.empty(grid.get_total_cell_count(), np.float32)
                tickets.append(srv.submit_grid(mid, grid, S.Raycast, o))
            else:
                o = np.empty(len(q), np.float32)
                tickets.append(srv.submit_points(mid, q, o))
            outs.append(o)
        for t in tickets:
            assert srv.wait(t)[0] == 0
        for k in range(2, 6):
            assert np.array_equal(bits(outs[k]), bits(outs[k - 2]))
        st = srv.stats()
        assert 0 < st["peak_reserved_bytes"] <= budget
    finally:
        srv.close()


def test_eviction_and_errors():
    meshes = [synth.star(3, seed=s) for s in (4, 5, 6)]
    # two resident meshes of this size (0.2 MB each) plus one build reservation
    # (1.48 MB) fit, three do not
    srv = m2s.Server(1_800_000)
    try:
        ids = []
        for v, idx in meshes:
            mid, t = srv.submit_upload(v, T.TriangleList(idx), A.rtree_bvh())
            assert srv.wait(t)[0] == 0
            ids.append(mid)
        st = srv.stats()
        assert st["evictions"] >= 1 and st["resident_meshes"] < 3
        with pytest.raises(m2s.M2SError):  # the least recently used mesh is gone
            srv.submit_points(ids[0], np.zeros((4, 3), np.float32), np.empty(4, np.float32))
        q = np.zeros((4, 3), np.float32)
        q[1, 2] = np.nan
        with pytest.raises(m2s.M2SError) as e:
            srv.submit_points(ids[2], q, np.empty(4, np.float32))
        assert e.value.status == 2
        with pytest.raises(m2s.M2SError):
            srv.submit_points(12345, np.zeros((4, 3), np.float32), np.empty(4, np.float32))
    finally:
        srv.close()


def test_grid_backlog_spans_batches():
    v, idx = synth.star(4, seed=21)
    lo, hi = synth.padded_bbox(v)
    srv = m2s.Server(64 << 30, point_streams=2)
    import torch

    try:
        mid, t = srv.submit_upload(v, T.TriangleList(idx), A.rtree_bvh())
        assert srv.wait(t)[0] == 0
        # 12 grids of 96^3..176^3 (about 32M cells): more than one batch of four
        # 4M-cell waves, submitted without waiting
        edges = [96, 176, 128, 160, 112, 144, 176, 96, 128, 160, 144, 112]
        jobs = []
        for k, e in enumerate(edges):
            grid = m2s.Grid.from_bounding_box(lo, hi, [e, e - 8, e + 8])
            sign = S.Normal if k % 4 == 3 else S.Raycast
            out = np.full(grid.get_total_cell_count(), np.nan, np.float32)
            jobs.append((grid, sign, out, srv.submit_grid(mid, grid, sign, out)))
        single = m2s.build_sdf_acceleration(v, T.TriangleList(idx), A.none())
        for grid, sign, out, t in jobs:
            assert srv.wait(t)[0] == 0
            d = torch.empty(grid.get_total_cell_count(), dtype=torch.float32, device="cuda")
            single.grid_device(grid, sign, d)
            assert np.array_equal(bits(out), bits(d.cpu().numpy()))
        st = srv.stats()
        assert st["grid_requests"] == len(edges) and st["failed"] == 0
        assert st["grid_batches"] >= 8  # waves of at most 4M cells
    finally:
        srv.close()


def test_grid_request_admitted_while_a_wave_runs():
    import time

    import torch

    v, idx = synth.star(4, seed=22)
    lo, hi = synth.padded_bbox(v)
    srv = m2s.Server(64 << 30, point_streams=2)
    try:
        mid, t = srv.submit_upload(v, T.TriangleList(idx), A.rtree_bvh())
        assert srv.wait(t)[0] == 0
        # a 256^3 grid (a wave of its own on one lane), then a small grid while it runs:
        # the free lane takes the small one at once and both run on the device together
        big = m2s.Grid.from_bounding_box(lo, hi, [256, 256, 256])
        bout = np.full(big.get_total_cell_count(), np.nan, np.float32)
        t_big = time.perf_counter()
        tb = srv.submit_grid(mid, big, S.Raycast, bout)
        time.sleep(0.002)
        small = m2s.Grid.from_bounding_box(lo, hi, [48, 48, 48])
        sout = np.full(small.get_total_cell_count(), np.nan, np.float32)
        t_small = time.perf_counter()
        ts = srv.submit_grid(mid, small, S.Raycast, sout)
        st, lat_small = srv.wait(ts)
        assert st == 0
        st, lat_big = srv.wait(tb)
        assert st == 0
        # completion = submission + the latency the server measured
        assert t_small + lat_small < t_big + lat_big, (t_small - t_big, lat_small, lat_big)
        single = m2s.build_sdf_acceleration(v, T.TriangleList(idx), A.none())
        for grid, out in ((small, sout), (big, bout)):
            d = torch.empty(grid.get_total_cell_count(), dtype=torch.float32, device="cuda")
            single.grid_device(grid, S.Raycast, d)
            assert np.array_equal(bits(out), bits(d.cpu().numpy()))
        st = srv.stats()
        assert st["grid_requests"] == 2 and st["failed"] == 0 and st["grid_batches"] == 2
    finally:
        srv.close()
