"""GPU tests of m2s_generate_sdf_none_noalloc, the entry point for callers that
cannot allocate device memory (a render loop that cannot afford the device-wide
synchronisation of cudaMalloc, or an application whose device-memory budget is
already committed to its own pool).  It keeps its scratch in a fixed array
inside the library instead of allocating.

Collected last on purpose.  Through the C ABI it checks that:
  * two calls in a row — the second reusing the array the first left behind —
    return exactly what the allocating entry point m2s_generate_sdf returns
    and what the oracle returns (the point-query bar of these tests: bit for
    bit);
  * every index encoding and topology (u32 and u16 lists, strips, no index
    buffer) and both brute-force kernels of each sign (the one-pass kernels
    from 2^17 queries) agree the same way;
  * the crate's panics come back as the same status codes as the allocating
    entry point (an index out of range, a non-finite query, a list length not
    divisible by 3), an empty mesh gives f32::MAX per query, and oversized
    meshes are refused;
  * the calls take nothing from the library's device-memory pool.
"""
import ctypes

import numpy as np
import pytest

import mesh_to_sdf_b200 as m2s
from mesh_to_sdf_b200 import _lib, synth

pytestmark = pytest.mark.gpu

S = m2s.SignMethod
ORC_SIGN = {S.Raycast: "raycast", S.Normal: "normal"}


def _noalloc(v_dev, ni, idx_dev, bits, topo, q_dev, nq, sign, out_dev):
    L = _lib.lib()
    return L.m2s_generate_sdf_none_noalloc(
        ctypes.c_void_p(v_dev.data_ptr()), v_dev.shape[0],
        None if idx_dev is None else ctypes.c_void_p(idx_dev.data_ptr()), ni, bits, topo,
        ctypes.c_void_p(q_dev.data_ptr()), nq, sign, ctypes.c_void_p(out_dev.data_ptr()), None)


def _pool():
    a = np.zeros(2, np.uint64)
    assert _lib.lib().m2s_pool_usage(a.ctypes.data) == 0
    return int(a[0]), int(a[1])


def _bits(a):
    return np.ascontiguousarray(a, np.float32).view(np.uint32)


def _run(v, idx, bits, strip, q, sign):
    """(status, result) of the no-alloc entry point on device copies of the inputs."""
    import torch

    v_dev = torch.from_numpy(np.ascontiguousarray(v, np.float32)).cuda()
    if idx is None:
        i_dev, ni = None, 0
    elif bits == 16:
        i_dev, ni = torch.from_numpy(np.ascontiguousarray(idx, np.uint16).view(np.int16)).cuda(), len(idx)
    else:
        i_dev, ni = torch.from_numpy(np.ascontiguousarray(idx, np.uint32).view(np.int32)).cuda(), len(idx)
    q_dev = torch.from_numpy(np.ascontiguousarray(q, np.float32)).cuda()
    out = torch.full((len(q),), float("nan"), dtype=torch.float32, device="cuda")
    st = _noalloc(v_dev, ni, i_dev, bits, 1 if strip else 0, q_dev, len(q), int(sign), out)
    torch.cuda.synchronize()
    return st, out.cpu().numpy()


def _topology(idx, strip):
    return m2s.Topology.TriangleStrip(idx) if strip else m2s.Topology.TriangleList(idx)


def test_no_alloc_matches_allocating_entry_point_twice(orc):
    assert m2s.device_available()
    cases = [
        (synth.star(4, seed=21), synth.uniform_points(4000, [-1.3] * 3, [1.3] * 3, seed=1), S.Raycast),
        (synth.icosphere(3), synth.uniform_points(2500, [-1.2] * 3, [1.2] * 3, seed=2), S.Normal),
    ]
    for (v, idx), q, sign in cases:
        ref = m2s.generate_sdf(v, m2s.Topology.TriangleList(idx), q, m2s.AccelerationMethod.none(sign))
        exp = orc.generate_sdf(v, idx, q, "none", ORC_SIGN[sign])
        for _ in range(2):  # the second call runs over the first call's leftovers
            st, got = _run(v, idx, 32, False, q, sign)
            assert st == 0, st
            assert np.array_equal(_bits(got), _bits(ref))
            assert np.array_equal(_bits(got), _bits(exp))


ENCODINGS = [("u32_list", 32, False), ("u16_list", 16, False), ("none_list", 0, False), ("u32_strip", 32, True),
             ("u16_strip", 16, True), ("none_strip", 0, True)]


@pytest.mark.parametrize("name,bits,strip", ENCODINGS)
def test_no_alloc_encodings_match_oracle(orc, name, bits, strip):
    v, idx = synth.star(3, seed=23)
    if strip:
        # a strip over the list's vertices in list order (every window is a triangle)
        v = v[idx[:900].astype(np.int64)]
        idx = np.arange(len(v), dtype=np.uint32)
    elif bits == 0:
        v = v[idx.astype(np.int64)]
        idx = np.arange(len(v), dtype=np.uint32)
    q = synth.uniform_points(3000, [-1.3] * 3, [1.3] * 3, seed=3)
    for sign in (S.Raycast, S.Normal):
        st, got = _run(v, None if bits == 0 else idx, bits, strip, q, sign)
        assert st == 0, (name, st)
        topo = _topology(None if bits == 0 else (idx.astype(np.uint16) if bits == 16 else idx), strip)
        ref = m2s.generate_sdf(v, topo, q, m2s.AccelerationMethod.none(sign))
        exp = orc.generate_sdf(v, None if bits == 0 else idx, q, "none", ORC_SIGN[sign], strip=strip)
        assert np.array_equal(_bits(got), _bits(ref)), (name, sign)
        assert np.array_equal(_bits(got), _bits(exp)), (name, sign)


@pytest.mark.parametrize("sign", [S.Raycast, S.Normal])
def test_no_alloc_one_pass_kernels_from_2_17_queries(orc, sign):
    # 2^17 queries and more take the one-pass brute-force kernels (one thread
    # per query, Normal included) instead of the chunked / warp-per-query ones
    v, idx = synth.icosphere(3)
    q = synth.uniform_points((1 << 17) + 4096, [-1.2] * 3, [1.2] * 3, seed=4)
    st, got = _run(v, idx, 32, False, q, sign)
    assert st == 0, st
    ref = m2s.generate_sdf(v, m2s.Topology.TriangleList(idx), q, m2s.AccelerationMethod.none(sign))
    assert np.array_equal(_bits(got), _bits(ref))
    pick = np.random.default_rng(5).choice(len(q), 4000, replace=False)
    exp = orc.generate_sdf(v, idx, q[pick], "none", ORC_SIGN[sign])
    assert np.array_equal(_bits(got[pick]), _bits(exp))


def test_no_alloc_error_statuses_match_allocating_entry_point():
    v, idx = synth.icosphere(1)
    q = synth.uniform_points(100, [-1.2] * 3, [1.2] * 3, seed=6)
    bad_idx = idx.copy()
    bad_idx[7] = len(v) + 3  # out of range (the crate's slice indexing panics)
    bad_q = q.copy()
    bad_q[11, 1] = np.inf  # lib.rs:374-376
    cases = [("index_range", v, bad_idx, q, 4), ("nonfinite_query", v, idx, bad_q, 2),
             ("index_count", v, idx[:-1], q, 3)]
    for name, vv, ii, qq, code in cases:
        st, _ = _run(vv, ii, 32, False, qq, S.Raycast)
        assert st == code, (name, st)
        with pytest.raises(m2s.M2SError) as e:
            m2s.generate_sdf(vv, m2s.Topology.TriangleList(ii), qq, m2s.AccelerationMethod.none())
        assert e.value.status == code, name


def test_no_alloc_empty_mesh_gives_f32_max():
    # default.rs:56: no triangle leaves every query at f32::MAX
    v = np.zeros((0, 3), np.float32)
    q = synth.uniform_points(10, [-1] * 3, [1] * 3, seed=7)
    import torch

    q_dev = torch.from_numpy(q).cuda()
    out = torch.zeros(len(q), dtype=torch.float32, device="cuda")
    v_dev = torch.zeros((1, 3), dtype=torch.float32, device="cuda")
    st = _noalloc(v_dev[:0], 0, None, 0, 0, q_dev, len(q), 0, out)
    assert st == 0, st
    assert np.all(out.cpu().numpy() == np.finfo(np.float32).max)


def test_no_alloc_takes_nothing_from_the_pool():
    v, idx = synth.star(3, seed=24)
    q = synth.uniform_points(5000, [-1.3] * 3, [1.3] * 3, seed=8)
    m2s.generate_sdf(v, m2s.Topology.TriangleList(idx), q, m2s.AccelerationMethod.none())  # the pool exists
    before = _pool()
    for sign in (S.Raycast, S.Normal):
        st, _ = _run(v, idx, 32, False, q, sign)
        assert st == 0
    after = _pool()
    assert after[0] == before[0], (before, after)  # nothing held
    assert after[1] <= before[1], (before, after)  # nothing reserved on top


def test_no_alloc_rejects_meshes_above_its_limit():
    import torch

    n_tris = (1 << 18) + 1
    v_dev = torch.zeros((3 * n_tris, 3), dtype=torch.float32, device="cuda")
    q_dev = torch.zeros((1, 3), dtype=torch.float32, device="cuda")
    out = torch.empty(1, dtype=torch.float32, device="cuda")
    st = _noalloc(v_dev, 0, None, 0, 0, q_dev, 1, 0, out)
    assert st == 1  # M2S_ERR_INVALID_ARGUMENT
    assert b"262144" in _lib.lib().m2s_last_error()
