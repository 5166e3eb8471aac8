"""GPU test of m2s_generate_sdf_none_noalloc, the entry point for callers that
cannot allocate device memory (a render loop that cannot afford the device-wide
synchronisation of cudaMalloc, or an application whose device-memory budget is
already committed to its own pool).  It keeps its scratch in a fixed array
inside the library instead of allocating.

Collected last on purpose: it checks, through the C ABI, that two calls in a
row — the second reusing the array the first left behind — return exactly what
the allocating entry point m2s_generate_sdf returns (the point-query bar of
these tests: bit for bit), and that oversized meshes are refused.
"""
import ctypes

import numpy as np
import pytest

import mesh_to_sdf_b200 as m2s
from mesh_to_sdf_b200 import _lib, synth

pytestmark = pytest.mark.gpu


def _noalloc(v_dev, ni, idx_dev, bits, topo, q_dev, nq, sign, out_dev):
    L = _lib.lib()
    return L.m2s_generate_sdf_none_noalloc(
        ctypes.c_void_p(v_dev.data_ptr()), v_dev.shape[0],
        None if idx_dev is None else ctypes.c_void_p(idx_dev.data_ptr()), ni, bits, topo,
        ctypes.c_void_p(q_dev.data_ptr()), nq, sign, ctypes.c_void_p(out_dev.data_ptr()), None)


def test_no_alloc_matches_allocating_entry_point_twice():
    import torch

    assert m2s.device_available()
    cases = [
        (synth.star(4, seed=21), synth.uniform_points(4000, [-1.3] * 3, [1.3] * 3, seed=1), m2s.SignMethod.Raycast),
        (synth.icosphere(3), synth.uniform_points(2500, [-1.2] * 3, [1.2] * 3, seed=2), m2s.SignMethod.Normal),
    ]
    for (v, idx), q, sign in cases:  # two calls in a row, the second over the first's leftovers
        v_dev = torch.from_numpy(np.ascontiguousarray(v)).cuda()
        i_dev = torch.from_numpy(idx.astype(np.int32)).cuda()
        q_dev = torch.from_numpy(np.ascontiguousarray(q)).cuda()
        out = torch.full((len(q),), float("nan"), dtype=torch.float32, device="cuda")
        st = _noalloc(v_dev, len(idx), i_dev, 32, 0, q_dev, len(q), int(sign), out)
        assert st == 0, st
        ref = m2s.generate_sdf(v, m2s.Topology.TriangleList(idx), q, m2s.AccelerationMethod.none(sign))
        got = out.cpu().numpy()
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_no_alloc_rejects_meshes_above_its_limit():
    import torch

    n_tris = (1 << 18) + 1
    v_dev = torch.zeros((3 * n_tris, 3), dtype=torch.float32, device="cuda")
    q_dev = torch.zeros((1, 3), dtype=torch.float32, device="cuda")
    out = torch.empty(1, dtype=torch.float32, device="cuda")
    st = _noalloc(v_dev, 0, None, 0, 0, q_dev, 1, 0, out)
    assert st == 1  # M2S_ERR_INVALID_ARGUMENT
    assert b"262144" in _lib.lib().m2s_last_error()
