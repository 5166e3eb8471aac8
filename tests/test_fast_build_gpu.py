"""The fast build (libm2s_fast.so, M2S_BUILD=fast): multiply-adds fused in the
closest-point and distance arithmetic only.  Bars, against the strict build on
the same inputs: every point-query distance within 4 ulp or 1e-6 of the bbox
diagonal and every point-query sign equal; grid Raycast signs equal in every
cell and grid distances within that tolerance in at least 99 % of cells (the
rest are cells where a fused and an unfused distance order two nearly tied
triangles differently; both are real-triangle distances)."""
import os
import subprocess
import sys

import numpy as np
import pytest

import mesh_to_sdf_b200 as m2s
from mesh_to_sdf_b200 import synth

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CASE = r'''
import sys, numpy as np
sys.path.insert(0, ROOT)
import mesh_to_sdf_b200 as m2s
from mesh_to_sdf_b200 import synth
T, A, S = m2s.Topology, m2s.AccelerationMethod, m2s.SignMethod
v, idx = synth.star(4, seed=3)
q = synth.mixed_points(v, idx, 3000, seed=4)
lo, hi = synth.padded_bbox(v)
grid = m2s.Grid.from_bounding_box(lo, hi, [48, 40, 56])
out = {}
for k, am in enumerate(m2s.ALL_SDF_ACCELERATION_METHODS):
    out[f"m{k}"] = m2s.generate_sdf(v, T.TriangleList(idx), q, am)
out["grid"] = m2s.generate_grid_sdf(v, T.TriangleList(idx), grid, S.Raycast)
np.savez(sys.argv[1], diag=np.linalg.norm(hi.astype(np.float64) - lo), **out)
'''


def _run(tmp_path, build):
    path = str(tmp_path / f"{build}.npz")
    env = dict(os.environ, M2S_BUILD=build)
    code = CASE.replace("ROOT", repr(ROOT))
    r = subprocess.run([sys.executable, "-c", code, path], capture_output=True, text=True, timeout=600, env=env,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    return np.load(path)


def test_fast_build_within_tolerance_of_strict(tmp_path):
    if not m2s.device_available():
        pytest.fail("no sm_100 device: the GPU suite must run on a B200")
    strict, fast = _run(tmp_path, "strict"), _run(tmp_path, "fast")
    diag = float(strict["diag"])

    def within(a, b):
        b64 = np.abs(b.astype(np.float64))
        tol = np.maximum(4 * np.spacing(np.abs(b)).astype(np.float64), 1e-6 * diag)
        return np.abs(np.abs(a.astype(np.float64)) - b64) <= tol

    for k in range(len(m2s.ALL_SDF_ACCELERATION_METHODS)):
        a, b = fast[f"m{k}"], strict[f"m{k}"]
        assert np.all(within(a, b)), (k, float(np.max(np.abs(np.abs(a) - np.abs(b)))))
        assert np.array_equal(np.signbit(a), np.signbit(b)), k
    a, b = fast["grid"], strict["grid"]
    assert np.array_equal(np.signbit(a), np.signbit(b))
    assert np.mean(within(a, b)) >= 0.99
    # the fast build really is a different build
    assert not all(np.array_equal(fast[f"m{k}"].view(np.uint32), strict[f"m{k}"].view(np.uint32))
                   for k in range(len(m2s.ALL_SDF_ACCELERATION_METHODS)))
