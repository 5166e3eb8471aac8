"""The GLB reader of the reference-asset tests (tests/glb.py), on files built
here in memory: node transforms (matrix and translation / rotation / scale)
composed down the hierarchy, u16 and u32 index accessors, an interleaved
vertex buffer with a byte stride, several primitives per mesh, and the
model order (a node's children before its own mesh).  CPU only; needs no
checkout of the reference."""
import json
import struct

import numpy as np
import pytest

import glb


def _pad(b, fill=b"\0"):
    return b + fill * (-len(b) % 4)


def _build(gltf, binary):
    js = _pad(json.dumps(gltf).encode(), b" ")
    bn = _pad(binary)
    body = struct.pack("<II", len(js), 0x4E4F534A) + js + struct.pack("<II", len(bn), 0x004E4942) + bn
    return struct.pack("<III", 0x46546C67, 2, 12 + len(body)) + body


def _quat_matrix(x, y, z, w):
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


@pytest.fixture
def scene(tmp_path):
    rng = np.random.default_rng(5)
    pos_a = rng.normal(size=(5, 3)).astype(np.float32)   # tightly packed, u16 indices
    idx_a = np.array([0, 1, 2, 2, 3, 4], np.uint16)
    pos_b = rng.normal(size=(4, 3)).astype(np.float32)   # interleaved with normals, u32 indices
    nrm_b = rng.normal(size=(4, 3)).astype(np.float32)
    idx_b = np.array([0, 1, 2, 1, 3, 2], np.uint32)
    idx_c = np.array([3, 2, 0], np.uint32)               # the second primitive of mesh B
    inter = np.concatenate([pos_b, nrm_b], axis=1).astype(np.float32)

    chunks, views = [], []
    def add(arr, stride=None):
        off = sum(len(c) for c in chunks)
        raw = _pad(arr.tobytes())
        chunks.append(raw)
        v = {"buffer": 0, "byteOffset": off, "byteLength": arr.nbytes}
        if stride:
            v["byteStride"] = stride
        views.append(v)
        return len(views) - 1
    va, via = add(pos_a), add(idx_a)
    vb, vib, vic = add(inter, stride=24), add(idx_b), add(idx_c)
    acc = [
        {"bufferView": va, "componentType": 5126, "count": 5, "type": "VEC3"},
        {"bufferView": via, "componentType": 5123, "count": 6, "type": "SCALAR"},
        {"bufferView": vb, "byteOffset": 0, "componentType": 5126, "count": 4, "type": "VEC3"},
        {"bufferView": vib, "componentType": 5125, "count": 6, "type": "SCALAR"},
        {"bufferView": vic, "componentType": 5125, "count": 3, "type": "SCALAR"},
    ]
    q = np.array([0.1, -0.3, 0.2, 0.9])
    q /= np.linalg.norm(q)
    mat_b = np.eye(4)
    mat_b[:3, :3] = _quat_matrix(*[0.0, 0.6, 0.0, 0.8])
    mat_b[:3, 3] = [1.0, -2.0, 0.5]
    gltf = {
        "asset": {"version": "2.0"},
        "scene": 0,
        "scenes": [{"nodes": [0]}],
        "nodes": [
            {"mesh": 0, "children": [1], "translation": [0.5, 1.0, -1.0], "rotation": q.tolist(),
             "scale": [2.0, 0.5, 1.5]},
            {"mesh": 1, "matrix": mat_b.T.reshape(-1).tolist()},  # column-major
        ],
        "meshes": [
            {"primitives": [{"attributes": {"POSITION": 0}, "indices": 1}]},
            {"primitives": [{"attributes": {"POSITION": 2}, "indices": 3},
                            {"attributes": {"POSITION": 2}, "indices": 4}]},
        ],
        "accessors": acc,
        "bufferViews": views,
        "buffers": [{"byteLength": sum(len(c) for c in chunks)}],
    }
    path = tmp_path / "scene.glb"
    path.write_bytes(_build(gltf, b"".join(chunks)))
    m_a = np.eye(4)
    m_a[:3, :3] = _quat_matrix(*q) * np.array([2.0, 0.5, 1.5])
    m_a[:3, 3] = [0.5, 1.0, -1.0]
    world_b = m_a @ mat_b
    want_a = pos_a.astype(np.float64) @ m_a[:3, :3].T + m_a[:3, 3]
    want_b = pos_b.astype(np.float64) @ world_b[:3, :3].T + world_b[:3, 3]
    return path, (want_a, idx_a), (want_b, idx_b), (want_b, idx_c)


def test_models_in_order_with_transforms(scene):
    path, a, b, c = scene
    got = glb.models(str(path))
    # node 0's child (mesh 1, two primitives) comes before node 0's own mesh
    assert len(got) == 3
    for (v, i), (wv, wi) in zip(got, [b, c, a]):
        assert v.dtype == np.float32 and i.dtype == np.uint32
        assert np.array_equal(i, wi.astype(np.uint32))
        np.testing.assert_allclose(v, wv, rtol=0, atol=1e-5)


def test_rejects_other_files(tmp_path):
    p = tmp_path / "not.glb"
    p.write_bytes(b"glTF" + struct.pack("<II", 1, 12))
    with pytest.raises(ValueError):
        glb.models(str(p))
