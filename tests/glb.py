"""A small reader of binary glTF (.glb) files, for the tests that run the
reference's own asset checks (the reference loads its meshes with the crate
easy-gltf 1.1.2, `easy_gltf::load(path)[0].models[i]`).

It reads what those checks need and nothing more: the JSON and BIN chunks,
each triangle primitive's POSITION (float32 VEC3) and index (u8/u16/u32
SCALAR) accessors, and the transforms of the nodes above the mesh (matrix or
translation / rotation / scale), applied to the positions; skins are not
applied.  One model per primitive, in a depth-first walk of the first scene
that visits a node's children before the node's own mesh.
"""
import json
import struct

import numpy as np

_COMPONENT = {5121: np.uint8, 5123: np.uint16, 5125: np.uint32, 5126: np.float32}
_WIDTH = {"SCALAR": 1, "VEC2": 2, "VEC3": 3, "VEC4": 4, "MAT4": 16}


def _chunks(data):
    magic, version, length = struct.unpack_from("<III", data, 0)
    if magic != 0x46546C67 or version != 2:
        raise ValueError("not a glTF 2.0 binary file")
    off, js, binary = 12, None, None
    while off < length:
        clen, ctype = struct.unpack_from("<II", data, off)
        body = data[off + 8: off + 8 + clen]
        if ctype == 0x4E4F534A:  # JSON
            js = json.loads(body)
        elif ctype == 0x004E4942:  # BIN
            binary = body
        off += 8 + clen
    return js, binary


def _accessor(js, binary, index):
    acc = js["accessors"][index]
    view = js["bufferViews"][acc["bufferView"]]
    dtype = np.dtype(_COMPONENT[acc["componentType"]])
    width = _WIDTH[acc["type"]]
    start = view.get("byteOffset", 0) + acc.get("byteOffset", 0)
    stride = view.get("byteStride", 0) or dtype.itemsize * width
    count = acc["count"]
    raw = np.frombuffer(binary, np.uint8, count=stride * (count - 1) + dtype.itemsize * width, offset=start)
    rows = np.lib.stride_tricks.as_strided(raw, shape=(count, dtype.itemsize * width), strides=(stride, 1))
    return np.ascontiguousarray(rows).view(dtype).reshape(count, width)


def _local(node):
    if "matrix" in node:
        return np.array(node["matrix"], np.float64).reshape(4, 4).T  # column-major
    t = np.array(node.get("translation", [0, 0, 0]), np.float64)
    x, y, z, w = node.get("rotation", [0, 0, 0, 1])
    s = np.array(node.get("scale", [1, 1, 1]), np.float64)
    r = np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                  [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                  [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
    m = np.eye(4)
    m[:3, :3] = r * s
    m[:3, 3] = t
    return m


def models(path):
    """[(vertices float32 (n, 3), indices uint32 (3t,))] in scene order."""
    with open(path, "rb") as f:
        js, binary = _chunks(f.read())
    out = []

    def walk(i, parent):
        node = js["nodes"][i]
        world = parent @ _local(node)
        for c in node.get("children", []):
            walk(c, world)
        for prim in js["meshes"][node["mesh"]]["primitives"] if "mesh" in node else []:
            if prim.get("mode", 4) != 4:
                raise ValueError("only triangle lists are read")
            pos = _accessor(js, binary, prim["attributes"]["POSITION"]).astype(np.float64)
            if not np.array_equal(world, np.eye(4)):
                pos = pos @ world[:3, :3].T + world[:3, 3]
            idx = _accessor(js, binary, prim["indices"]).reshape(-1).astype(np.uint32)
            out.append((pos.astype(np.float32), idx))

    scene = js["scenes"][js.get("scene", 0)]
    for root in scene["nodes"]:
        walk(root, np.eye(4))
    return out
