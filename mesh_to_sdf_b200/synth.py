"""Seeded synthetic meshes and query sets for the benchmark workloads.

All inputs are generated from a seed (numpy PCG64), so every machine builds the
same bytes.  Shapes:

* ``icosphere(s)`` — unit icosphere, 10*4^s + 2 vertices, 20*4^s triangles,
  outward counter-clockwise winding, u32 TriangleList.
* ``star(s, seed)`` — the icosphere with every vertex pushed to radius
  ``1 + sum_k a_k sin(f_k (d_k . u) + phi_k)``: 16 terms, f_k ~ U[1, 6],
  phi_k ~ U[0, 2 pi), d_k random unit vectors, sum |a_k| = 0.15.  The radius
  stays in [0.85, 1.15], so the mesh is a closed, star-shaped surface.
* ``terrain(n, seed)`` — an open n x n height field on [0, 1]^2, height 0.2 *
  fBm (6 octaves of value noise), emitted as ONE u32 TriangleStrip.  Rows are
  joined with two repeated indices, which adds 4 zero-area windows per row
  boundary; the reference processes those windows too (strip windows are never
  re-wound, lib.rs:210-213), so they stay in the mesh.
"""
from __future__ import annotations

import functools

import numpy as np

_ICO_V = None


def _icosahedron():
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array([(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0), (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
                  (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)], np.float64)
    f = np.array([(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11), (1, 5, 9), (5, 11, 4), (11, 10, 2),
                  (10, 7, 6), (7, 1, 8), (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9), (4, 9, 5),
                  (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)], np.int64)
    return v / np.linalg.norm(v, axis=1, keepdims=True), f


@functools.lru_cache(maxsize=8)
def _icosphere_f64_cached(subdiv: int):
    v, f = _icosphere_build(subdiv)
    v.setflags(write=False)
    f.setflags(write=False)
    return v, f


def icosphere_f64(subdiv: int):
    """Unit icosphere in float64: (vertices (V,3), faces (T,3) int64)."""
    v, f = _icosphere_f64_cached(subdiv)
    return v.copy(), f.copy()


def _icosphere_build(subdiv: int):
    v, f = _icosahedron()
    for _ in range(subdiv):
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        uniq, inv = np.unique(e, axis=0, return_inverse=True)
        inv = inv.reshape(-1)
        mid = v[uniq[:, 0]] + v[uniq[:, 1]]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        base = len(v)
        v = np.concatenate([v, mid])
        T = len(f)
        ab, bc, ca = inv[:T] + base, inv[T:2 * T] + base, inv[2 * T:] + base
        a, b, c = f[:, 0], f[:, 1], f[:, 2]
        f = np.concatenate([np.stack([a, ab, ca], 1), np.stack([b, bc, ab], 1), np.stack([c, ca, bc], 1),
                            np.stack([ab, bc, ca], 1)])
    return v, f


def icosphere(subdiv: int):
    v, f = icosphere_f64(subdiv)
    return v.astype(np.float32), f.astype(np.uint32).reshape(-1)


def star_radius(u: np.ndarray, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    K = 16
    freq = rng.uniform(1.0, 6.0, K)
    phase = rng.uniform(0.0, 2.0 * np.pi, K)
    d = rng.normal(size=(K, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    w = rng.uniform(0.2, 1.0, K) * rng.choice([-1.0, 1.0], K)
    amp = 0.15 * w / np.abs(w).sum()
    return 1.0 + (amp[None, :] * np.sin(freq[None, :] * (u @ d.T) + phase[None, :])).sum(1)


def star(subdiv: int, seed: int = 0):
    """Displaced (star-shaped, watertight) icosphere: (vertices f32 (V,3), u32 list indices)."""
    u, f = icosphere_f64(subdiv)
    r = star_radius(u, seed)
    return (u * r[:, None]).astype(np.float32), f.astype(np.uint32).reshape(-1)


def random_rotation(rng) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def _value_noise(x, y, freq, rng_seed):
    rng = np.random.default_rng(rng_seed)
    lat = rng.uniform(-1.0, 1.0, (freq + 2, freq + 2))
    fx, fy = x * freq, y * freq
    ix, iy = np.floor(fx).astype(np.int64), np.floor(fy).astype(np.int64)
    tx, ty = fx - ix, fy - iy
    sx, sy = tx * tx * (3 - 2 * tx), ty * ty * (3 - 2 * ty)
    v00, v10 = lat[iy, ix], lat[iy, ix + 1]
    v01, v11 = lat[iy + 1, ix], lat[iy + 1, ix + 1]
    a = v00 + (v10 - v00) * sx
    b = v01 + (v11 - v01) * sx
    return a + (b - a) * sy


def terrain(n: int = 512, seed: int = 0):
    """Open height field as a single TriangleStrip: (vertices f32 (n*n,3), u32 strip indices)."""
    g = np.linspace(0.0, 1.0, n)
    X, Y = np.meshgrid(g, g)  # Y varies along rows
    h = np.zeros_like(X)
    amp, freq = 1.0, 4
    norm = 0.0
    for o in range(6):
        h += amp * _value_noise(X, Y, freq, seed * 1000 + o)
        norm += amp
        amp *= 0.5
        freq *= 2
    Z = 0.2 * h / norm
    verts = np.stack([X, Y, Z], -1).reshape(-1, 3).astype(np.float32)
    rows = []
    idx = np.arange(n * n, dtype=np.uint32).reshape(n, n)
    for i in range(n - 1):
        row = np.empty(2 * n, np.uint32)
        row[0::2] = idx[i]
        row[1::2] = idx[i + 1]
        if i > 0:
            rows.append(np.array([rows[-1][-1], row[0]], np.uint32))
        rows.append(row)
    return verts, np.concatenate(rows)


def bbox(vertices):
    v = np.asarray(vertices, np.float32).reshape(-1, 3)
    return v.min(0), v.max(0)


def padded_bbox(vertices, frac: float = 0.1):
    """Mesh bounding box grown by `frac` of its extent on every side (float32)."""
    lo, hi = bbox(vertices)
    ext = (hi - lo).astype(np.float32)
    return (lo - np.float32(frac) * ext).astype(np.float32), (hi + np.float32(frac) * ext).astype(np.float32)


def uniform_points(n, lo, hi, seed):
    rng = np.random.default_rng(seed)
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    return (lo + rng.random((n, 3)) * (hi - lo)).astype(np.float32)


def near_surface_points(vertices, indices, n, sigma, seed):
    """Uniform random points on random triangles, jittered by N(0, sigma^2) per axis."""
    rng = np.random.default_rng(seed)
    v = np.asarray(vertices, np.float64).reshape(-1, 3)
    f = np.asarray(indices, np.int64).reshape(-1, 3)
    t = rng.integers(0, len(f), n)
    r1, r2 = rng.random(n), rng.random(n)
    s = np.sqrt(r1)
    a, b, c = v[f[t, 0]], v[f[t, 1]], v[f[t, 2]]
    p = a * (1 - s)[:, None] + b * (s * (1 - r2))[:, None] + c * (s * r2)[:, None]
    return (p + rng.normal(0.0, sigma, (n, 3))).astype(np.float32)


def mixed_points(vertices, indices, n, seed, frac_uniform=0.8, sigma=0.02, pad=0.1):
    lo, hi = padded_bbox(vertices, pad)
    nu = int(round(n * frac_uniform))
    u = uniform_points(nu, lo, hi, seed)
    s = near_surface_points(vertices, indices, n - nu, sigma, seed + 1)
    out = np.concatenate([u, s])
    rng = np.random.default_rng(seed + 2)
    return out[rng.permutation(n)]


BATCH_SUBDIVS = (2, 3, 4, 5, 6)
BATCH_EDGES = (32, 64, 96, 128, 192)


def batch_meshes(n: int = 256, seed: int = 0, subdivs=BATCH_SUBDIVS, edges=BATCH_EDGES):
    """The batched-grid workload: n displaced icospheres (subdivision uniform
    over `subdivs`, so log-uniform in triangle count), each scaled by U[0.5, 2]
    and turned by a uniform random rotation, with a cubic grid of edge drawn
    from `edges` over its bounding box padded 10 %.  Returns a list of
    (vertices f32 (V,3), u32 list indices, grid lo, grid hi, edge)."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        s = int(rng.choice(subdivs))
        scale = rng.uniform(0.5, 2.0)
        rot = random_rotation(rng)
        edge = int(rng.choice(edges))
        u, f = icosphere_f64(s)
        r = star_radius(u, seed * 100003 + k)
        v = ((u * r[:, None]) @ rot.T * scale).astype(np.float32)
        lo, hi = padded_bbox(v)
        out.append((v, f.astype(np.uint32).reshape(-1), lo, hi, edge))
    return out
