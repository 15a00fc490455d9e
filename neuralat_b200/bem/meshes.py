"""Synthetic boundary meshes and right-hand sides for the BEM workloads.

Icospheres (optionally anisotropically scaled, rotated or radially perturbed),
smoothed complex Gaussian Neumann fields and listener points on a sphere.  All
randomness is seeded through ``numpy.random.default_rng``.

Vertex and triangle numbering is locality-preserving: triangles come out in
the recursive-subdivision order (the four children of a face are adjacent)
and vertices are renumbered by first appearance in that order, so that
neighbouring triangles touch nearby matrix rows and columns.
"""
from __future__ import annotations

import math

import numpy as np


def _icosahedron():
    t = (1.0 + math.sqrt(5.0)) / 2.0
    v = np.array(
        [[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0],
         [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
         [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]], dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array(
        [[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11],
         [1, 5, 9], [5, 11, 4], [11, 10, 2], [10, 7, 6], [7, 1, 8],
         [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9],
         [4, 9, 5], [2, 4, 11], [6, 2, 10], [8, 6, 7], [9, 8, 1]], dtype=np.int64)
    return v, f


def icosphere(subdivisions: int, radius: float = 1.0):
    """Unit icosphere scaled to ``radius``: (V, 3) float64, (T, 3) int32.

    V = 10*4^s + 2, T = 20*4^s, outward-oriented faces.
    """
    verts, faces = _icosahedron()
    vlist = [tuple(p) for p in verts]
    for _ in range(subdivisions):
        cache = {}

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            idx = cache.get(key)
            if idx is None:
                p = (np.asarray(vlist[a]) + np.asarray(vlist[b])) * 0.5
                p /= np.linalg.norm(p)
                vlist.append(tuple(p))
                idx = len(vlist) - 1
                cache[key] = idx
            return idx

        nf = np.empty((faces.shape[0] * 4, 3), dtype=np.int64)
        for n, (a, b, c) in enumerate(faces):
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            nf[4 * n + 0] = (a, ab, ca)
            nf[4 * n + 1] = (ab, b, bc)
            nf[4 * n + 2] = (ab, bc, ca)
            nf[4 * n + 3] = (ca, bc, c)
        faces = nf
    v = np.asarray(vlist, dtype=np.float64)
    # renumber vertices by first appearance in triangle order (locality)
    order = -np.ones(v.shape[0], dtype=np.int64)
    nxt = 0
    for idx in faces.reshape(-1):
        if order[idx] < 0:
            order[idx] = nxt
            nxt += 1
    newv = np.empty_like(v)
    newv[order] = v
    faces = order[faces]
    # orient outward
    p0, p1, p2 = newv[faces[:, 0]], newv[faces[:, 1]], newv[faces[:, 2]]
    n = np.cross(p1 - p0, p2 - p0)
    flip = np.einsum("ij,ij->i", n, p0 + p1 + p2) < 0
    faces[flip] = faces[flip][:, [0, 2, 1]]
    return newv * radius, faces.astype(np.int32)


def random_rotation(rng) -> np.ndarray:
    q = rng.standard_normal(4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([
        [a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
        [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
        [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def vertex_neighbours(nv: int, triangles) -> list:
    nb = [set() for _ in range(nv)]
    for a, b, c in np.asarray(triangles):
        nb[a].update((b, c)); nb[b].update((a, c)); nb[c].update((a, b))
    return [np.fromiter(s, dtype=np.int64) for s in nb]


def smoothed_gaussian_field(nv: int, triangles, m: int, seed: int, passes: int = 5) -> np.ndarray:
    """m complex fields, i.i.d. N(0,1) real+imag per vertex, then `passes`
    umbrella-Laplacian smoothing steps x <- x + 1/2 (mean_neighbours(x) - x).
    Returns (nv, m) complex128."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((nv, m)) + 1j * rng.standard_normal((nv, m))
    tri = np.asarray(triangles, dtype=np.int64)
    # sparse umbrella operator via edge lists
    e = np.concatenate([tri[:, [0, 1]], tri[:, [1, 2]], tri[:, [2, 0]]])
    e = np.unique(np.sort(e, axis=1), axis=0)
    i = np.concatenate([e[:, 0], e[:, 1]])
    j = np.concatenate([e[:, 1], e[:, 0]])
    deg = np.bincount(i, minlength=nv).astype(np.float64)
    for _ in range(passes):
        s = np.zeros_like(x)
        np.add.at(s, i, x[j])
        x = x + 0.5 * (s / deg[:, None] - x)
    return x


def sphere_points(n: int, radius: float, seed: int) -> np.ndarray:
    """n points uniform on a sphere (normalised Gaussian 3-vectors)."""
    rng = np.random.default_rng(seed)
    p = rng.standard_normal((n, 3))
    p /= np.linalg.norm(p, axis=1, keepdims=True)
    return p * radius


def wavenumber(freq_hz: float, c: float = 343.0) -> float:
    return 2.0 * math.pi * freq_hz / c


def vertex_normals(vertices, triangles) -> np.ndarray:
    v = np.asarray(vertices, np.float64)
    t = np.asarray(triangles, np.int64)
    fn = np.cross(v[t[:, 1]] - v[t[:, 0]], v[t[:, 2]] - v[t[:, 0]])
    vn = np.zeros_like(v)
    for a in range(3):
        np.add.at(vn, t[:, a], fn)
    return vn / np.linalg.norm(vn, axis=1, keepdims=True)


# ---- the named workloads ---------------------------------------------------

def plain_small():
    """Icosphere s3, r 0.1 m, k at 1 kHz, monopole Neumann data, 256 listeners at r 0.5 m."""
    v, t = icosphere(3, 0.1)
    k = wavenumber(1000.0)
    pts = sphere_points(256, 0.5, seed=0)
    return dict(vertices=v, triangles=t, k=k, points=pts)


def precision_large(m: int = 8):
    """Icosphere s5, r 0.15 m, axes scaled by U[0.7, 1.3] (seed 1), k at 4 kHz,
    m smoothed complex Gaussian Neumann fields (seed 2), 256 listeners at r 0.5 m (seed 0)."""
    v, t = icosphere(5, 0.15)
    rng = np.random.default_rng(1)
    v = v * rng.uniform(0.7, 1.3, size=3)
    k = wavenumber(4000.0)
    g = smoothed_gaussian_field(v.shape[0], t, m, seed=2)
    pts = sphere_points(256, 0.5, seed=0)
    return dict(vertices=v, triangles=t, k=k, neumann=g, points=pts)


def differentiation():
    """Icosphere s4, r 0.1 m, k at 2 kHz, one smoothed field, 128 listeners at r 0.5 m."""
    v, t = icosphere(4, 0.1)
    k = wavenumber(2000.0)
    g = smoothed_gaussian_field(v.shape[0], t, 1, seed=3)[:, 0]
    pts = sphere_points(128, 0.5, seed=4)
    return dict(vertices=v, triangles=t, k=k, neumann=g, points=pts)


def batching(n_meshes: int = 64, n_k: int = 16, n_rhs: int = 16, seed: int = 5, max_subdiv: int = 5):
    """64 icospheres of subdivision U{2..5}, scaled U[0.6,1.4]^3 and rotated,
    16 log-uniform frequencies in [100, 10000] Hz, 16 smoothed RHS, 512 listeners at r 1 m."""
    rng = np.random.default_rng(seed)
    cache = {}
    problems = []
    for p in range(n_meshes):
        s = int(rng.integers(2, max_subdiv + 1))
        if s not in cache:
            cache[s] = icosphere(s, 0.1)
        v, t = cache[s]
        v = (v * rng.uniform(0.6, 1.4, size=3)) @ random_rotation(rng).T
        freqs = np.exp(rng.uniform(math.log(100.0), math.log(10000.0), size=n_k))
        g = smoothed_gaussian_field(v.shape[0], t, n_rhs, seed=int(rng.integers(1 << 30)))
        problems.append(dict(vertices=v, triangles=t, ks=[wavenumber(f) for f in freqs], neumann=g))
    pts = sphere_points(512, 1.0, seed=seed + 1)
    return problems, pts


def large_multi_rhs(m: int = 64):
    """Icosphere s6 with 5% radial noise (seed 6), r 0.2 m, k at 8 kHz, m RHS, 4096 listeners at r 1 m."""
    v, t = icosphere(6, 0.2)
    rng = np.random.default_rng(6)
    v = v * (1.0 + 0.05 * rng.uniform(-1.0, 1.0, size=(v.shape[0], 1)))
    k = wavenumber(8000.0)
    g = smoothed_gaussian_field(v.shape[0], t, m, seed=7)
    pts = sphere_points(4096, 1.0, seed=8)
    return dict(vertices=v, triangles=t, k=k, neumann=g, points=pts)
