"""Seeded synthetic meshes in the layout manapy's mesh reader hands to ``Domain``.

manapy reads a gmsh file, tags boundary vertices and writes per-rank HDF5
(``manapy/partitions/meshpartitioning.py:160-275``); ``Domain`` then reads back
``elements`` (int32 ``[Nc, k+1]``, last column = k) and ``nodes`` (float64
``[Nn, 4]`` = ``[x, y, z, tag]``) (``manapy/ddm/pure_ddm.py:13-33``).  The
generators below produce exactly those two arrays from a seed, so both the
reference and this package can be driven with identical inputs.

Vertex tags follow the reference's precedence rule
(``manapy/partitions/partitions_utils.py:44-60``): tags 1/2 (x = 0 / x = 1) win,
then 3/4 (y = 1 / y = 0), then 5/6 (z = 0 / z = 1); interior vertices are 0.

Random draws use ``numpy.random.default_rng(seed)`` in this fixed order:
vertex jitter (for every vertex, applied to interior ones only), then the
per-square diagonal coin (2D only), then the cell permutation.
"""
from __future__ import annotations

import numpy as np

__all__ = ["square_triangles", "cube_tetrahedra", "mesh_sizes_2d", "mesh_sizes_3d"]

# Hex-to-tet split of manapy (manapy/ddm/ddm_utils3d.py:730-734) with the hex
# corner order (0,0,0),(1,0,0),(1,1,0),(0,1,0),(0,0,1),(1,0,1),(1,1,1),(0,1,1).
HEX_TO_TETS = np.array([[0, 1, 3, 4], [1, 3, 4, 5], [4, 5, 3, 7],
                        [1, 3, 5, 2], [3, 7, 5, 2], [5, 7, 6, 2]], dtype=np.int64)


def mesh_sizes_2d(n: int) -> dict:
    """Cell/face/node counts of ``square_triangles(n)``."""
    return {"cells": 2 * n * n, "faces": 3 * n * n + 2 * n, "nodes": (n + 1) ** 2}


def mesh_sizes_3d(n: int) -> dict:
    """Cell/node counts of ``cube_tetrahedra(n)``."""
    return {"cells": 6 * n ** 3, "nodes": (n + 1) ** 3}


def square_triangles(n: int, seed: int = 0, jitter: float = 0.2, permute: bool = True):
    """Unit square, ``n x n`` squares each split along a random diagonal.

    Returns ``(elements, vertex)``: int32 ``[2n^2, 4]`` rows ``[a, b, c, 3]``
    (counter-clockwise) and float64 ``[(n+1)^2, 4]`` rows ``[x, y, 0, tag]``.
    Vertex ``(i, j)`` (x = i h, y = j h) has index ``j (n+1) + i``.
    """
    if n < 1:
        raise ValueError("n must be >= 1")
    rng = np.random.default_rng(seed)
    h = 1.0 / n
    nv = n + 1
    j, i = np.meshgrid(np.arange(nv), np.arange(nv), indexing="ij")
    i = i.ravel()
    j = j.ravel()
    x = i * h
    y = j * h
    jit = rng.uniform(-jitter * h, jitter * h, size=(nv * nv, 2))
    interior = (i > 0) & (i < n) & (j > 0) & (j < n)
    x = np.where(interior, x + jit[:, 0], x)
    y = np.where(interior, y + jit[:, 1], y)
    tag = np.zeros(nv * nv, dtype=np.float64)
    tag[j == 0] = 4
    tag[j == n] = 3
    tag[i == n] = 2
    tag[i == 0] = 1
    vertex = np.stack([x, y, np.zeros_like(x), tag], axis=1).astype(np.float64)

    sj, si = np.meshgrid(np.arange(n), np.arange(n), indexing="ij")
    si = si.ravel()
    sj = sj.ravel()
    a = sj * nv + si
    b = a + 1
    c = a + nv + 1
    d = a + nv
    diag = rng.integers(0, 2, size=n * n)
    t1 = np.where(diag[:, None] == 0, np.stack([a, b, c], 1), np.stack([a, b, d], 1))
    t2 = np.where(diag[:, None] == 0, np.stack([a, c, d], 1), np.stack([b, c, d], 1))
    tri = np.empty((2 * n * n, 3), dtype=np.int64)
    tri[0::2] = t1
    tri[1::2] = t2
    if permute:
        tri = tri[rng.permutation(len(tri))]
    elements = np.empty((len(tri), 4), dtype=np.int32)
    elements[:, :3] = tri
    elements[:, 3] = 3
    return elements, vertex


def cube_tetrahedra(n: int, seed: int = 0, jitter: float = 0.15, permute: bool = True):
    """Unit cube, ``n^3`` hexes each split into 6 tetrahedra by manapy's rule.

    Returns ``(elements, vertex)``: int32 ``[6n^3, 5]`` rows ``[a, b, c, d, 4]``
    and float64 ``[(n+1)^3, 4]`` rows ``[x, y, z, tag]``.  Vertex
    ``(i, j, k)`` has index ``(k (n+1) + j) (n+1) + i``.
    """
    if n < 1:
        raise ValueError("n must be >= 1")
    rng = np.random.default_rng(seed)
    h = 1.0 / n
    nv = n + 1
    k, j, i = np.meshgrid(np.arange(nv), np.arange(nv), np.arange(nv), indexing="ij")
    i = i.ravel()
    j = j.ravel()
    k = k.ravel()
    pos = np.stack([i * h, j * h, k * h], axis=1)
    jit = rng.uniform(-jitter * h, jitter * h, size=(nv ** 3, 3))
    interior = (i > 0) & (i < n) & (j > 0) & (j < n) & (k > 0) & (k < n)
    pos = np.where(interior[:, None], pos + jit, pos)
    tag = np.zeros(nv ** 3, dtype=np.float64)
    tag[k == n] = 6
    tag[k == 0] = 5
    tag[j == 0] = 4
    tag[j == n] = 3
    tag[i == n] = 2
    tag[i == 0] = 1
    vertex = np.concatenate([pos, tag[:, None]], axis=1).astype(np.float64)

    hk, hj, hi = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    base = ((hk * nv + hj) * nv + hi).ravel()
    dx, dy, dz = 1, nv, nv * nv
    corners = np.stack([base, base + dx, base + dx + dy, base + dy,
                        base + dz, base + dx + dz, base + dx + dy + dz, base + dy + dz], axis=1)
    tets = corners[:, HEX_TO_TETS].reshape(-1, 4)
    if permute:
        tets = tets[rng.permutation(len(tets))]
    elements = np.empty((len(tets), 5), dtype=np.int32)
    elements[:, :4] = tets
    elements[:, 4] = 4
    return elements, vertex
