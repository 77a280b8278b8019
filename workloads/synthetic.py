"""Seeded synthetic meshes for the SignedDistances workloads.

The reference ships no benchmark meshes for its hot path; these generators produce the closed
meshes of the five workloads (icosphere, torus, Gaussian blobs, gyroid sheet, uneven batch) with
the shapes, sizes and noise distributions the workloads name.  Every generator returns
``(X, IEN)`` with ``X`` an ``(nnp, 3)`` float64 array and ``IEN`` an ``(nel, 3)`` int64 array of
1-based vertex indices, the layout ``TriangularMesh`` packs (src/MeshGrid/MeshInformations.jl:68-83).

Meshes are meant to be written as binary STL (float32) and read back with
:func:`stl2sdf.DataImport.import_stl`, so the GPU path and the oracle see exactly the
float32-rounded vertices the reference would read.
"""

from __future__ import annotations

import numpy as np


def _orient_outward(V: np.ndarray, F: np.ndarray, center=None) -> np.ndarray:
    c = V.mean(axis=0) if center is None else np.asarray(center, float)
    a, b, d = V[F[:, 0]], V[F[:, 1]], V[F[:, 2]]
    n = np.cross(b - a, d - a)
    flip = np.einsum("ij,ij->i", n, (a + b + d) / 3.0 - c) < 0
    F = F.copy()
    F[flip, 1], F[flip, 2] = F[flip, 2].copy(), F[flip, 1].copy()
    return F


def icosahedron():
    """The 12 vertices and 20 outward faces of the unit icosahedron."""
    p = (1.0 + 5.0 ** 0.5) / 2.0
    V = np.array(
        [[-1, p, 0], [1, p, 0], [-1, -p, 0], [1, -p, 0],
         [0, -1, p], [0, 1, p], [0, -1, -p], [0, 1, -p],
         [p, 0, -1], [p, 0, 1], [-p, 0, -1], [-p, 0, 1]], dtype=np.float64)
    V /= np.linalg.norm(V, axis=1, keepdims=True)
    # Faces = triples of mutually adjacent vertices (edge length is the minimum pair distance).
    D = np.linalg.norm(V[:, None, :] - V[None, :, :], axis=2)
    e = D[D > 1e-9].min()
    adj = np.abs(D - e) < 1e-6
    F = [(i, j, k) for i in range(12) for j in range(i + 1, 12) for k in range(j + 1, 12)
         if adj[i, j] and adj[j, k] and adj[i, k]]
    F = np.array(F, dtype=np.int64)
    return V, _orient_outward(V, F, center=(0, 0, 0))


def icosphere(level: int = 4, radius: float = 1.0, jitter: float = 0.01, seed: int = 0):
    """Subdivided icosahedron on a sphere; each vertex scaled radially by 1 + N(0, jitter).

    level 4 gives 5,120 triangles and 2,562 vertices.
    """
    V, F = icosahedron()
    verts = [tuple(v) for v in V]
    for _ in range(level):
        cache = {}
        newF = []

        def mid(a, b):
            key = (a, b) if a < b else (b, a)
            idx = cache.get(key)
            if idx is None:
                m = (np.asarray(verts[a]) + np.asarray(verts[b])) / 2.0
                m /= np.linalg.norm(m)
                verts.append(tuple(m))
                idx = len(verts) - 1
                cache[key] = idx
            return idx

        for a, b, c in F:
            ab, bc, ca = mid(a, b), mid(b, c), mid(c, a)
            newF += [(a, ab, ca), (b, bc, ab), (c, ca, bc), (ab, bc, ca)]
        F = np.array(newF, dtype=np.int64)
    V = np.array(verts, dtype=np.float64) * radius
    rng = np.random.default_rng(seed)
    if jitter:
        V = V * (1.0 + rng.normal(0.0, jitter, size=(V.shape[0], 1)))
    return V, F + 1


def torus(R: float = 1.0, r: float = 0.3, nu: int = 512, nv: int = 128, noise: float = 0.02, seed: int = 1):
    """Watertight torus: nu x nv parametric quads split into 2 triangles each.

    The tube offset of every vertex is scaled by 1 + U(-noise, +noise).  512 x 128 gives
    131,072 triangles and 65,536 vertices.
    """
    rng = np.random.default_rng(seed)
    i = np.arange(nu)
    j = np.arange(nv)
    u = 2.0 * np.pi * i / nu
    v = 2.0 * np.pi * j / nv
    uu, vv = np.meshgrid(u, v, indexing="ij")
    rr = r * (1.0 + rng.uniform(-noise, noise, size=uu.shape))
    X = np.stack([(R + rr * np.cos(vv)) * np.cos(uu), (R + rr * np.cos(vv)) * np.sin(uu), rr * np.sin(vv)], axis=-1)
    X = X.reshape(-1, 3)
    ii, jj = np.meshgrid(i, j, indexing="ij")
    a = ii * nv + jj
    b = ((ii + 1) % nu) * nv + jj
    c = ((ii + 1) % nu) * nv + (jj + 1) % nv
    d = ii * nv + (jj + 1) % nv
    F = np.concatenate([np.stack([a, b, c], -1).reshape(-1, 3), np.stack([a, c, d], -1).reshape(-1, 3)], axis=0)
    # interleave the two triangles of each quad so neighbouring triangles have neighbouring ids
    F = F.reshape(2, -1, 3).transpose(1, 0, 2).reshape(-1, 3)
    return X, F.astype(np.int64) + 1


def box(lo=(0.0, 0.0, 0.0), hi=(1.0, 1.0, 1.0)):
    """Axis-aligned box as 12 outward triangles."""
    lo = np.asarray(lo, float); hi = np.asarray(hi, float)
    V = np.array([[lo[0] if (k & 1) == 0 else hi[0], lo[1] if (k & 2) == 0 else hi[1],
                   lo[2] if (k & 4) == 0 else hi[2]] for k in range(8)])
    quads = [(0, 2, 3, 1), (4, 5, 7, 6), (0, 1, 5, 4), (2, 6, 7, 3), (0, 4, 6, 2), (1, 3, 7, 5)]
    F = []
    for a, b, c, d in quads:
        F += [(a, b, c), (a, c, d)]
    F = _orient_outward(V, np.array(F, dtype=np.int64))
    return V, F + 1


_MG = None


def _meshgen():
    global _MG
    if _MG is None:
        import ctypes
        import os

        path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_build", "libmeshgen.so")
        if not os.path.exists(path):
            import subprocess

            subprocess.run(["make", "-s", "-C", os.path.dirname(os.path.abspath(__file__))], check=True)
        L = ctypes.CDLL(os.path.abspath(path))
        dp, i64p = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_int64)
        L.mg_blobs.argtypes = [dp, dp, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_double, ctypes.c_double]
        L.mg_blobs.restype = ctypes.c_void_p
        L.mg_gyroid.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.mg_gyroid.restype = ctypes.c_void_p
        L.mg_sizes.argtypes = [ctypes.c_void_p, i64p, i64p]
        L.mg_copy.argtypes = [ctypes.c_void_p, dp, i64p]
        L.mg_free.argtypes = [ctypes.c_void_p]
        L.mg_table.argtypes = [ctypes.POINTER(ctypes.c_int8), ctypes.POINTER(ctypes.c_int32)]
        _MG = L
    return _MG


def _collect(h):
    import ctypes

    L = _meshgen()
    nv, nt = ctypes.c_int64(), ctypes.c_int64()
    L.mg_sizes(h, ctypes.byref(nv), ctypes.byref(nt))
    V = np.empty((nv.value, 3)); T = np.empty((nt.value, 3), dtype=np.int64)
    L.mg_copy(h, V.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), T.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)))
    L.mg_free(h)
    return V, T


def blob_params(nblobs: int = 64, seed: int = 2, lo_sigma: float = 0.1, hi_sigma: float = 0.3):
    """Centres U[-1,1]^3 and sigmas U[lo,hi] from numpy's default_rng(seed)."""
    rng = np.random.default_rng(seed)
    centers = rng.uniform(-1.0, 1.0, size=(nblobs, 3))
    sigmas = rng.uniform(lo_sigma, hi_sigma, size=nblobs)
    return centers, sigmas


def blobs(nblobs: int = 64, seed: int = 2, cells: int = 512, iso: float = 0.5, box: float = 2.0):
    """Marching-cubes surface of the iso level of a sum of unit-amplitude Gaussian blobs.

    The lattice spans [-box, box]^3 with `cells` cells per axis; at distance >= 1 from every
    centre each blob is below exp(-1/0.18) < 0.004, so the field stays below 0.5 on the border
    of the default box and the surface is closed.  64 blobs at 512^3 give about 1.5M triangles.
    """
    import ctypes

    c, s = blob_params(nblobs, seed)
    c = np.ascontiguousarray(c); s = np.ascontiguousarray(s)
    dp = ctypes.POINTER(ctypes.c_double)
    h = _meshgen().mg_blobs(c.ctypes.data_as(dp), s.ctypes.data_as(dp), nblobs, iso, cells + 1, -box, box)
    return _collect(h)


def gyroid(cells: int = 384, thickness: float = 0.04, periods: float = 2.0):
    """Thin gyroid sheet |sin x cos y + sin y cos z + sin z cos x| <= thickness over
    [0, 2*pi*periods]^3, capped by an outside lattice border (closed)."""
    h = _meshgen().mg_gyroid(cells + 1, 0.0, 2.0 * np.pi * periods, thickness)
    return _collect(h)


def uneven_batch(count: int = 256, seed: int = 3, k_lo: int = 32, k_hi: int = 160):
    """Recipes of an uneven batch of meshes from numpy's default_rng(seed): the even entries are
    icospheres of level 2..6 (320..81,920 triangles, radial jitter N(0, 0.01)), the odd entries
    marching-cubes meshes of 8..32 Gaussian blobs extracted at 32..320 cells per axis (log-uniform;
    about 1k..400k triangles).  Each gets its own grid with K nodes on the longest axis, K uniform
    in [k_lo, k_hi].  Returns a list of dicts (kind, level | nblobs/cells/seed, K); `batch_mesh`
    builds one."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        K = int(rng.integers(k_lo, k_hi + 1))
        if i % 2 == 0:
            out.append(dict(kind="icosphere", level=int(rng.integers(2, 7)), seed=int(rng.integers(1 << 30)), K=K))
        else:
            cells = int(round(32.0 * 10.0 ** rng.uniform(0.0, 1.0)))
            out.append(dict(kind="blobs", nblobs=int(rng.integers(8, 33)), cells=cells,
                            seed=int(rng.integers(1 << 30)), K=K))
    return out


def batch_mesh(recipe: dict):
    """(V, F) of one `uneven_batch` entry (before the float32 STL round trip)."""
    if recipe["kind"] == "icosphere":
        return icosphere(recipe["level"], jitter=0.01, seed=recipe["seed"])
    return blobs(recipe["nblobs"], seed=recipe["seed"], cells=recipe["cells"])


def mc_table():
    """The derived marching-cubes table: (256, 16, 3) edge ids (-1 padded), (12, 2) edge corners."""
    import ctypes

    tri = np.empty(256 * 48, dtype=np.int8); ec = np.empty(24, dtype=np.int32)
    _meshgen().mg_table(tri.ctypes.data_as(ctypes.POINTER(ctypes.c_int8)), ec.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    return tri.reshape(256, 16, 3), ec.reshape(12, 2)


def is_oriented(IEN: np.ndarray) -> bool:
    """Every directed edge appears once and its reverse once (consistently oriented, closed)."""
    F = np.asarray(IEN, dtype=np.int64)
    d = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]])
    key = d[:, 0] * (F.max() + 1) + d[:, 1]
    rkey = d[:, 1] * (F.max() + 1) + d[:, 0]
    u, cnt = np.unique(key, return_counts=True)
    return bool(np.all(cnt == 1) and np.array_equal(np.sort(key), np.sort(rkey)))


def signed_volume(X: np.ndarray, IEN: np.ndarray) -> float:
    F = np.asarray(IEN, dtype=np.int64) - 1
    a, b, c = X[F[:, 0]], X[F[:, 1]], X[F[:, 2]]
    return float(np.einsum("ij,ij->i", a, np.cross(b, c)).sum() / 6.0)


def is_closed(IEN: np.ndarray) -> bool:
    """Every undirected edge is used by exactly two triangles."""
    F = np.asarray(IEN, dtype=np.int64)
    e = np.concatenate([F[:, [0, 1]], F[:, [1, 2]], F[:, [2, 0]]])
    e.sort(axis=1)
    _, counts = np.unique(e, axis=0, return_counts=True)
    return bool(np.all(counts == 2))
