"""CPU restatement of process_stl_mesh (src/DataImport/ImportStlData.jl:198-309) -- TEST
INFRASTRUCTURE ONLY.

`sequential` follows the reference line by line: the triangle stream is walked vertex by vertex;
a vertex merges into the first unique vertex, in creation order, with norm < 1e-10 in its hash
cell floor(v * 1e10) (:226-235) or, when it has none, in the first neighbour cell (dx, then dy,
then dz from -1 to 1, only cells the vertex is within 1e-10 of its border for, :238-278);
otherwise it becomes a new unique vertex (:281-291).

`exact` is the vectorised form for meshes without two distinct vertices closer than 1e-10, where
the walk above merges exactly the equal vertices (-0.0 equals +0.0) and numbers them in order of
first appearance: a stable lexicographic sort, group heads, first appearances.  `near_pairs`
tells whether a mesh is of that kind.
"""

from __future__ import annotations

import math

import numpy as np

TOL = 1e-10
SCALE = 10000000000  # floor(Int, 1 / tol)


def _norm(a, b) -> float:
    dx, dy, dz = a[0] - b[0], a[1] - b[1], a[2] - b[2]
    return math.sqrt((dx * dx + dy * dy) + dz * dz)


def sequential(V: np.ndarray, T: np.ndarray):
    """V: (n, 3) vertices; T: (nel, 3) 1-based indices into V.  Returns (X (nnp, 3), IEN (nel, 3))."""
    V = np.asarray(V, np.float64)
    T = np.asarray(T, np.int64)
    cells: dict = {}
    uniq: list = []
    out = np.empty(T.shape, np.int64)
    lim = TOL * SCALE
    for e in range(T.shape[0]):
        for c in range(3):
            v = tuple(float(x) for x in V[T[e, c] - 1])
            key = tuple(math.floor(x * SCALE) for x in v)
            found = 0
            for idx in cells.get(key, ()):
                if _norm(v, uniq[idx - 1]) < TOL:
                    found = idx
                    break
            if not found:
                pos = [x * SCALE - math.floor(x * SCALE) for x in v]
                for dx in (-1, 0, 1):
                    for dy in (-1, 0, 1):
                        for dz in (-1, 0, 1):
                            if found:
                                break
                            if dx == 0 and dy == 0 and dz == 0:
                                continue
                            near_border = ((dx == -1 and pos[0] < lim) or (dx == 1 and pos[0] > 1 - lim) or
                                           (dy == -1 and pos[1] < lim) or (dy == 1 and pos[1] > 1 - lim) or
                                           (dz == -1 and pos[2] < lim) or (dz == 1 and pos[2] > 1 - lim))
                            if not near_border:
                                continue
                            for idx in cells.get((key[0] + dx, key[1] + dy, key[2] + dz), ()):
                                if _norm(v, uniq[idx - 1]) < TOL:
                                    found = idx
                                    break
            if not found:
                uniq.append(v)
                found = len(uniq)
                cells.setdefault(key, []).append(found)
            out[e, c] = found
    return np.asarray(uniq, np.float64).reshape(-1, 3), out


def exact(V: np.ndarray, T: np.ndarray):
    """Exact deduplication in first-appearance order (equal to `sequential` when near_pairs is 0)."""
    V = np.asarray(V, np.float64)
    S = V[np.asarray(T, np.int64).reshape(-1) - 1]
    o = np.lexsort((S[:, 2], S[:, 1], S[:, 0]))  # stable, x primary
    Ss = S[o]
    head = np.ones(o.shape[0], bool)
    head[1:] = np.any(Ss[1:] != Ss[:-1], axis=1)
    gid = np.cumsum(head) - 1
    first = o[head]
    by_first = np.argsort(first, kind="stable")
    rank = np.empty_like(by_first)
    rank[by_first] = np.arange(by_first.shape[0])
    IEN = np.empty(o.shape[0], np.int64)
    IEN[o] = rank[gid] + 1
    return S[first[by_first]], IEN.reshape(-1, 3)


def near_pairs(X: np.ndarray) -> int:
    """Ordered pairs of distinct rows of X closer than 1e-10."""
    from scipy.spatial import cKDTree

    if X.shape[0] < 2:
        return 0
    P = cKDTree(X).query_pairs(r=TOL, output_type="ndarray")
    n = sum(1 for a, b in P if _norm(X[a], X[b]) < TOL)
    return 2 * n
