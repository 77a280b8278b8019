"""CPU restatement of remove_sdf_artifacts! / analyze_sdf_components -- TEST INFRASTRUCTURE ONLY.

Follows src/SignedDistances/SdfArtifactRemoval.jl:
  * interior mask sdf .>= threshold (:153);
  * 6-connected union-find over the grid, x fastest (:66-117, :163-182);
  * component sizes, the largest one (argmax over the sizes), min size
    max(1, round(Int, ratio * largest)) with Julia's ties-to-even rounding (:186-208);
  * nodes of the other components below the min size get -abs(sdf) (:211-236).

`union_find_labels` is a literal sequential union-find (for small grids, to pin the fast path);
`labels` uses scipy's 6-connected labelling, which yields the same components.  Component labels
are reported as the smallest linear node index of each component, a deterministic choice (the
reference's roots depend on its racy threaded union order).  Ties for the largest component go to
the smallest label.
"""

from __future__ import annotations

import numpy as np


def union_find_labels(mask: np.ndarray, n) -> np.ndarray:
    """Sequential union-find (SdfArtifactRemoval.jl:24-62, :163-182) on a flat mask of a grid with
    n = (nx, ny, nz) nodes; returns the smallest linear index of each node's component, -1 outside."""
    nx, ny, nz = (int(v) for v in n)
    parent = np.arange(mask.size)

    def find(x):
        while parent[x] != x:
            parent[x] = parent[parent[x]]
            x = parent[x]
        return x

    for idx in np.flatnonzero(mask):
        i, j, k = idx % nx, (idx // nx) % ny, idx // (nx * ny)
        for di, dj, dk in ((-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)):
            a, b, c = i + di, j + dj, k + dk
            if 0 <= a < nx and 0 <= b < ny and 0 <= c < nz:
                nb = a + nx * (b + ny * c)
                if mask[nb]:
                    ra, rb = find(idx), find(nb)
                    if ra != rb:
                        parent[max(ra, rb)] = min(ra, rb)
    out = np.full(mask.size, -1, np.int64)
    for idx in np.flatnonzero(mask):
        out[idx] = find(idx)
    return out


def labels(mask: np.ndarray, n) -> np.ndarray:
    """Same as union_find_labels, through scipy.ndimage.label (6-connectivity)."""
    from scipy import ndimage

    nx, ny, nz = (int(v) for v in n)
    lab, k = ndimage.label(mask.reshape(nz, ny, nx), structure=ndimage.generate_binary_structure(3, 1))
    lab = lab.reshape(-1)
    first = np.full(k + 1, -1, np.int64)
    idx = np.flatnonzero(lab)
    # smallest linear index per label: the first occurrence in index order
    uniq, pos = np.unique(lab[idx], return_index=True)
    first[uniq] = idx[pos]
    return first[lab]


def remove_sdf_artifacts(sdf: np.ndarray, N, threshold: float = 0.0, min_component_ratio: float = 0.01,
                         labeller=labels):
    """Returns (new sdf, flipped, components, largest); the input is not modified."""
    sdf = np.array(sdf, dtype=np.float64, copy=True)
    n = np.asarray(N, np.int64) + 1
    mask = sdf >= threshold
    if not mask.any():
        return sdf, 0, 0, 0
    lab = labeller(mask, n)
    roots, counts = np.unique(lab[mask], return_counts=True)
    order = np.lexsort((roots, -counts))  # largest size first, then smallest label
    keep, largest = int(roots[order[0]]), int(counts[order[0]])
    min_size = max(1, int(np.round(min_component_ratio * largest)))  # numpy rounds ties to even
    small = {int(r) for r, c in zip(roots, counts) if c < min_size and int(r) != keep}
    flip = mask & np.isin(lab, np.fromiter(small, np.int64, len(small)))
    sdf[flip] = -np.abs(sdf[flip])
    return sdf, int(flip.sum()), int(roots.size), largest
