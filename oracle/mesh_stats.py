"""CPU restatement of calculate_edge_distances + analyze_mesh -- TEST INFRASTRUCTURE ONLY.

Follows src/MeshGrid/Grid_setup.jl:
  * calculate_edge_distances (:28-57): a 3 x nel matrix, entry (i, e) the length of the edge from
    vertex i to vertex mod1(i + 1, 3) of triangle e, norm(end_point - start_point);
  * analyze_mesh (:64-102): minimum, maximum, mean and median of all entries; the columns with the
    smallest / largest sum (argmin / argmax: the first on ties) and the mean of those columns.

Julia's norm of a 3-vector without overflow risk is sqrt(x^2 + y^2 + z^2) summed left to right
(LinearAlgebra.generic_norm2), which numpy reproduces here with no fused multiply-add.  Statistics'
median of an even count is middle(a, b) = a/2 + b/2 of the two middle values.  Julia sums the mean
pairwise, so only the mean may differ from another summation order in its last bits.
"""

from __future__ import annotations

import numpy as np


def calculate_edge_distances(X: np.ndarray, IEN: np.ndarray) -> np.ndarray:
    """X: nnp x 3 vertex rows; IEN: nel x 3 triangle rows, 1-based.  Returns 3 x nel."""
    X = np.asarray(X, np.float64)
    T = np.asarray(IEN, np.int64) - 1
    out = np.empty((3, T.shape[0]), np.float64)
    for i in range(3):
        d = X[T[:, (i + 1) % 3]] - X[T[:, i]]
        out[i] = np.sqrt((d[:, 0] * d[:, 0] + d[:, 1] * d[:, 1]) + d[:, 2] * d[:, 2])
    return out


def analyze_mesh(distances: np.ndarray) -> dict:
    """The statistics analyze_mesh prints, as a dict (indices 0-based)."""
    flat = np.sort(distances.ravel(order="F"))
    n = flat.size
    median = flat[n // 2] if n % 2 else flat[n // 2 - 1] / 2 + flat[n // 2] / 2
    sums = (distances[0] + distances[1]) + distances[2]
    imin, imax = int(np.argmin(sums)), int(np.argmax(sums))
    return {"shortest": float(flat[0]), "longest": float(flat[-1]), "mean": float(distances.mean()),
            "median": float(median), "smallest_mean": float(sums[imin] / 3.0),
            "largest_mean": float(sums[imax] / 3.0), "smallest_index": imin, "largest_index": imax}
