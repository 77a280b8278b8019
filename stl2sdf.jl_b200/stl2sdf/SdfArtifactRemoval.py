"""Small-component removal, mirroring src/SignedDistances/SdfArtifactRemoval.jl:134-318, on the GPU.

Interior nodes are ``sdf >= threshold``; 6-connected interior components smaller than
``max(1, round(ratio * largest))`` (other than the largest) are flipped to ``-|sdf|``.  The
labelling runs in libsdfgpu.so (``sdfgpu_remove_artifacts``, a lock-free union-find); the
reference's threaded union-find (:164-182) is racy in its roots but not in its components, and
the components are all the result depends on.  Component labels here are the smallest linear node
index of each component (1-based in the returned dict, like the reference's linear indices).
"""

from __future__ import annotations

import numpy as np

from . import _native


def analyze_sdf_components(sdf_values, grid, threshold: float = 0.0, device: int = 0) -> dict:
    """Component label -> size of the interior components (SdfArtifactRemoval.jl:259-318)."""
    ctx = _native.default_context(device)
    roots, count, largest = ctx.components(np.asarray(grid.N, np.int64), np.asarray(sdf_values, np.float64),
                                           threshold)
    r = roots[roots >= 0]
    labels, sizes = np.unique(r, return_counts=True)
    return {int(a) + 1: int(b) for a, b in zip(labels, sizes)}


def remove_sdf_artifacts(sdf_values: np.ndarray, grid, threshold: float = 0.0, min_component_ratio: float = 0.01,
                         device: int = 0) -> int:
    """In place: flip small interior components; returns the number of nodes flipped."""
    sdf = sdf_values
    if sdf.shape[0] != grid.ngp:
        raise ValueError(f"SDF values length ({sdf.shape[0]}) doesn't match grid points ({grid.ngp})")
    if sdf.dtype != np.float64 or not sdf.flags.c_contiguous:
        raise TypeError("sdf_values must be a contiguous float64 vector")
    ctx = _native.default_context(device)
    flipped, _, _ = ctx.remove_artifacts(np.asarray(grid.N, np.int64), sdf, threshold, min_component_ratio)
    return flipped


remove_sdf_artifacts_ = remove_sdf_artifacts
