"""Small-component removal, mirroring src/SignedDistances/SdfArtifactRemoval.jl:134-318.

Interior nodes are ``sdf >= threshold``; 6-connected interior components smaller than
``max(1, round(ratio * largest))`` (other than the largest) are flipped to ``-|sdf|``.  The
reference labels components with a union-find inside ``@threads`` (racy, :164-182); component
membership does not depend on the union order, so a deterministic labelling gives the
reference's result.  Ties for the largest component do not matter: a tied component is at least
the minimum size and is kept either way.
"""

from __future__ import annotations

import numpy as np


def _labels(mask3d: np.ndarray):
    from scipy import ndimage

    structure = ndimage.generate_binary_structure(3, 1)  # 6-connectivity
    return ndimage.label(mask3d, structure=structure)


def analyze_sdf_components(sdf_values, grid, threshold: float = 0.0) -> dict:
    """Component label -> size of the interior components (SdfArtifactRemoval.jl:259-318)."""
    n = np.asarray(grid.N, dtype=np.int64) + 1
    mask = (np.asarray(sdf_values) >= threshold).reshape(n[2], n[1], n[0])
    lab, k = _labels(mask)
    sizes = np.bincount(lab.reshape(-1), minlength=k + 1)[1:]
    return {i + 1: int(s) for i, s in enumerate(sizes)}


def remove_sdf_artifacts(sdf_values: np.ndarray, grid, threshold: float = 0.0, min_component_ratio: float = 0.01) -> int:
    """In place: flip small interior components; returns the number of nodes flipped."""
    sdf = sdf_values
    if sdf.shape[0] != grid.ngp:
        raise ValueError(f"SDF values length ({sdf.shape[0]}) doesn't match grid points ({grid.ngp})")
    n = np.asarray(grid.N, dtype=np.int64) + 1
    mask = (sdf >= threshold).reshape(n[2], n[1], n[0])
    if not mask.any():
        return 0
    lab, k = _labels(mask)
    sizes = np.bincount(lab.reshape(-1), minlength=k + 1)
    sizes[0] = 0
    largest = int(np.argmax(sizes))
    min_size = max(1, int(round(min_component_ratio * sizes[largest])))
    small = sizes < min_size
    small[0] = False
    small[largest] = False
    flip = small[lab.reshape(-1)]
    sdf[flip] = -np.abs(sdf[flip])
    return int(np.count_nonzero(flip))


remove_sdf_artifacts_ = remove_sdf_artifacts
