"""RBF smoothing of the SDF, mirroring ``stl2sdf.SdfSmoothing`` (src/SdfSmoothing/RBFs4Smoothing.jl).

``RBFs_smoothing(dist, grid, is_interpolation, smooth, threshold=1e-3) -> (fine_sdf, fine_grid)``
(:275-320) runs in libsdfgpu.so (``sdfgpu_rbf_smoothing``): Gaussian RBFs of width
``grid.cell_size`` centred on the grid nodes, weights by conjugate gradients (interpolation) or the
values themselves (approximation), evaluated on the grid refined ``smooth`` times.  The fine values
are Float32, like the reference's; ``fine_grid`` is ``Grid(AABB_min, AABB_max, maximum(N) * smooth,
0)`` as in the reference (:315).
"""

from __future__ import annotations

import numpy as np

from . import _native
from .MeshGrid import Grid


def RBFs_smoothing(dist, my_grid: Grid, Is_interpolation: bool, smooth: int, threshold: float = 1e-3,
                   device: int = 0):
    name = "Interpolation" if Is_interpolation else "Approximation"
    dist = np.ascontiguousarray(dist, np.float64)
    N = np.asarray(my_grid.N, np.int64)
    print("Original grid size: ", N.tolist())
    print("Fine grid size: ", (N * int(smooth) + 1).tolist())
    ctx = _native.default_context(device)
    fine, _, iters, res = ctx.rbf_smoothing(my_grid.AABB_min, my_grid.AABB_max, N, my_grid.cell_size, dist,
                                            interpolation=Is_interpolation, smooth=int(smooth), threshold=threshold)
    if Is_interpolation:
        print(f"{name}: CG converged in {iters} iterations (|r| = {res:.3e})")
    new_grid = Grid(my_grid.AABB_min, my_grid.AABB_max, int(N.max()) * int(smooth), 0)
    return fine, new_grid
