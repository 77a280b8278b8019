"""The SignedDistances hot path, mirroring ``stl2sdf.SignedDistances`` (src/SignedDistances/).

Both functions keep the reference signatures and run on the GPU through libsdfgpu.so:

* ``evalDistancesOnTriMesh(mesh, grid, points) -> (dist, xp)`` -- dfOnTriangularMesh.jl:19-209
* ``raycast_sign_detection(mesh, grid, points; min_rays=6, max_rays=30, confidence_threshold=0.6,
  use_winding_fallback=true) -> (signs, confidences)`` -- RaycastingSignDetection.jl:337-404

``points`` must be the node matrix of ``grid`` (what every caller of the reference passes,
stl_to_sdf.jl:101-109); the library regenerates node coordinates from the grid with the same
rounding, so the 3 x ngp matrix never crosses the boundary.  There is no CPU fallback: without the
CUDA library or an sm_100 device these functions raise ``SdfGpuError``.
"""

from __future__ import annotations

import numpy as np

from . import _native
from .MeshGrid import Grid, GridPoints, TriangularMesh, generateGridPoints

MODES = {"ref": _native.MODE_REF_RULE, "exact": _native.MODE_EXACT, "unbounded": _native.MODE_UNBOUNDED}


def _check_points(grid: Grid, points) -> None:
    if points is None:
        return
    if isinstance(points, GridPoints) and points.grid is not None and points.grid == grid:
        return
    P = np.asarray(points)
    if P.shape != (3, grid.ngp) or not np.array_equal(P, generateGridPoints(grid)):
        raise NotImplementedError("points must be generateGridPoints(grid); arbitrary point sets are not supported")


def _ctx(mesh: TriangularMesh, device: int = 0):
    ctx = _native.default_context(device)
    ctx.set_mesh(mesh.vertex_rows(), mesh.triangle_rows(), key=mesh._key)
    return ctx


def evalDistancesOnTriMesh(mesh: TriangularMesh, grid: Grid, points=None, mode: str = "ref", want_xp: bool = True,
                           device: int = 0):
    """Truncated unsigned distance of every grid node (clamped to grid.cell_size).

    mode: "ref" (the reference's candidate rule, default), "exact" (true minimum, clamped) or
    "unbounded" (true minimum, not clamped).  Returns (dist, xp) with xp 3 x ngp (None when
    want_xp is False).
    """
    _check_points(grid, points)
    ctx = _ctx(mesh, device)
    dist, xp = ctx.distances(grid.AABB_min, grid.cell_size, grid.N, MODES[mode], want_xp=want_xp)
    return dist, (xp.T if xp is not None else None)


def raycast_sign_detection(mesh: TriangularMesh, grid: Grid, points=None, min_rays: int = 6, max_rays: int = 30,
                           confidence_threshold: float = 0.6, use_winding_fallback: bool = True, device: int = 0,
                           verbose: bool = False):
    """Adaptive ray-cast sign (+1 inside, -1 outside) and confidence of every grid node."""
    _check_points(grid, points)
    ctx = _ctx(mesh, device)
    signs, conf = ctx.signs(grid.AABB_min, grid.cell_size, grid.N, min_rays, max_rays, confidence_threshold,
                            use_winding_fallback)
    if verbose:
        low = int(np.count_nonzero(conf < confidence_threshold))
        print(f"Mean confidence: {conf.mean():.3f}")
        print(f"Low confidence points: {low}/{grid.ngp} ({100.0 * low / grid.ngp:.1f}%)")
    return signs, conf


def signed_distance_field(mesh: TriangularMesh, grid: Grid, mode: str = "ref", min_rays: int = 6, max_rays: int = 30,
                          confidence_threshold: float = 0.6, use_winding_fallback: bool = True, device: int = 0,
                          parts=("dist", "sign", "conf")):
    """Fused ``dists .* signs`` (stl_to_sdf.jl:105-119) in one library call: (sdf, dist, sign, conf).
    Only the named parts are copied back to the host; the others are None."""
    ctx = _ctx(mesh, device)
    return ctx.sdf(grid.AABB_min, grid.cell_size, grid.N, MODES[mode], min_rays, max_rays, confidence_threshold,
                   use_winding_fallback, want_parts=tuple(parts))


def last_stats(device: int = 0) -> dict:
    return _native.default_context(device).stats()
