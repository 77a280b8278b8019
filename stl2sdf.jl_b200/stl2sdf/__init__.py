"""stl2sdf (B200 build): the SignedDistances hot path of stl2sdf.jl on sm_100a.

Mirrors the reference module ``stl2sdf`` (src/stl2sdf.jl): ``stl_to_sdf(stl_filename;
options=Options(...))`` plus the submodules ``DataImport``, ``MeshGrid``, ``SignedDistances`` and
``DataExport``.  The distance and sign stages run in libsdfgpu.so (hand-written CUDA for
sm_100a); the Julia host code of the reference binds the same C ABI through ``ccall``.
"""

from __future__ import annotations

import os

import numpy as np

from . import DataExport, DataImport, MeshGrid, SdfSmoothing, SignedDistances
from .DataExport import exportSdfToVTI
from .DataImport import import_stl
from .MeshGrid import (Grid, TriangularMesh, generateGridPoints, getMesh_AABB, interactive_sdf_grid_setup,
                       noninteractive_sdf_grid_setup)
from .SdfArtifactRemoval import analyze_sdf_components, remove_sdf_artifacts
from .SdfSmoothing import RBFs_smoothing
from .SignedDistances import evalDistancesOnTriMesh, raycast_sign_detection, signed_distance_field
from ._native import SdfGpuError

__all__ = [
    "Options", "stl_to_sdf", "import_stl", "TriangularMesh", "Grid", "generateGridPoints", "getMesh_AABB",
    "noninteractive_sdf_grid_setup", "interactive_sdf_grid_setup", "evalDistancesOnTriMesh",
    "raycast_sign_detection", "signed_distance_field", "remove_sdf_artifacts", "analyze_sdf_components",
    "exportSdfToVTI", "RBFs_smoothing", "SdfGpuError",
]


class Options:
    """Options (src/stl_to_sdf.jl:21-43)."""

    def __init__(self, smoothing_method=None, grid_refinement: int = 1, cell_size=None, remove_artifacts: bool = False,
                 artifact_ratio: float = 0.01, distance_mode: str = "ref"):
        self.smoothing_method = smoothing_method
        self.grid_refinement = grid_refinement
        self.cell_size = cell_size
        self.remove_artifacts = remove_artifacts
        self.artifact_ratio = artifact_ratio
        self.distance_mode = distance_mode


def stl_to_sdf(stl_filename: str, options: Options = None, out_dir: str = ".", timings: dict = None):
    """stl_to_sdf (src/stl_to_sdf.jl:75-147): STL -> mesh -> grid -> distances x signs -> VTI.

    Writes ``<base>_sdf.vti`` (point field "distance") into out_dir, and with a smoothing method
    also ``<base>_fine_sdf.vti`` (the RBF-smoothed field on the refined grid, Float32).  Returns
    (sdf, grid, path).  timings: a dict to receive the host wall-clock seconds of each stage
    ("import", "grid", "sdf", "artifacts", "export", "smoothing"; the stages that ran).
    """
    import time

    clock = [time.perf_counter()]

    def lap(name):
        now = time.perf_counter()
        if timings is not None:
            timings[name] = now - clock[0]
        clock[0] = now

    options = options or Options()
    if options.smoothing_method is not None and options.smoothing_method not in ("interpolation", "approximation"):
        raise AssertionError("smoothing_method must be :interpolation, :approximation, or nothing")
    if options.grid_refinement not in (1, 2):
        raise AssertionError("grid_refinement must be 1 or 2")
    if not (0.0 < options.artifact_ratio < 1.0):
        raise AssertionError("artifact_ratio must be in range (0, 1)")
    base = os.path.splitext(os.path.basename(stl_filename))[0]
    X, IEN = import_stl(stl_filename)
    mesh = TriangularMesh(X, IEN)
    lap("import")
    if options.cell_size is None:
        grid = interactive_sdf_grid_setup(mesh)
    else:
        grid = noninteractive_sdf_grid_setup(mesh, float(options.cell_size))
    lap("grid")
    sdf, _, _, conf = signed_distance_field(mesh, grid, mode=options.distance_mode, parts=("conf",))
    lap("sdf")
    low = int(np.count_nonzero(conf < 0.6))
    if low:
        print(f"{low} points have low confidence (<0.6)")
    if options.remove_artifacts:
        flipped = remove_sdf_artifacts(sdf, grid, min_component_ratio=options.artifact_ratio)
        print(f"Artifact removal completed: {flipped} nodes modified")
        lap("artifacts")
    path = exportSdfToVTI(os.path.join(out_dir, f"{base}_sdf.vti"), grid, sdf, "distance")
    lap("export")
    if options.smoothing_method is not None:
        fine_sdf, fine_grid = RBFs_smoothing(sdf, grid, options.smoothing_method == "interpolation",
                                             options.grid_refinement)
        exportSdfToVTI(os.path.join(out_dir, f"{base}_fine_sdf.vti"), fine_grid, fine_sdf, "distance")
        lap("smoothing")
    return sdf, grid, path
