"""Command line for stl_to_sdf (src/stl_to_sdf.jl:75-147):

    PYTHONPATH=stl2sdf.jl_b200 python -m stl2sdf part.stl --cell-size 0.5 [--remove-artifacts]
        [--artifact-ratio 0.01] [--smoothing interpolation|approximation] [--grid-refinement 1|2]
        [--out-dir DIR] [--timings]

Writes <base>_sdf.vti (and <base>_fine_sdf.vti with smoothing) like the reference.
"""

from __future__ import annotations

import argparse
import sys

from . import Options, stl_to_sdf


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(prog="python -m stl2sdf", description="Signed distance field of an STL mesh (VTI)")
    ap.add_argument("stl")
    ap.add_argument("--cell-size", type=float, required=True)
    ap.add_argument("--remove-artifacts", action="store_true")
    ap.add_argument("--artifact-ratio", type=float, default=0.01)
    ap.add_argument("--smoothing", choices=["interpolation", "approximation"], default=None)
    ap.add_argument("--grid-refinement", type=int, default=1)
    ap.add_argument("--out-dir", default=".")
    ap.add_argument("--timings", action="store_true", help="print the wall-clock seconds of each stage")
    a = ap.parse_args(argv)
    opts = Options(smoothing_method=a.smoothing, grid_refinement=a.grid_refinement, cell_size=a.cell_size,
                   remove_artifacts=a.remove_artifacts, artifact_ratio=a.artifact_ratio)
    t = {}
    if a.timings:  # the CUDA context first, so that its creation is not counted in the first stage
        import time

        from . import _native

        t0 = time.perf_counter()
        _native.default_context(0)
        t["context"] = time.perf_counter() - t0
    sdf, grid, path = stl_to_sdf(a.stl, opts, out_dir=a.out_dir, timings=t)
    print(f"{path}: {grid.ngp} nodes, sdf in [{sdf.min():.6g}, {sdf.max():.6g}]")
    if a.timings:
        print("stage seconds: " + ", ".join(f"{k} {v:.3f}" for k, v in t.items()))
    return 0


if __name__ == "__main__":
    sys.exit(main())
