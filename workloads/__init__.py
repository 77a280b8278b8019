"""Benchmark and test workloads of the SignedDistances hot path -- not part of the product.

* :mod:`workloads.synthetic` generates the seeded closed meshes (icosphere, torus, Gaussian-blob and
  gyroid marching-cubes surfaces, the uneven batch); the marching cubes run in
  ``_build/libmeshgen.so`` (``meshgen.cpp``).
* :func:`ensure_stl` writes a named workload mesh once as a binary STL (float32 vertices, the
  format the reference imports) and returns its path.  The mesh is generated in a child process, so
  the process that reads the STL (for example the reference arm of ``bench.py``) loads neither
  ``libmeshgen.so`` nor the product library.
* :data:`WORKLOADS` holds each workload's grid rule; :func:`grid_args` turns it into the arguments
  of the reference's ``Grid`` constructor or ``noninteractive_sdf_grid_setup``.
* :func:`measure_fp32_peak` runs the FP32 FMA-chain probe (``_build/libfp32peak.so``), the
  denominator of the hot path's FP32 roofline.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)

# name -> (mesh recipe, grid rule, description).  Grid rule ("nmax", K) is Grid(Xmin, Xmax, K - 7, 3):
# K nodes on the longest axis before Grid.jl's ceil (the way test/runtests.jl:65-66 builds grids);
# ("cell", B) is noninteractive_sdf_grid_setup with cell size B (Grid_setup.jl:104-124).
WORKLOADS = {
    "icosphere": (("icosphere", 4, 0.01, 0), ("cell", 0.05),
                  "icosphere L4 (5120 tris) r=1 jitter N(0,0.01) seed 0, cell_size 0.05, pad 3"),
    "torus128": (("torus", 1.0, 0.3, 512, 128, 0.02, 1), ("nmax", 128),
                 "torus R=1 r=0.3 512x128 quads (131072 tris) noise U(-2%,2%) seed 1, 128 nodes on the long axis"),
    "blobs256": (("blobs", 64, 2, 512), ("nmax", 256),
                 "marching cubes (512^3) of the 0.5 level of 64 Gaussian blobs (centres U[-1,1]^3, sigma U[0.1,0.3], "
                 "seed 2), 256 nodes on the long axis"),
    "gyroid320": (("gyroid", 384, 0.04, 2.0), ("nmax", 320),
                  "marching cubes (384^3) of the gyroid sheet |g| <= 0.04 over [0,4pi]^3 with an outside border, "
                  "320 nodes on the long axis"),
}


def cache_dir() -> str:
    d = os.environ.get("STL2SDF_WORKLOAD_CACHE") or os.path.join(os.environ.get("TMPDIR", "/tmp"), "stl2sdf_workloads")
    os.makedirs(d, exist_ok=True)
    return d


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def mesh(name: str):
    """(V, F) of a named workload before the float32 STL round trip (in this process)."""
    from . import synthetic

    recipe = WORKLOADS[name][0]
    kind, args = recipe[0], recipe[1:]
    if kind == "icosphere":
        level, jitter, seed = args
        return synthetic.icosphere(level, jitter=jitter, seed=seed)
    if kind == "torus":
        R, r, nu, nv, noise, seed = args
        return synthetic.torus(R, r, nu, nv, noise, seed=seed)
    if kind == "blobs":
        nblobs, seed, cells = args
        return synthetic.blobs(nblobs, seed=seed, cells=cells)
    if kind == "gyroid":
        cells, thickness, periods = args
        return synthetic.gyroid(cells, thickness, periods)
    raise KeyError(name)


def write_stl(name: str, path: str) -> None:
    """Generate a workload mesh and write it as a binary STL (atomically: temp file + rename)."""
    sys.path.insert(0, os.path.join(ROOT, "stl2sdf.jl_b200"))
    from stl2sdf import DataImport

    V, F = mesh(name)
    X, IEN = DataImport.roundtrip_float32(V, F)  # checks that no vertices merge after the rounding
    tmp = path + f".tmp{os.getpid()}"
    DataImport.write_binary_stl(tmp, X, IEN)
    os.replace(tmp, path)


def ensure_stl(name: str) -> str:
    """Path of the workload's binary STL, written once by a child process when it is missing."""
    if name not in WORKLOADS:
        raise KeyError(f"unknown workload {name}")
    path = os.path.join(cache_dir(), f"{name}.stl")
    if not os.path.exists(path):
        subprocess.run([sys.executable, "-c", f"import sys; sys.path.insert(0, {ROOT!r}); import workloads; "
                        f"workloads.write_stl({name!r}, {path!r})"], check=True)
    return path


def grid_args(name: str):
    """('nmax', K - 7) or ('cell', B): the grid rule of a workload."""
    kind, v = WORKLOADS[name][1]
    return (kind, v - 7) if kind == "nmax" else (kind, v)


def description(name: str) -> str:
    return WORKLOADS[name][2]


_PEAK = None


def measure_fp32_peak(device: int = 0) -> float:
    """Measured FP32 CUDA-core throughput of `device` in TFLOP/s (best of five timed launches of
    independent FMA chains on every SM at full occupancy)."""
    global _PEAK
    if _PEAK is None:
        path = os.path.join(HERE, "_build", "libfp32peak.so")
        if not os.path.exists(path):
            build()
        _PEAK = ctypes.CDLL(path)
        _PEAK.fp32_peak_tflops.argtypes = [ctypes.c_int32, ctypes.POINTER(ctypes.c_double)]
        _PEAK.fp32_peak_tflops.restype = ctypes.c_int
    t = ctypes.c_double(0.0)
    rc = _PEAK.fp32_peak_tflops(int(device), ctypes.byref(t))
    if rc:
        raise RuntimeError(f"fp32_peak_tflops failed ({rc})")
    return t.value
