"""Shared test setup: import paths, the ``gpu`` marker, and seeded workload fixtures.

``-m "not gpu"`` tests run on any machine (oracle vs known answers, host logic, C-ABI symbol
exports); ``-m gpu`` tests call the CUDA path through the C ABI and compare with the oracle.
"""

from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "stl2sdf.jl_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA sm_100 device and libsdfgpu.so")


@pytest.fixture(scope="session")
def icosphere_mesh():
    """Workload 1: icosphere L4 (5,120 triangles), radial jitter N(0, 0.01), seed 0, float32 STL."""
    from stl2sdf import DataImport
    from workloads import synthetic

    V, F = synthetic.icosphere(4, jitter=0.01, seed=0)
    return DataImport.roundtrip_float32(V, F)


@pytest.fixture(scope="session")
def torus_mesh():
    """Workload 2: torus R=1, r=0.3, 512 x 128 quads (131,072 triangles), tube noise U(-2%,2%), seed 1."""
    from stl2sdf import DataImport
    from workloads import synthetic

    V, F = synthetic.torus(1.0, 0.3, 512, 128, 0.02, seed=1)
    return DataImport.roundtrip_float32(V, F)


@pytest.fixture(scope="session")
def gpu_ctx():
    from stl2sdf import _native

    ctx = _native.Context(0)
    yield ctx
    ctx.close()


def grid_of(X, n_nodes_long_axis=None, cell=None):
    """Grid over the mesh box: either K nodes on the longest axis (Grid(Xmin, Xmax, K-7, 3)) or a
    cell size through noninteractive_sdf_grid_setup."""
    import oracle

    if cell is not None:
        return oracle.grid_from_cell_size(X, cell)
    return oracle.grid(X.min(axis=0), X.max(axis=0), n_nodes_long_axis - 7, 3)


def sample_nodes(ngp: int, k: int, seed: int = 42) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(ngp, size=min(k, ngp), replace=False)).astype(np.int64)
