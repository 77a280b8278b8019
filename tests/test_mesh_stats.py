"""Mesh analysis printed by the grid setup (calculate_edge_distances + analyze_mesh,
src/MeshGrid/Grid_setup.jl:28-102): the oracle against a known answer on the CPU, and
sdfgpu_mesh_edge_stats against the oracle on the GPU."""

from __future__ import annotations

import math

import numpy as np
import pytest

from oracle import mesh_stats


def _two_triangles():
    X = np.array([[0, 0, 0], [3, 0, 0], [3, 4, 0],
                  [0, 0, 1], [1, 0, 1], [0.5, math.sqrt(3) / 2, 1]], np.float64)
    IEN = np.array([[1, 2, 3], [4, 5, 6]], np.int64)
    return X, IEN


def test_oracle_known_answer():
    X, IEN = _two_triangles()
    D = mesh_stats.calculate_edge_distances(X, IEN)
    assert D.shape == (3, 2)
    assert D[:, 0].tolist() == [3.0, 4.0, 5.0]  # v1->v2, v2->v3, v3->v1
    st = mesh_stats.analyze_mesh(D)
    assert st["longest"] == 5.0
    assert st["shortest"] == pytest.approx(1.0, abs=1e-15)
    assert st["mean"] == pytest.approx(2.5, abs=1e-15)
    assert st["median"] == pytest.approx(2.0, abs=1e-15)  # (1 + 3) / 2 of six values
    assert (st["smallest_index"], st["largest_index"]) == (1, 0)
    assert st["largest_mean"] == 4.0
    assert st["smallest_mean"] == pytest.approx(1.0, abs=1e-15)


def _check(ctx, X, IEN):
    ctx.set_mesh(X, IEN)
    got = ctx.mesh_edge_stats()
    want = mesh_stats.analyze_mesh(mesh_stats.calculate_edge_distances(X, IEN))
    for k in ("shortest", "longest", "median", "smallest_mean", "largest_mean", "smallest_index", "largest_index"):
        assert got[k] == want[k], k
    assert got["mean"] == pytest.approx(want["mean"], rel=1e-13)  # summation order differs


@pytest.mark.gpu
def test_edge_stats_icosphere(gpu_ctx, icosphere_mesh):
    X, IEN = icosphere_mesh
    _check(gpu_ctx, X, IEN)  # 15,360 edges: the median is the middle of two


@pytest.mark.gpu
def test_edge_stats_odd_count_and_soup(gpu_ctx):
    rng = np.random.default_rng(5)
    X = rng.normal(size=(1500, 3)) * rng.uniform(0.01, 10.0, size=(1500, 1))
    IEN = rng.integers(1, 1501, size=(100_001, 3))  # 300,003 edges over many blocks: one middle
    _check(gpu_ctx, X, IEN)


@pytest.mark.gpu
def test_edge_stats_ties_take_the_first_triangle(gpu_ctx):
    # unit squares split into two congruent right triangles: every edge sum ties
    n = 40
    xs, ys = np.meshgrid(np.arange(n + 1, dtype=np.float64), np.arange(n + 1, dtype=np.float64), indexing="ij")
    X = np.stack([xs.ravel(), ys.ravel(), np.zeros(xs.size)], axis=1)
    vid = lambda i, j: i * (n + 1) + j + 1
    tris = []
    for i in range(n):
        for j in range(n):
            tris.append([vid(i, j), vid(i + 1, j), vid(i + 1, j + 1)])
            tris.append([vid(i, j), vid(i + 1, j + 1), vid(i, j + 1)])
    IEN = np.array(tris, np.int64)
    _check(gpu_ctx, X, IEN)


@pytest.mark.gpu
def test_edge_stats_needs_a_mesh():
    from stl2sdf import _native

    ctx = _native.Context(0)
    try:
        with pytest.raises(_native.SdfGpuError):
            ctx.mesh_edge_stats()
    finally:
        ctx.close()


@pytest.mark.gpu
def test_grid_setup_prints_the_analysis(icosphere_mesh, capsys):
    from stl2sdf import MeshGrid

    X, IEN = icosphere_mesh
    mesh = MeshGrid.TriangularMesh(X, IEN)
    g = MeshGrid.noninteractive_sdf_grid_setup(mesh, 0.05)
    out = capsys.readouterr().out
    assert "Mesh Statistics:" in out and f"Number of elements: {mesh.nel}" in out
    assert f"Number of all grid points: {g.ngp}" in out
