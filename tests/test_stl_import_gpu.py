"""STL import on the GPU (sdfgpu_stl_dedupe, process_stl_mesh of ImportStlData.jl:198-309) against
the oracle's restatements."""

from __future__ import annotations

import os

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import stl_dedupe

pytestmark = pytest.mark.gpu


def _same(a, b):
    return np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


def test_reference_fixture(gpu_ctx):
    from stl2sdf import DataImport

    V, T = DataImport.read_binary_stl(os.path.join(GOLDEN, "artifacts.stl"))
    X, IEN, near = gpu_ctx.stl_dedupe(V[T.reshape(-1) - 1])
    assert near == 0
    assert _same((X, IEN), stl_dedupe.exact(V, T))
    assert _same((X, IEN), stl_dedupe.sequential(V, T))
    assert _same(DataImport.import_stl(os.path.join(GOLDEN, "artifacts.stl")), (X, IEN))


@pytest.mark.parametrize("which", ["icosphere", "torus"])
def test_binary_file_matches_oracle_and_roundtrip(tmp_path, which):
    from stl2sdf import DataImport
    from workloads import synthetic

    V, F = synthetic.icosphere(4, jitter=0.01, seed=0) if which == "icosphere" else \
        synthetic.torus(1.0, 0.3, 512, 128, 0.02, seed=1)
    path = str(tmp_path / "m.stl")
    DataImport.write_binary_stl(path, V, F)
    got = DataImport.import_stl(path)
    assert _same(got, stl_dedupe.exact(*DataImport.read_binary_stl(path)))
    assert _same(got, DataImport.roundtrip_float32(V, F))


def test_shuffled_soup_with_repeats(gpu_ctx):
    # many copies of few vertices in a random stream order; negative and zero coordinates
    rng = np.random.default_rng(11)
    P = rng.integers(-3, 4, size=(500, 3)).astype(np.float64) * 0.25
    V = P[rng.integers(0, P.shape[0], size=3 * 20_001)]
    T = np.arange(1, V.shape[0] + 1).reshape(-1, 3)
    X, IEN, near = gpu_ctx.stl_dedupe(V)
    assert near == 0
    assert _same((X, IEN), stl_dedupe.exact(V, T))


def test_signed_zero_merges_into_the_first_appearance(gpu_ctx):
    V = np.array([[-0.0, 1, 2], [3, 4, 5], [0.0, 1, 2], [3, 4, 5], [6, 7, 8], [0.0, 1, -0.0]], np.float64)
    T = np.arange(1, 7).reshape(2, 3)
    X, IEN, near = gpu_ctx.stl_dedupe(V)
    assert near == 0 and IEN.tolist() == [[1, 2, 1], [2, 3, 4]]
    assert np.signbit(X[0, 0])  # the first appearance's value is kept
    assert _same((X, IEN), stl_dedupe.sequential(V, T))


def test_distinct_vertices_within_the_tolerance_take_the_reference_walk(gpu_ctx):
    from stl2sdf import DataImport

    V = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1e-11, 0, 0], [1, 1, 0], [0, 1, 0]], np.float64)
    T = np.array([[1, 2, 3], [4, 5, 6]])
    X, IEN, near = gpu_ctx.stl_dedupe(V[T.reshape(-1) - 1])
    assert near == 2 and X.shape[0] == 5  # exact deduplication, flagged
    assert _same(DataImport.process_stl_mesh(V, T), stl_dedupe.sequential(V, T))
    # across a cell border: 0.99999999999e-10 and 1.00000000001e-10 sit in neighbouring cells
    V2 = np.array([[0.99999999999e-10, 5, 5], [1, 0, 0], [0, 1, 0], [1.00000000001e-10, 5, 5], [1, 1, 0], [0, 1, 0]])
    X2, IEN2, near2 = gpu_ctx.stl_dedupe(V2)
    assert near2 == 2 == stl_dedupe.near_pairs(X2)
    assert _same(DataImport.process_stl_mesh(V2, T), stl_dedupe.sequential(V2, T))


def test_errors(gpu_ctx):
    from stl2sdf import _native

    with pytest.raises(_native.SdfGpuError, match="finite"):
        gpu_ctx.stl_dedupe(np.array([[0, 0, np.nan], [1, 0, 0], [0, 1, 0]], np.float64))
    with pytest.raises(_native.SdfGpuError, match="Int64"):  # floor(Int, 1e9 * 1e10) throws in the reference
        gpu_ctx.stl_dedupe(np.array([[1e9, 0, 0], [1, 0, 0], [0, 1, 0]], np.float64))


def test_cli_reports_stage_timings(tmp_path, capsys):
    from stl2sdf.__main__ import main

    assert main([os.path.join(GOLDEN, "artifacts.stl"), "--cell-size", "0.5", "--timings",
                 "--out-dir", str(tmp_path)]) == 0
    out = capsys.readouterr().out
    line = [x for x in out.splitlines() if x.startswith("stage seconds: ")]
    assert line and all(k in line[0] for k in ("context", "import", "grid", "sdf", "export"))
    assert os.path.exists(tmp_path / "artifacts_sdf.vti")
