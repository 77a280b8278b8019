"""RBF smoothing (RBFs_smoothing, src/SdfSmoothing/RBFs4Smoothing.jl:275-320).

CPU: the oracle restatement against analytic known answers.  GPU: sdfgpu_rbf_smoothing against
the oracle.  Tolerances: the approximation form is a fixed sum of Gaussian terms, so the two agree
to FP32 rounding (the GPU builds the 3-D Gaussian from per-axis factors and accumulates in FP64,
the reference takes exp of an FP32 distance and accumulates in FP32): 2e-6 of the largest |value|.
The interpolation form adds a CG solve stopped at |r| <= sqrt(eps(Float32)) |b| (3.45e-4
relative); two FP32 CG runs of the same recurrence stop within a couple of iterations of each
other and their solutions differ by up to the solver's own error, so the weights are checked
against the stopping rule itself and the fields to 2e-3 of the largest |value|.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import rbf

GAUSS_SUM = sum(c * np.exp(-r2) for r2, c in ((0, 1), (1, 6), (2, 12), (3, 8), (4, 6), (5, 24), (6, 24)))


def _grid(N=(12, 10, 8), h=0.1, o=(0.0, 0.0, 0.0)):
    N = np.asarray(N, np.int64)
    o = np.asarray(o, np.float64)
    return o, o + N * h, N, h


def test_oracle_approximation_of_ones_is_the_lattice_gaussian_sum():
    o, amax, N, h = _grid()
    fine, dims, _, _ = rbf.rbf_smoothing(np.ones(int(np.prod(N + 1))), o, amax, N, h, False, 2)
    vol = fine.reshape(dims[2], dims[1], dims[0])
    # fine node (2i, 2j, 2k) sits on coarse node (i, j, k); well inside, all 81 stencil terms count
    assert abs(float(vol[8, 10, 12]) - GAUSS_SUM) < 1e-5 * GAUSS_SUM


def test_oracle_interpolation_reproduces_nodes():
    o, amax, N, h = _grid()
    rng = np.random.default_rng(1)
    b = rng.normal(size=int(np.prod(N + 1)))
    fine, dims, w, its = rbf.rbf_smoothing(b, o, amax, N, h, True, 1)
    assert 5 < its < 500
    K = rbf.kernel_matrix(rbf.coarse_axes(o, amax, N), h, 1e-3)
    b32 = b.astype(np.float32)
    assert np.linalg.norm(K @ w - b32) <= 1.01 * np.sqrt(np.finfo(np.float32).eps) * np.linalg.norm(b32)
    assert np.max(np.abs(fine - b32)) < 0.05 * np.max(np.abs(b32))


def test_oracle_process_vector_replaces_placeholders():
    v = np.array([0.5, -1.0e10, 0.25, 1.0e10, -0.75])
    out = rbf.process_vector(v)
    assert out.dtype == np.float32 and out.tolist() == [0.5, -0.75, 0.25, 0.75, -0.75]


@pytest.mark.gpu
@pytest.mark.parametrize("N,smooth", [((12, 10, 8), 2), ((20, 7, 15), 1), ((9, 9, 9), 3)])
def test_gpu_approximation_matches_oracle(gpu_ctx, N, smooth):
    o, amax, N, h = _grid(N, 0.05, (-0.3, 0.2, 1.0))
    rng = np.random.default_rng(int(N.sum()))
    d = rng.normal(size=int(np.prod(N + 1))) * 0.05
    ref, dims, _, _ = rbf.rbf_smoothing(d, o, amax, N, h, False, smooth)
    got, _, its, _ = gpu_ctx.rbf_smoothing(o, amax, N, h, d, interpolation=False, smooth=smooth)
    assert its == 0 and got.dtype == np.float32 and got.shape == ref.shape
    assert np.max(np.abs(got - ref)) <= 2e-6 * np.max(np.abs(ref))


@pytest.mark.gpu
def test_gpu_interpolation_matches_oracle(gpu_ctx):
    o, amax, N, h = _grid((16, 12, 10), 0.1, (0.5, -1.0, 0.0))
    rng = np.random.default_rng(3)
    d = rng.normal(size=int(np.prod(N + 1))) * 0.1
    ref, dims, w_ref, its_ref = rbf.rbf_smoothing(d, o, amax, N, h, True, 2)
    got, w, its, res = gpu_ctx.rbf_smoothing(o, amax, N, h, d, interpolation=True, smooth=2, want_weights=True)
    K = rbf.kernel_matrix(rbf.coarse_axes(o, amax, N), h, 1e-3)
    b32 = rbf.process_vector(d)
    tol = np.sqrt(np.finfo(np.float32).eps) * np.linalg.norm(b32)
    assert np.linalg.norm(K @ w - b32) <= 1.05 * tol
    assert abs(its - its_ref) <= 3
    assert np.max(np.abs(got - ref)) <= 2e-3 * np.max(np.abs(ref))


@pytest.mark.gpu
@pytest.mark.parametrize("refinement", [1, 2])
def test_stl_to_sdf_with_smoothing_reference_test_config(tmp_path, refinement):
    """The reference's own test run (test/runtests.jl:39-49): artifacts.stl, cell size 0.5,
    :interpolation smoothing, grid_refinement 1, artifact removal (and the same with refinement 2);
    the fine field against the oracle's smoothing of the same coarse field, and the written files."""
    import os

    import stl2sdf
    from conftest import GOLDEN
    from stl2sdf import DataExport

    sdf, grid, path = stl2sdf.stl_to_sdf(os.path.join(GOLDEN, "artifacts.stl"),
                                         stl2sdf.Options(smoothing_method="interpolation", grid_refinement=refinement,
                                                         cell_size=0.5, remove_artifacts=True), out_dir=str(tmp_path))
    fine_path = os.path.join(str(tmp_path), "artifacts_fine_sdf.vti")
    vals, dims, origin, spacing, label = DataExport.read_vti(fine_path)
    assert vals.dtype == np.float32 and label == "distance"
    ref, rdims, _, _ = rbf.rbf_smoothing(sdf, grid.AABB_min, grid.AABB_max, grid.N, grid.cell_size, True, refinement)
    assert np.array_equal(dims, rdims)
    assert np.max(np.abs(vals - ref)) <= 2e-3 * np.max(np.abs(ref))
