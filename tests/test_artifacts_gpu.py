"""GPU artifact removal (sdfgpu_remove_artifacts, sdfgpu_sdf_components) against the CPU
restatement of src/SignedDistances/SdfArtifactRemoval.jl in oracle/artifacts.py.  Labels, counts
and the flipped field are integer/sign work, so every comparison is exact."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import artifacts

pytestmark = pytest.mark.gpu


def _field(N, density, seed):
    rng = np.random.default_rng(seed)
    n = np.asarray(N) + 1
    sdf = rng.normal(size=int(np.prod(n)))
    # smooth-ish structure: a few large blobs plus speckle
    sdf += (rng.random(sdf.size) < density) * 2.0
    return sdf


@pytest.mark.parametrize("N,density,ratio,thr", [
    ([31, 27, 23], 0.05, 0.01, 0.0),
    ([40, 40, 40], 0.20, 0.05, 0.5),
    ([63, 1, 50], 0.30, 0.5, -0.2),
    ([0, 0, 0], 0.0, 0.01, 0.0),
    ([127, 0, 0], 0.4, 0.3, 0.1),
])
def test_remove_artifacts_matches_oracle(gpu_ctx, N, density, ratio, thr):
    sdf = _field(N, density, seed=sum(N))
    ref, flipped_ref, comps_ref, largest_ref = artifacts.remove_sdf_artifacts(sdf, N, thr, ratio)
    out = sdf.copy()
    flipped, comps, largest = gpu_ctx.remove_artifacts(N, out, thr, ratio)
    assert (flipped, comps, largest) == (flipped_ref, comps_ref, largest_ref)
    assert np.array_equal(out, ref)


def test_components_labels_match_oracle(gpu_ctx):
    N = [45, 38, 29]
    sdf = _field(N, 0.1, seed=11)
    roots, comps, largest = gpu_ctx.components(N, sdf, 0.0)
    ref = artifacts.labels(sdf >= 0.0, np.asarray(N) + 1)
    assert np.array_equal(roots.astype(np.int64), ref)
    assert comps == np.unique(ref[ref >= 0]).size


def test_nan_and_empty(gpu_ctx):
    N = [9, 9, 9]
    sdf = -np.ones(1000)
    assert gpu_ctx.remove_artifacts(N, sdf.copy(), 0.0, 0.01) == (0, 0, 0)
    sdf[::7] = np.nan
    sdf[3] = 1.0
    out = sdf.copy()
    ref, f, c, l = artifacts.remove_sdf_artifacts(sdf, N, 0.0, 0.01)
    assert gpu_ctx.remove_artifacts(N, out, 0.0, 0.01) == (f, c, l)
    assert np.array_equal(out, ref, equal_nan=True)


def test_stl_to_sdf_pipeline_with_artifacts(gpu_ctx, tmp_path):
    """The reference test's configuration (runtests.jl:39-49 without smoothing): artifacts.stl at
    cell size 0.5 with artifact removal, against the oracle's sdf passed through the oracle's
    artifact removal."""
    import os

    import oracle
    import stl2sdf
    from conftest import GOLDEN

    sdf, grid, path = stl2sdf.stl_to_sdf(os.path.join(GOLDEN, "artifacts.stl"),
                                         stl2sdf.Options(cell_size=0.5, remove_artifacts=True), out_dir=str(tmp_path))
    assert os.path.exists(path)
    X, IEN = stl2sdf.import_stl(os.path.join(GOLDEN, "artifacts.stl"))
    d, _, _ = oracle.distances(X, IEN, grid.AABB_min, grid.cell_size, grid.N, mode=0)
    s = oracle.signs(X, IEN, grid.AABB_min, grid.cell_size, grid.N)["sign"]
    ref, _, _, _ = artifacts.remove_sdf_artifacts(d * s, grid.N, 0.0, 0.01)
    assert np.array_equal(sdf, ref)
