"""z-slab calls (sdfgpu_sdf_slab): every value equals the same node of the full-grid call, so
slabs split as the multi-GPU path splits them concatenate into the full field."""

from __future__ import annotations

import numpy as np
import pytest

from conftest import grid_of

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("mesh", ["torus_mesh", "icosphere_mesh"])
def test_slabs_equal_full_grid(gpu_ctx, mesh, request):
    from stl2sdf import sharding

    X, IEN = request.getfixturevalue(mesh)
    g = grid_of(X, n_nodes_long_axis=72)
    gpu_ctx.set_mesh(X, IEN)
    full = gpu_ctx.sdf(g["origin"], g["h"], g["N"], want_parts=True)
    N = g["N"]
    layer = int((N[0] + 1) * (N[1] + 1))
    nz = int(N[2]) + 1
    cases = [(0, 0), (0, nz - 1), (5, 17), (nz - 1, nz - 1), (nz // 2, nz - 1)]
    for k0, k1 in cases:
        got = gpu_ctx.sdf_slab(g["origin"], g["h"], N, k0, k1, want_parts=True)
        for a, b in zip(got, full):
            assert np.array_equal(a, b[k0 * layer:(k1 + 1) * layer]), (k0, k1)
    for world in (2, 3, 8):
        parts = [gpu_ctx.sdf_slab(g["origin"], g["h"], N, *sharding.zslab_bounds(nz, world, r))
                 for r in range(world)]
        assert np.array_equal(np.concatenate(parts), full[0])


def test_slab_rejects_bad_layers(gpu_ctx, icosphere_mesh):
    from stl2sdf import _native

    X, IEN = icosphere_mesh
    g = grid_of(X, n_nodes_long_axis=24)
    gpu_ctx.set_mesh(X, IEN)
    N = g["N"]
    for k0, k1 in [(0, int(N[2]) + 1), (3, 2), (-1, 0)]:
        with pytest.raises(_native.SdfGpuError) as e:
            gpu_ctx.sdf_slab(g["origin"], g["h"], N, k0, k1)
        assert e.value.code == 1
