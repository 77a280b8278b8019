"""sdfgpu_distances_noalloc: the entry point for callers that cannot allocate GPU memory.

Such callers (code inside a host callback or an allocator hook, processes whose device memory is
owned by another framework's pool, real-time loops that must not take the allocator's locks) get
the same distances as sdfgpu_distances, computed with a fixed device array instead of allocated
scratch.  This file runs last so that a failure here never hides the other GPU tests; it is also
self-contained, so it passes alone in a fresh process.
"""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DIST_TOL_DIAG = 1e-6  # the |d| tolerance of the parity tests, relative to the bounding-box diagonal


def _mesh(seed=4, level=3):
    from stl2sdf import DataImport
    from workloads import synthetic

    V, F = synthetic.icosphere(level, jitter=0.01, seed=seed)
    return DataImport.roundtrip_float32(V, F)


def _call(X_dev, nnp, IEN_dev, nel, origin, h, N, mode, out_dev):
    from stl2sdf import _native

    L = _native.lib()
    o = np.ascontiguousarray(origin, np.float64)
    n = np.ascontiguousarray(N, np.int64)
    rc = L.sdfgpu_distances_noalloc(ctypes.c_void_p(X_dev), nnp, ctypes.c_void_p(IEN_dev), nel,
                                    o.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), float(h),
                                    n.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), int(mode),
                                    ctypes.c_void_p(out_dev), None)
    return rc, L.sdfgpu_last_error(None).decode()


@pytest.mark.parametrize("mode", [1, 2])
def test_noalloc_matches_allocating_entry_point_and_oracle_twice(mode):
    """Two calls in a row with different meshes -- the second one smaller, so records the first
    call left in the array past the second mesh's triangles must be ignored -- each equal to the
    allocating entry point and to the oracle on the same mesh and grid."""
    import torch

    import oracle
    from stl2sdf import _native

    torch.cuda.set_device(0)
    for seed, level, cell in ((4, 3, 0.1), (9, 2, 0.12)):
        X, IEN = _mesh(seed, level)
        o, _, N, h, ngp = _native.grid_from_cell_size(X, cell)
        ctx = _native.Context(0)
        ctx.set_mesh(X, IEN)
        expected, _ = ctx.distances(o, h, N, mode)
        ctx.close()
        want, _, _ = oracle.distances(X, IEN, o, h, N, mode=mode)
        dX = torch.from_numpy(np.ascontiguousarray(X)).cuda()
        dIEN = torch.from_numpy(np.ascontiguousarray(IEN)).cuda()
        diag = float(np.linalg.norm(X.max(0) - X.min(0)))
        out = torch.full((ngp,), float("nan"), dtype=torch.float64, device="cuda")
        rc, msg = _call(dX.data_ptr(), X.shape[0], dIEN.data_ptr(), IEN.shape[0], o, h, N, mode, out.data_ptr())
        assert rc == 0, msg
        got = out.cpu().numpy()
        assert np.abs(got - want).max() <= DIST_TOL_DIAG * diag
        assert np.array_equal(got, want)
        assert np.array_equal(got, expected)


def test_noalloc_bad_index_leaves_the_output_unchanged():
    import torch

    X, IEN = _mesh(4, 1)
    IEN = IEN.copy()
    IEN[5, 1] = X.shape[0] + 7  # outside 1..nnp: the prep kernel flags it, the distance kernel skips
    dX = torch.from_numpy(np.ascontiguousarray(X)).cuda()
    dIEN = torch.from_numpy(np.ascontiguousarray(IEN)).cuda()
    out = torch.full((27,), 3.25, dtype=torch.float64, device="cuda")
    rc, msg = _call(dX.data_ptr(), X.shape[0], dIEN.data_ptr(), IEN.shape[0], [-1, -1, -1], 1.0, [2, 2, 2], 2,
                    out.data_ptr())
    assert rc == 1 and "1..nnp" in msg
    assert np.all(out.cpu().numpy() == 3.25)


def test_noalloc_rejects_meshes_beyond_its_array():
    import torch

    X = np.zeros((3, 3))
    IEN = np.ones((16385, 3), dtype=np.int64)
    dX = torch.zeros((3, 3), dtype=torch.float64, device="cuda")
    dIEN = torch.from_numpy(IEN).cuda()
    out = torch.empty(8, dtype=torch.float64, device="cuda")
    rc, msg = _call(dX.data_ptr(), X.shape[0], dIEN.data_ptr(), IEN.shape[0], [0, 0, 0], 0.1, [1, 1, 1], 1,
                    out.data_ptr())
    assert rc == 6 and "16384" in msg
    # nodes x triangles beyond 2^36 FP64 steps is refused before any launch
    IEN = np.ones((16384, 3), dtype=np.int64)
    dIEN = torch.from_numpy(IEN).cuda()
    rc, msg = _call(dX.data_ptr(), X.shape[0], dIEN.data_ptr(), IEN.shape[0], [0, 0, 0], 0.1, [2047, 2048, 0], 1,
                    out.data_ptr())
    assert rc == 6 and "2^36" in msg
