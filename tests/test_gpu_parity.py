"""GPU parity: libsdfgpu.so (through its C ABI) against the FP64 oracle on the same inputs.

Bars (from the workload definitions): sign bit-exact; |d| error at most 1e-6 of the bounding-box
diagonal.  The GPU replays the reference's FP64 arithmetic for every decision that matters, so
distances are expected to be bit-identical as well; both properties are asserted.
"""

from __future__ import annotations

import os

import numpy as np
import pytest

import oracle
from conftest import GOLDEN, grid_of, sample_nodes

pytestmark = pytest.mark.gpu

DIST_TOL_DIAG = 1e-6  # |d| error bound, relative to the mesh bounding-box diagonal


def diag_of(X):
    return float(np.linalg.norm(X.max(axis=0) - X.min(axis=0)))


def check_dist(d_gpu, d_ref, X, exact=True):
    err = np.abs(d_gpu - d_ref)
    assert err.max() <= DIST_TOL_DIAG * diag_of(X), f"max |d| error {err.max()}"
    if exact:
        bad = np.flatnonzero(d_gpu != d_ref)
        assert bad.size == 0, f"{bad.size} distances differ bit-wise, first at {bad[:5]}: {d_gpu[bad[:5]]} vs {d_ref[bad[:5]]}"


def run_pair(ctx, X, IEN, g, mode=0, nodes=None, want_xp=False):
    ctx.set_mesh(X, IEN)
    d, xp = ctx.distances(g["origin"], g["h"], g["N"], mode, want_xp=want_xp)
    dr, xpr, fl = oracle.distances(X, IEN, g["origin"], g["h"], g["N"], mode=mode, nodes=nodes, want_xp=want_xp)
    if nodes is not None:
        d = d[nodes]
        xp = xp[nodes] if xp is not None else None
    return d, dr, xp, xpr, fl


def test_icosphere_ref_rule_full(gpu_ctx, icosphere_mesh):
    X, IEN = icosphere_mesh
    g = grid_of(X, cell=0.05)
    assert g["N"].tolist() == [46, 46, 46]
    d, dr, _, _, _ = run_pair(gpu_ctx, X, IEN, g, mode=0)
    check_dist(d, dr, X)
    assert np.all(d <= g["h"]) and np.all(d >= 0)


def test_icosphere_exact_full(gpu_ctx, icosphere_mesh):
    X, IEN = icosphere_mesh
    g = grid_of(X, cell=0.05)
    d, dr, _, _, _ = run_pair(gpu_ctx, X, IEN, g, mode=1)
    check_dist(d, dr, X)


def test_icosphere_unbounded_sample(gpu_ctx, icosphere_mesh):
    X, IEN = icosphere_mesh
    g = grid_of(X, cell=0.05)
    nodes = sample_nodes(g["ngp"], 4000)
    d, dr, _, _, _ = run_pair(gpu_ctx, X, IEN, g, mode=2, nodes=nodes)
    check_dist(d, dr, X)


def test_icosphere_signs_full(gpu_ctx, icosphere_mesh):
    X, IEN = icosphere_mesh
    g = grid_of(X, cell=0.05)
    gpu_ctx.set_mesh(X, IEN)
    s, c = gpu_ctx.signs(g["origin"], g["h"], g["N"])
    ref = oracle.signs(X, IEN, g["origin"], g["h"], g["N"])
    assert np.array_equal(s, ref["sign"])
    assert np.array_equal(c, ref["conf"])


def test_icosphere_fused_sdf(gpu_ctx, icosphere_mesh):
    X, IEN = icosphere_mesh
    g = grid_of(X, cell=0.05)
    gpu_ctx.set_mesh(X, IEN)
    sdf, dist, sign, conf = gpu_ctx.sdf(g["origin"], g["h"], g["N"], want_parts=True)
    assert np.array_equal(sdf, dist * sign)
    d2, _ = gpu_ctx.distances(g["origin"], g["h"], g["N"], 0)
    s2, _ = gpu_ctx.signs(g["origin"], g["h"], g["N"])
    assert np.array_equal(dist, d2) and np.array_equal(sign, s2)


def test_icosphere_closest_points(gpu_ctx, icosphere_mesh):
    X, IEN = icosphere_mesh
    g = grid_of(X, cell=0.05)
    d, dr, xp, xpr, _ = run_pair(gpu_ctx, X, IEN, g, mode=0, want_xp=True)
    check_dist(d, dr, X)
    assert np.array_equal(xp, xpr)


def test_torus_sample(gpu_ctx, torus_mesh):
    X, IEN = torus_mesh
    g = grid_of(X, n_nodes_long_axis=128)
    assert int(g["N"].max()) == 127
    nodes = sample_nodes(g["ngp"], 20000)
    d, dr, _, _, _ = run_pair(gpu_ctx, X, IEN, g, mode=0, nodes=nodes)
    check_dist(d, dr, X)
    s, c = gpu_ctx.signs(g["origin"], g["h"], g["N"])
    ref = oracle.signs(X, IEN, g["origin"], g["h"], g["N"], nodes=nodes)
    assert np.array_equal(s[nodes], ref["sign"])
    assert np.array_equal(c[nodes], ref["conf"])


def _open_box():
    from workloads import synthetic

    V, F = synthetic.box((0.0, 0.0, 0.0), (1.0, 0.7, 0.4))
    return V, F[2:]  # drop one face: rays through the hole disagree, winding fallback runs


def test_open_box_adaptive_and_winding(gpu_ctx):
    X, IEN = _open_box()
    g = grid_of(X, n_nodes_long_axis=24)
    gpu_ctx.set_mesh(X, IEN)
    s, c = gpu_ctx.signs(g["origin"], g["h"], g["N"])
    st = gpu_ctx.stats()
    ref = oracle.signs(X, IEN, g["origin"], g["h"], g["N"])
    assert st["undecided_nodes"] > 0
    assert np.array_equal(s, ref["sign"])
    assert np.array_equal(c, ref["conf"])
    d, dr, _, _, _ = run_pair(gpu_ctx, X, IEN, g, mode=0)
    check_dist(d, dr, X)


@pytest.mark.parametrize("min_rays,max_rays,thr,wind", [(4, 10, 0.6, True), (6, 30, 0.9, False), (1, 36, 0.99, True),
                                                        (8, 60, 0.6, True)])
def test_vote_parameters(gpu_ctx, min_rays, max_rays, thr, wind):
    X, IEN = _open_box()
    g = grid_of(X, n_nodes_long_axis=20)
    gpu_ctx.set_mesh(X, IEN)
    s, c = gpu_ctx.signs(g["origin"], g["h"], g["N"], min_rays, max_rays, thr, wind)
    ref = oracle.signs(X, IEN, g["origin"], g["h"], g["N"], min_rays, max_rays, thr, wind)
    assert np.array_equal(s, ref["sign"])
    assert np.array_equal(c, ref["conf"])


def test_single_triangle():
    from stl2sdf import _native

    ctx = _native.Context(0)
    X = np.array([[0.0, 0.0, 0.0], [1.0, 0.1, 0.0], [0.2, 0.9, 0.3]])
    IEN = np.array([[1, 2, 3]])
    g = oracle.grid(X.min(0), X.max(0), 10, 3)
    d, dr, _, _, _ = run_pair(ctx, X, IEN, g, mode=0)
    check_dist(d, dr, X)
    d, dr, _, _, _ = run_pair(ctx, X, IEN, g, mode=1)
    check_dist(d, dr, X)
    s, c = ctx.signs(g["origin"], g["h"], g["N"])
    ref = oracle.signs(X, IEN, g["origin"], g["h"], g["N"])
    assert np.array_equal(s, ref["sign"]) and np.array_equal(c, ref["conf"])
    ctx.close()


def test_degenerate_triangles(gpu_ctx, icosphere_mesh):
    """Zero-area triangles (NaN normals in the reference) take only the edge and vertex branches."""
    X, IEN = icosphere_mesh
    X2 = np.vstack([X, X[:1] + [0.0, 0.0, 0.0], X[:1] * 1.05])
    n = X.shape[0]
    extra = np.array([[1, n + 1, n + 2], [n + 1, n + 1, n + 2]])  # collinear and repeated-vertex triangles
    IEN2 = np.vstack([IEN, extra])
    g = grid_of(X2, cell=0.08)
    d, dr, _, _, _ = run_pair(gpu_ctx, X2, IEN2, g, mode=0)
    check_dist(d, dr, X2)


def test_ragged_grids(gpu_ctx, icosphere_mesh):
    X, IEN = icosphere_mesh
    gpu_ctx.set_mesh(X, IEN)
    for N in ([0, 5, 17], [33, 0, 0], [7, 40, 3]):
        N = np.array(N, np.int64)
        o = np.array([-1.2, -1.1, -0.3])
        h = 0.061
        d, _ = gpu_ctx.distances(o, h, N, 0)
        dr, _, _ = oracle.distances(X, IEN, o, h, N, mode=0)
        check_dist(d, dr, X)
        s, c = gpu_ctx.signs(o, h, N)
        ref = oracle.signs(X, IEN, o, h, N)
        assert np.array_equal(s, ref["sign"]) and np.array_equal(c, ref["conf"])


def test_artifacts_stl_reference_fixture(gpu_ctx):
    """The reference's own test input (data/artifacts.stl) at its test cell size 0.5: large
    triangles, so the 3-nearest-vertex fallback of the candidate rule is exercised."""
    from stl2sdf import DataImport

    X, IEN = DataImport.import_stl(os.path.join(GOLDEN, "artifacts.stl"))
    g = grid_of(X, cell=0.5)
    d, dr, _, _, fl = run_pair(gpu_ctx, X, IEN, g, mode=0)
    assert (fl & 1).any()
    check_dist(d, dr, X)
    s, c = gpu_ctx.signs(g["origin"], g["h"], g["N"])
    ref = oracle.signs(X, IEN, g["origin"], g["h"], g["N"])
    assert np.array_equal(s, ref["sign"]) and np.array_equal(c, ref["conf"])


def test_errors_are_reported(gpu_ctx):
    from stl2sdf import _native

    ctx = _native.Context(0)
    with pytest.raises(_native.SdfGpuError) as e:
        ctx.distances([0, 0, 0], 0.1, [3, 3, 3])
    assert e.value.code == 5  # no mesh
    with pytest.raises(_native.SdfGpuError) as e:
        ctx.set_mesh(np.zeros((3, 3)), np.array([[1, 2, 4]]))
    assert e.value.code == 1
    ctx.set_mesh(np.eye(3), np.array([[1, 2, 3]]))
    with pytest.raises(_native.SdfGpuError):
        ctx.distances([0, 0, 0], -1.0, [3, 3, 3])
    with pytest.raises(_native.SdfGpuError):
        ctx.signs([0, 0, 0], 0.1, [3, 3, 3], min_rays=0)
    # a grid beyond 2^31 - 1 nodes is refused before anything is allocated (z slabs split it)
    with pytest.raises(_native.SdfGpuError, match="2\\^31") as e:
        ctx.distances([0, 0, 0], 0.1, [2000, 2000, 2000])
    assert e.value.code == 1
    # non-finite vertices are rejected by the mesh upload
    Xn = np.eye(3)
    Xn[1, 2] = np.nan
    with pytest.raises(_native.SdfGpuError, match="finite") as e:
        ctx.set_mesh(Xn, np.array([[1, 2, 3]]))
    assert e.value.code == 1
    ctx.close()


def test_blobs_small_full(gpu_ctx):
    """Marching-cubes blob mesh (16 blobs, 96^3 lattice) on a 64-node grid, every node."""
    from stl2sdf import DataImport
    from workloads import synthetic

    V, F = synthetic.blobs(16, seed=5, cells=96)
    X, IEN = DataImport.roundtrip_float32(V, F)
    g = grid_of(X, n_nodes_long_axis=64)
    d, dr, _, _, fl = run_pair(gpu_ctx, X, IEN, g, mode=0)
    check_dist(d, dr, X)
    s, c = gpu_ctx.signs(g["origin"], g["h"], g["N"])
    ref = oracle.signs(X, IEN, g["origin"], g["h"], g["N"])
    assert np.array_equal(s, ref["sign"]) and np.array_equal(c, ref["conf"])


def test_gyroid_small_full(gpu_ctx):
    """Capped gyroid sheet (one period, 48^3 lattice): thin walls, grazing axis rays, adaptive
    vote and winding fallback; every node of a 48-node grid."""
    from stl2sdf import DataImport
    from workloads import synthetic

    V, F = synthetic.gyroid(48, 0.04, 1.0)
    X, IEN = DataImport.roundtrip_float32(V, F)
    g = grid_of(X, n_nodes_long_axis=48)
    d, dr, _, _, _ = run_pair(gpu_ctx, X, IEN, g, mode=0)
    check_dist(d, dr, X)
    d, dr, _, _, _ = run_pair(gpu_ctx, X, IEN, g, mode=1)
    check_dist(d, dr, X)
    s, c = gpu_ctx.signs(g["origin"], g["h"], g["N"])
    st = gpu_ctx.stats()
    ref = oracle.signs(X, IEN, g["origin"], g["h"], g["N"])
    assert np.array_equal(s, ref["sign"]) and np.array_equal(c, ref["conf"])
    assert st["undecided_nodes"] == int(np.count_nonzero(ref["rays"] > 6))


def _bipyramid(k=24):
    """Closed double fan: two apexes shared by k triangles each (a vertex far above the number of
    triangles the unbounded search keeps per node in its FP32 band, so nodes on the axis take
    the exact re-search)."""
    ang = 2 * np.pi * np.arange(k) / k
    V = np.concatenate([[[0.0, 0.0, 1.0], [0.0, 0.0, -1.0]], np.stack([np.cos(ang), np.sin(ang), np.zeros(k)], 1)])
    F = []
    for q in range(k):
        a, b = 2 + q, 2 + (q + 1) % k
        F.append([0, a, b])
        F.append([1, b, a])
    return V, np.asarray(F)


@pytest.mark.parametrize("brick", [(4, 2, 4), (32, 1, 1)])
def test_unbounded_high_valence_vertex(gpu_ctx, brick):
    from stl2sdf import DataImport

    X, IEN = DataImport.roundtrip_float32(*_bipyramid())
    g = grid_of(X, cell=0.1)
    gpu_ctx.set_brick(brick)
    try:
        d, dr, _, _, _ = run_pair(gpu_ctx, X, IEN, g, mode=2)
    finally:
        gpu_ctx.set_brick((4, 2, 4))
    check_dist(d, dr, X)


def test_unbounded_brick_autotune(gpu_ctx, icosphere_mesh):
    X, IEN = icosphere_mesh
    g = grid_of(X, cell=0.05)
    gpu_ctx.set_mesh(X, IEN)
    d0, _ = gpu_ctx.distances(g["origin"], g["h"], g["N"], 2)
    brick, ms = gpu_ctx.autotune(g["origin"], g["h"], g["N"], mode=2)
    assert int(np.prod(brick)) == 32 and ms > 0
    d1, _ = gpu_ctx.distances(g["origin"], g["h"], g["N"], 2)
    gpu_ctx.set_brick((4, 2, 4))
    assert np.array_equal(d0, d1)


def test_fp32_peak_probe():
    import workloads

    t = workloads.measure_fp32_peak(0)
    # 148 SMs x 128 FP32 lanes x 2 FLOPs at 1.0-2.0 GHz: well inside (20, 100) TFLOP/s
    assert 20.0 < t < 100.0, t
