"""Uneven batch (many meshes, each on its own grid, one call) and the tile autotuner.

The batch must give, per mesh, exactly what one sdfgpu_set_mesh + sdfgpu_sdf call gives with the
default tile; the autotuner may change the tile, never a result.  A few batch nodes are also
checked against the oracle directly.
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import sample_nodes

pytestmark = pytest.mark.gpu


def _batch(count, seed, k_lo, k_hi):
    from stl2sdf import DataImport, _native
    from workloads import synthetic

    out = []
    for r in synthetic.uneven_batch(count, seed=seed, k_lo=k_lo, k_hi=k_hi):
        if r["kind"] == "blobs":
            r["cells"] = min(r["cells"], 96)  # keep the oracle checks below quick
        X, IEN = DataImport.roundtrip_float32(*synthetic.batch_mesh(r))
        o, _, N, h, _ = _native.grid_setup(X.min(0), X.max(0), r["K"] - 7, 3)
        out.append((X, IEN, o, h, N))
    return out


@pytest.fixture(scope="module")
def small_batch():
    return _batch(12, seed=3, k_lo=24, k_hi=56)


def test_batch_equals_single_calls(gpu_ctx, small_batch):
    got = gpu_ctx.sdf_batch(small_batch, streams=4, autotune=True, want_parts=True)
    st = gpu_ctx.stats()
    assert st["ngp"] == sum(int(np.prod(np.asarray(m[4]) + 1)) for m in small_batch)
    for (X, IEN, o, h, N), parts in zip(small_batch, got):
        gpu_ctx.set_mesh(X, IEN)
        want = gpu_ctx.sdf(o, h, N, want_parts=True)
        for a, b in zip(parts, want):
            assert np.array_equal(a, b)
    # a second call reuses the workers and the tuned tiles
    again = gpu_ctx.sdf_batch(small_batch, streams=3, autotune=True)
    for a, parts in zip(again, got):
        assert np.array_equal(a, parts[0])


def test_batch_matches_oracle(gpu_ctx, small_batch):
    picks = sorted(range(len(small_batch)), key=lambda k: small_batch[k][1].shape[0])[:3]
    sub = [small_batch[k] for k in picks]
    got = gpu_ctx.sdf_batch(sub, streams=2, autotune=False, want_parts=True)
    for (X, IEN, o, h, N), (sdf, dist, sign, conf) in zip(sub, got):
        nodes = sample_nodes(sdf.shape[0], 1500, seed=11)
        d_ref, _, _ = oracle.distances(X, IEN, o, h, N, mode=0, nodes=nodes)
        r = oracle.signs(X, IEN, o, h, N, nodes=nodes)
        s_ref, c_ref = r["sign"], r["conf"]
        assert np.array_equal(dist[nodes], d_ref)
        assert np.array_equal(sign[nodes], s_ref)
        assert np.array_equal(conf[nodes], c_ref)
        assert np.array_equal(sdf[nodes], d_ref * s_ref)


def test_autotune_keeps_results(gpu_ctx, torus_mesh):
    from conftest import grid_of

    X, IEN = torus_mesh
    g = grid_of(X, n_nodes_long_axis=64)
    gpu_ctx.set_mesh(X, IEN)
    base, _ = gpu_ctx.distances(g["origin"], g["h"], g["N"], 0)
    tile, ms = gpu_ctx.autotune(g["origin"], g["h"], g["N"], 0)
    assert tile in [(4, 4, 4), (8, 4, 2), (4, 4, 2), (8, 4, 4), (4, 4, 8), (8, 8, 4)] and ms > 0
    tuned, _ = gpu_ctx.distances(g["origin"], g["h"], g["N"], 0)
    assert np.array_equal(base, tuned)
    for t in [(8, 8, 4), (4, 4, 2), (8, 4, 2)]:  # every shape, not only the winner, gives the same field
        from stl2sdf import _native

        c = _native.Context(0, tile=t)
        c.set_mesh(X, IEN)
        d, _ = c.distances(g["origin"], g["h"], g["N"], 0)
        c.close()
        assert np.array_equal(base, d), t


def test_batch_reports_failing_item(gpu_ctx, small_batch):
    from stl2sdf import _native

    bad = list(small_batch[:3])
    X, IEN, o, h, N = bad[1]
    bad[1] = (X, IEN, o, -1.0, N)
    with pytest.raises(_native.SdfGpuError) as e:
        gpu_ctx.sdf_batch(bad, streams=2)
    assert "batch item 1" in str(e.value)
    assert gpu_ctx.sdf_batch([], streams=2) == []


def _coarse_sphere_item():
    """80 large triangles on a fine grid: triangles reach farther than 1.5 cells from their
    centroids, so the 3-nearest-vertex fallback runs (inside the batch's graph)."""
    from stl2sdf import DataImport, _native
    from workloads import synthetic

    X, IEN = DataImport.roundtrip_float32(*synthetic.icosphere(1, jitter=0.01, seed=4))
    o, _, N, h, _ = _native.grid_setup(X.min(0), X.max(0), 48 - 7, 3)
    return (X, IEN, o, h, N)


@pytest.mark.parametrize("persistent", [False, True])
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_batch_modes_equal_single_calls(gpu_ctx, small_batch, mode, persistent):
    """Both batch forms (per-item pipelines; prepared items with one persistent fold launch in a
    CUDA graph) give every item exactly its single-call result, twice in a row."""
    items = list(small_batch[:5]) + [_coarse_sphere_item()]
    got = gpu_ctx.sdf_batch(items, mode=mode, streams=3, autotune=(mode != 1), want_parts=True, persistent=persistent)
    again = gpu_ctx.sdf_batch(items, mode=mode, streams=3, autotune=(mode != 1), persistent=persistent)
    for a, parts in zip(again, got):
        assert np.array_equal(a, parts[0])
    st = gpu_ctx.stats()
    if mode == 0:
        assert st["knn_fallback_nodes"] > 0  # the coarse sphere took the fallback
    for (X, IEN, o, h, N), parts in zip(items, got):
        gpu_ctx.set_mesh(X, IEN)
        want = gpu_ctx.sdf(o, h, N, mode=mode, want_parts=True)
        for a, b in zip(parts, want):
            assert np.array_equal(a, b)


def test_workload_batch_items_match_oracle(gpu_ctx):
    """Workload 4's own recipe (256 meshes, seed 3, grids of 32-160 nodes): the largest icosphere,
    the largest blob mesh and the coarsest blob mesh (big triangles on a fine grid: the
    nearest-vertex fallback) through the batch, in both forms, against the oracle on 1,500 seeded
    nodes each."""
    from stl2sdf import DataImport, _native
    from workloads import synthetic

    recipes = synthetic.uneven_batch(256, seed=3)
    ico = [r for r in recipes if r["kind"] == "icosphere"]
    blob = [r for r in recipes if r["kind"] == "blobs"]
    picks = [max(ico, key=lambda r: (r["level"], r["K"])), max(blob, key=lambda r: (r["cells"], r["K"])),
             min(blob, key=lambda r: (r["cells"], -r["K"]))]
    items = []
    for r in picks:
        X, IEN = DataImport.roundtrip_float32(*synthetic.batch_mesh(r))
        o, _, N, h, _ = _native.grid_setup(X.min(0), X.max(0), r["K"] - 7, 3)
        items.append((X, IEN, o, h, N))
    for persistent in (False, True):
        got = gpu_ctx.sdf_batch(items, streams=3, autotune=True, want_parts=True, persistent=persistent)
        for (X, IEN, o, h, N), (sdf, dist, sign, conf) in zip(items, got):
            nodes = sample_nodes(sdf.shape[0], 1500, seed=23)
            d_ref, _, _ = oracle.distances(X, IEN, o, h, N, mode=0, nodes=nodes)
            r = oracle.signs(X, IEN, o, h, N, nodes=nodes)
            assert np.array_equal(dist[nodes], d_ref)
            assert np.array_equal(sign[nodes], r["sign"]) and np.array_equal(conf[nodes], r["conf"])


def test_learned_batch_equals_unbounded_and_oracle(gpu_ctx, small_batch):
    """SDFGPU_MODE_LEARNED over the uneven batch, in both forms (per-item pipelines; prepared items
    whose searches all run in one persistent launch, two with the radius, inside a CUDA graph): every
    mesh trains its own radius network inside the call; the fields equal the plain unbounded batch
    bit for bit, every node is certified or counted as a fallback, and sampled nodes of three meshes
    equal the oracle's unbounded distance and its sign."""
    from stl2sdf import _native

    plain = gpu_ctx.sdf_batch(small_batch, mode=_native.MODE_UNBOUNDED, streams=4, autotune=True, want_parts=True)
    for persistent in (False, True):
        learned = gpu_ctx.sdf_batch(small_batch, mode=_native.MODE_LEARNED, streams=4, autotune=True, want_parts=True,
                                    persistent=persistent)
        st = gpu_ctx.stats()
        assert st["certified_nodes"] + st["unbounded_fallbacks"] == st["ngp"]
        assert st["certified_nodes"] > 0.9 * st["ngp"]
        assert st["train_launches"] > 0 and st["ms_train"] > 0
        for a, b in zip(learned, plain):
            for x, y in zip(a, b):
                assert np.array_equal(x, y)
    picks = sorted(range(len(small_batch)), key=lambda k: small_batch[k][1].shape[0])[:3]
    for k in picks:
        X, IEN, o, h, N = small_batch[k]
        sdf, dist, sign, conf = learned[k]
        nodes = sample_nodes(sdf.shape[0], 800, seed=5)
        d_ref, _, _ = oracle.distances(X, IEN, o, h, N, mode=2, nodes=nodes)
        assert np.array_equal(dist[nodes], d_ref)
        assert np.array_equal(sign[nodes], oracle.signs(X, IEN, o, h, N, nodes=nodes)["sign"])


def test_learned_batch_fallbacks_rerun_in_the_graph(gpu_ctx, small_batch):
    """The persistent learned batch with a zero search margin: the radius is the network's bare
    prediction, so many bricks are not certified and rerun in the graph's second launch (the listed
    plain search); the fields still equal the plain unbounded batch bit for bit."""
    from stl2sdf import _native

    plain = gpu_ctx.sdf_batch(small_batch, mode=_native.MODE_UNBOUNDED, streams=4, autotune=False, persistent=True)
    try:
        gpu_ctx.set_radius_margin(0.0, 0.0)
        learned = gpu_ctx.sdf_batch(small_batch, mode=_native.MODE_LEARNED, streams=4, autotune=False, persistent=True)
        st = gpu_ctx.stats()
    finally:
        gpu_ctx.set_radius_margin()
    assert st["unbounded_fallbacks"] > 0.05 * st["ngp"]
    assert st["certified_nodes"] + st["unbounded_fallbacks"] == st["ngp"]
    for a, b in zip(learned, plain):
        assert np.array_equal(a, b)
