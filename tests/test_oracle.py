"""The FP64 oracle against analytic known answers (the reference ships no golden vectors).

Covers: the Grid constructor arithmetic (Grid.jl:9-32), the per-triangle distance in its face,
edge and vertex regions including the reference's vertex-skip rule (dfOnTriangularMesh.jl:140-176),
Möller–Trumbore decisions (RaycastingSignDetection.jl:64-106), the prioritized ray directions
(:162-227), the winding number (:295-328) and the sign/distance of closed analytic shapes.
"""

from __future__ import annotations

import math

import numpy as np
import pytest

import oracle
from conftest import grid_of

TRI = (np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]]), np.array([[1, 2, 3]]))


def one_node(p, mode, h=10.0):
    """Distance of the single node p (a 1-node grid with a large cell so the clamp is inactive)."""
    X, IEN = TRI
    d, xp, fl = oracle.distances(X, IEN, np.asarray(p, float), h, [0, 0, 0], mode=mode, want_xp=True)
    return d[0], xp[0], fl[0]


def test_grid_constructor_by_hand():
    g = oracle.grid([0.0, 0.0, 0.0], [1.0, 2.0, 4.0], 8, 3)
    assert g["h"] == 0.5
    assert g["origin"].tolist() == [-1.5, -1.5, -1.5]
    assert g["N"].tolist() == [8, 10, 14]
    assert g["amax"].tolist() == [-1.5 + 8 * 0.5, -1.5 + 10 * 0.5, -1.5 + 14 * 0.5]
    assert g["ngp"] == 9 * 11 * 15


def test_grid_from_cell_size_by_hand():
    X = np.array([[0.0, 0.0, 0.0], [3.0, 1.0, 0.5]])
    g = oracle.grid_from_cell_size(X, 0.7)  # N_new = floor(3 / 0.7) = 4 -> h = 0.75
    assert g["h"] == 0.75
    assert g["N"][0] == math.ceil((3.0 + 6 * 0.75) / 0.75)


def test_face_region():
    d, xp, _ = one_node([0.2, 0.2, 0.5], 0)
    assert d == pytest.approx(0.5, abs=1e-15)
    assert np.allclose(xp, [0.2, 0.2, 0.0], atol=1e-15)


def test_edge_region():
    d, xp, _ = one_node([0.5, -0.3, 0.4], 0)
    assert d == pytest.approx(0.5, abs=1e-15)
    assert np.allclose(xp, [0.5, 0.0, 0.0], atol=1e-15)


def test_vertex_skip_rule():
    """p projects outside the triangle next to v1; the foot on the opposite edge (v2-v3) is valid
    and improves the initial minimum, so the reference never looks at the vertices: it returns
    the distance to that foot (1.2021), not the true distance to v1 (0.5)."""
    p = [-0.3, -0.4, 0.0]
    d_ref, xp_ref, fl = one_node(p, 0)
    foot = np.array([1.0, 0.0, 0.0]) + np.array([-1.0, 1.0, 0.0]) / math.sqrt(2) * (0.9 / math.sqrt(2))
    assert d_ref == pytest.approx(np.linalg.norm(np.array(p) - foot), rel=1e-14)
    assert fl & 2  # flagged as order sensitive (differs from the true minimum)
    d_ex, xp_ex, _ = one_node(p, 1)
    assert d_ex == pytest.approx(0.5, abs=1e-15)
    assert np.allclose(xp_ex, [0.0, 0.0, 0.0])


def test_clamp_to_cell_size():
    X, IEN = TRI
    d, _, _ = oracle.distances(X, IEN, np.array([0.2, 0.2, 5.0]), 1.0, [0, 0, 0], mode=0)
    assert d[0] == 1.0  # |d| > cell_size -> cell_size


def test_unbounded_is_true_distance():
    X, IEN = TRI
    d, _, _ = oracle.distances(X, IEN, np.array([0.2, 0.2, 5.0]), 1.0, [0, 0, 0], mode=2)
    assert d[0] == pytest.approx(5.0, abs=1e-15)


def test_barycentric_of_projection():
    lam = oracle.barycentric([0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0.25, 0.5, 3.0])
    assert np.allclose(lam, [0.25, 0.25, 0.5], atol=1e-15)


def test_moller_trumbore_known_answers():
    v1, v2, v3 = [0, 0, 0], [1, 0, 0], [0, 1, 0]
    assert oracle.ray_triangle([0.2, 0.2, -1.0], [0, 0, 1], v1, v2, v3) == pytest.approx(1.0)
    assert oracle.ray_triangle([0.2, 0.2, 1.0], [0, 0, 1], v1, v2, v3) is None  # behind
    assert oracle.ray_triangle([0.2, 0.2, -1.0], [1, 0, 0], v1, v2, v3) is None  # parallel
    assert oracle.ray_triangle([0.2, 0.2, 0.0], [0, 0, 1], v1, v2, v3) is None  # t = 0 <= eps
    assert oracle.ray_triangle([0.0, 0.5, -1.0], [0, 0, 1], v1, v2, v3) == pytest.approx(1.0)  # on an edge: u = 0 counts
    assert oracle.ray_triangle([0.6, 0.6, -1.0], [0, 0, 1], v1, v2, v3) is None  # u + v > 1


def test_ray_directions():
    D = oracle.ray_directions()
    assert D.shape == (36, 3)
    assert D[:6].tolist() == [[1, 0, 0], [0, 1, 0], [0, 0, 1], [-1, 0, 0], [0, -1, 0], [0, 0, -1]]
    s2 = 1.0 * (1.0 / math.sqrt(2.0))
    assert D[6].tolist() == [s2, s2, 0.0]
    s3 = 1.0 * (1.0 / math.sqrt(3.0))
    assert D[18].tolist() == [s3, s3, s3]
    phi = (1.0 + math.sqrt(5.0)) / 2.0
    for i in range(1, 11):
        th = 2.0 * math.pi * math.fmod(i * phi, 1.0)
        z = 1.0 - 2.0 * (i / 10.0)
        r = math.sqrt(1.0 - z * z)
        assert D[25 + i] == pytest.approx([r * math.cos(th), r * math.sin(th), z], abs=1e-15)
    assert np.allclose(np.linalg.norm(D, axis=1), 1.0, atol=1e-15)


def test_winding_number_of_box():
    from workloads import synthetic

    X, IEN = synthetic.box((0, 0, 0), (1, 1, 1))
    s, w = oracle.winding(X, IEN, [[0.5, 0.5, 0.5], [2.0, 0.5, 0.5], [0.1, 0.9, 0.5]])
    assert s.tolist() == [1.0, -1.0, 1.0]
    assert abs(abs(w[0]) - 1.0) < 1e-12 and abs(w[1]) < 1e-12


def test_sphere_signs_and_distances(icosphere_mesh):
    X, IEN = icosphere_mesh
    g = grid_of(X, cell=0.05)
    s = oracle.signs(X, IEN, g["origin"], g["h"], g["N"])
    n = g["N"] + 1
    i, j, k = np.meshgrid(np.arange(n[0]), np.arange(n[1]), np.arange(n[2]), indexing="ij")
    P = np.stack([g["origin"][0] + g["h"] * i.T.ravel(), g["origin"][1] + g["h"] * j.T.ravel(),
                  g["origin"][2] + g["h"] * k.T.ravel()], 1)
    r = np.linalg.norm(P, axis=1)
    assert np.all(s["sign"][r < 0.95] == 1.0) and np.all(s["sign"][r > 1.05] == -1.0)
    assert np.all(s["conf"] == 1.0)
    d, _, fl = oracle.distances(X, IEN, g["origin"], g["h"], g["N"], mode=0)
    de, _, _ = oracle.distances(X, IEN, g["origin"], g["h"], g["N"], mode=1)
    assert np.array_equal(d, de)  # convex mesh with small triangles: the rule finds the true minimum
    assert not (fl & 2).any()
    near = np.abs(r - 1.0) < 0.5 * g["h"]
    assert np.all(np.abs(d[near] - np.abs(r[near] - 1.0)) < 0.04)  # radial jitter N(0, 0.01)


def test_unjittered_sphere_distance_bound():
    from stl2sdf import DataImport
    from workloads import synthetic

    V, F = synthetic.icosphere(3, jitter=0.0)
    X, IEN = DataImport.roundtrip_float32(V, F)
    g = grid_of(X, cell=0.1)
    d, _, _ = oracle.distances(X, IEN, g["origin"], g["h"], g["N"], mode=2)
    n = g["N"] + 1
    i, j, k = np.meshgrid(np.arange(n[0]), np.arange(n[1]), np.arange(n[2]), indexing="ij")
    P = np.stack([g["origin"][0] + g["h"] * i.T.ravel(), g["origin"][1] + g["h"] * j.T.ravel(),
                  g["origin"][2] + g["h"] * k.T.ravel()], 1)
    r = np.linalg.norm(P, axis=1)
    # inscribed polyhedron: true sphere distance minus the faceting sagitta <= d <= sphere distance + sagitta
    assert np.all(np.abs(d - np.abs(r - 1.0)) < 0.02)


def test_work_model_counts_single_triangle():
    """The roofline's work counts on one triangle (0,0,0)-(1,0,0)-(0,1,0), grid nodes at
    (0.25|0.75, 0.25|0.75, 0.3|0.8) with h = 0.5, worked out by hand:
    D*(p) = triangles whose box lies within min(d_true, h) of p; D*_u with d_true alone; row hits =
    triangles whose box meets the grid line through p along x, y, z."""
    X = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0]])
    IEN = np.array([[1, 2, 3]])
    o, h, N = np.array([0.25, 0.25, 0.3]), 0.5, np.array([1, 1, 1])
    nodes = np.array([0, 3, 4], dtype=np.int64)  # (0.25,0.25,0.3), (0.75,0.75,0.3), (0.25,0.25,0.8)
    c = oracle.work_model(X, IEN, o, h, N, nodes)
    # d_true: 0.3 (face), sqrt(2 * 0.25^2 + 0.3^2) = 0.464 (hypotenuse), 0.8 (> h)
    assert c["nD"].tolist() == [1, 1, 0]
    assert c["nD_unb"].tolist() == [1, 1, 1]
    # only the z line through (x, y) inside the box meets it (z = 0.3 / 0.8 is outside [0, 0])
    assert c["nrow"].tolist() == [[0, 0, 1], [0, 0, 1], [0, 0, 1]]
    assert np.all(c["rays"] >= 6)


def test_tile_list_model_orders_the_lists():
    """The tile-list model on the icosphere workload: the least certified list (triangles within
    d_true(p) of some node) is contained in the perfect-radius ball list, which the default-margin
    list contains; every list is a count of triangles of the mesh."""
    import importlib

    r = importlib.import_module("oracle.work_model").tile_lists("icosphere")
    nel = 5120
    assert 0 < r["mean_list_union_perfect_radius"] <= r["mean_list_perfect_radius"] <= r["mean_list_default_margin"] <= nel
    assert 0 < r["mean_list_ref_rule"] <= nel
    assert r["mean_tile_radius_h"] > 0
