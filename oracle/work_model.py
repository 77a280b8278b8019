"""Work model of the FP32 roofline -- TEST INFRASTRUCTURE (runs the CPU oracle).

For every bench workload, on a seeded uniform sample of grid nodes (2^16 nodes, seed 42; the
whole grid when it is smaller), the oracle counts the work any implementation of the hot path
must do per node:

    W(p) = F_PT * |D*(p)| + F_MT * ( sum_a rowhits_a(p) / (N_a + 1) + extrahits(p) )

* D*(p): triangles whose AABB lies within min(d_true(p), h) of p (d_true: the unbounded minimum)
  -- the candidates no box-pruned nearest search can skip.
* rowhits_a(p): triangles whose AABB meets the grid line through p along axis a.  The +a / -a
  rays of all N_a + 1 nodes on that line test the same triangles (the axis-ray hit set does not
  depend on the node's coordinate along the line), so each node is charged its share.
* extrahits(p): AABB hits of the rays beyond the six axis rays that the reference's adaptive
  vote casts at p (RaycastingSignDetection.jl:234-288).
* F_PT, F_MT: FP32 FLOPs (FMA = 2, division = 1) of the closed-form point-triangle distance
  (three segment distances, three edge-side tests, the plane distance) and of Moller-Trumbore.

Roofline nodes/s = P_fp32 / mean W.  The distance stage alone is bounded by F_PT |D*(p)|, and the
unclamped (unbounded) distance by F_PT |D*_u(p)| with D*_u(p) the triangles whose AABB lies within
d_true(p) of p.  Results go to profiles/roofline.json, which bench.py reads.

    python oracle/work_model.py [workload ...]      (default: icosphere torus128 blobs256 gyroid320)
    python oracle/work_model.py --tile-lists [workload ...]   (tile_lists below; default blobs256)
"""

from __future__ import annotations

import json
import os
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path[:0] = [ROOT, os.path.join(ROOT, "stl2sdf.jl_b200")]

import numpy as np  # noqa: E402

import oracle  # noqa: E402

F_PT = 162  # 9 (edges) + 3 x 25 (segment distances) + 17 (normal) + 51 (edge-side tests) + 10 (plane)
F_MT = 52   # 6 (edges) + 9 (h) + 5 (a) + 1 (1/a) + 3 (s) + 6 (u) + 9 (q) + 6 (v) + 1 (u+v) + 6 (t)
SAMPLE = 1 << 16
SEED = 42


def model(name: str) -> dict:
    import bench
    import workloads

    X, IEN, g = bench.load_reference(name)
    desc = workloads.description(name)
    ngp = int(g["ngp"])
    rng = np.random.default_rng(SEED)
    nodes = np.arange(ngp, dtype=np.int64) if ngp <= SAMPLE else np.sort(rng.choice(ngp, SAMPLE, replace=False))
    t0 = time.perf_counter()
    c = oracle.work_model(X, IEN, g["origin"], g["h"], g["N"], nodes)
    n_line = np.asarray(g["N"], np.float64) + 1.0
    ray_share = (c["nrow"] / n_line[None, :]).sum(axis=1) + c["nextra"]
    W = F_PT * c["nD"] + F_MT * ray_share
    return {
        "mean_W_dist_flop": float(F_PT * c["nD"].mean()),
        "mean_W_dist_unbounded_flop": float(F_PT * c["nD_unb"].mean()),
        "mean_Dstar_unbounded": float(c["nD_unb"].mean()),
        "workload": name, "description": desc, "ngp": ngp, "nel": int(IEN.shape[0]),
        "sample": f"{nodes.shape[0]} nodes" + (" (whole grid)" if nodes.shape[0] == ngp else f", uniform, seed {SEED}"),
        "F_pt": F_PT, "F_mt": F_MT, "mean_W_flop": float(W.mean()),
        "mean_Dstar": float(c["nD"].mean()), "mean_row_hits": [float(v) for v in c["nrow"].mean(axis=0)],
        "mean_ray_share": float(ray_share.mean()), "mean_extra_hits": float(c["nextra"].mean()),
        "mean_rays": float(c["rays"].mean()), "oracle_s": time.perf_counter() - t0,
    }


TILE_SAMPLE = 400


def _box_gap(lo, hi, blo, bhi):
    """Euclidean distance between axis-aligned boxes [lo, hi] (k x 3) and [blo, bhi] (3,)."""
    gap = np.maximum(0.0, np.maximum(lo - bhi[None, :], blo[None, :] - hi))
    return np.sqrt((gap * gap).sum(axis=1))


def tile_lists(name: str, tile=(4, 4, 2)) -> dict:
    """Candidate-list sizes of a radius-bounded tile fold against the reference rule's.

    A tile fold bounded per tile by a radius -- the learned radius's other use: every triangle whose
    AABB lies within R of the tile's node box is listed and tested at every node of the tile -- can
    be no better than its perfect radius, R = max over the tile's nodes of d_true(p).  On a seeded
    sample of tiles this counts that list, the least list any certified fold of the tile needs (the
    triangles whose AABB lies within d_true(p) of some node p), the list at the library's default
    certification margin with a perfect network, and with the same box rule the list for R = 2.5 h (the
    reference rule, dfOnTriangularMesh.jl:48,79, which the tile fold runs today).  The per-node work
    of a fold is its list length, so the ratio of the two means scales the measured fold time to
    what the radius-bounded fold would take."""
    import bench
    from scipy.spatial import cKDTree

    X, IEN, g = bench.load_reference(name)
    N = np.asarray(g["N"], np.int64)
    n = N + 1
    h = float(g["h"])
    o = np.asarray(g["origin"], np.float64)
    b = np.asarray(tile, np.int64)
    nt = (n + b - 1) // b
    rng = np.random.default_rng(SEED)
    k = min(TILE_SAMPLE, int(np.prod(nt)))
    tiles = np.sort(rng.choice(int(np.prod(nt)), k, replace=False))
    tz, rem = np.divmod(tiles, nt[0] * nt[1])
    ty, tx = np.divmod(rem, nt[0])
    lo_idx = np.stack([tx, ty, tz], axis=1) * b[None, :]
    hi_idx = np.minimum(lo_idx + b[None, :] - 1, N[None, :])
    nodes, owner = [], []
    for t in range(k):
        ii, jj, kk = (np.arange(lo_idx[t, a], hi_idx[t, a] + 1) for a in range(3))
        K, J, I = np.meshgrid(kk, jj, ii, indexing="ij")
        lin = (I + n[0] * (J + n[1] * K)).ravel()
        nodes.append(lin)
        owner.append(np.full(lin.shape[0], t))
    nodes = np.concatenate(nodes)
    owner = np.concatenate(owner)
    t0 = time.perf_counter()
    d, _, _ = oracle.distances(X, IEN, o, h, N, mode=oracle.MODE_UNBOUNDED, nodes=nodes)
    t_oracle = time.perf_counter() - t0
    r_tile = np.full(k, -np.inf)
    np.maximum.at(r_tile, owner, d)
    # the radius the library certifies with by default, r = 1.5 dhat + 4 H (alpha 0.5, beta 4 spacings H
    # of the 32-node training grid, H = mesh extent / 29), here with a perfect network (dhat = d_true)
    H = float((X.max(0) - X.min(0)).max()) / 29.0
    r_margin = np.full(k, -np.inf)
    np.maximum.at(r_margin, owner, 1.5 * d + 4.0 * H)
    V = X[IEN - 1]  # (nel, 3, 3); IEN is 1-based
    tlo, thi = V.min(axis=1), V.max(axis=1)
    cen = 0.5 * (tlo + thi)
    half = 0.5 * np.sqrt(((thi - tlo) ** 2).sum(axis=1)).max()
    tree = cKDTree(cen)
    n_learned = np.empty(k, np.int64)
    n_ref = np.empty(k, np.int64)
    n_union = np.empty(k, np.int64)
    n_margin = np.empty(k, np.int64)
    ijk = np.stack([nodes % n[0], (nodes // n[0]) % n[1], nodes // (n[0] * n[1])], axis=1)
    P = o[None, :] + ijk * h
    for t in range(k):
        # the least list any certified tile fold needs: the triangles within d_true(p) of some node
        sel = np.nonzero(owner == t)[0]
        hit = set()
        for q in sel:
            cand = np.asarray(tree.query_ball_point(P[q], d[q] + half), np.int64)
            if cand.size:
                hit.update(cand[_box_gap(tlo[cand], thi[cand], P[q], P[q]) <= d[q]].tolist())
        n_union[t] = len(hit)
        blo = o + lo_idx[t] * h
        bhi = o + hi_idx[t] * h
        bc = 0.5 * (blo + bhi)
        bh = 0.5 * np.sqrt(((bhi - blo) ** 2).sum())
        for R, out in ((r_tile[t], n_learned), (2.5 * h, n_ref), (r_margin[t], n_margin)):
            cand = np.asarray(tree.query_ball_point(bc, R + bh + half), np.int64)
            out[t] = int((_box_gap(tlo[cand], thi[cand], blo, bhi) <= R).sum()) if cand.size else 0
    return {
        "workload": name, "tile": [int(v) for v in b], "sample": f"{k} tiles, uniform, seed {SEED}",
        "mean_tile_radius_h": float((r_tile / h).mean()),
        "mean_list_perfect_radius": float(n_learned.mean()),
        "median_list_perfect_radius": float(np.median(n_learned)),
        "mean_list_union_perfect_radius": float(n_union.mean()),
        "mean_list_default_margin": float(n_margin.mean()),
        "mean_list_ref_rule": float(n_ref.mean()),
        "list_ratio": float(n_learned.mean() / max(n_ref.mean(), 1e-30)),
        "oracle_s": t_oracle,
    }


def main(argv):
    if argv[:1] == ["--tile-lists"]:
        path = os.path.join(ROOT, "profiles", "tile_lists.json")
        out = json.load(open(path)) if os.path.exists(path) else {}
        for n in argv[1:] or ["blobs256"]:
            out[n] = tile_lists(n)
            print(json.dumps(out[n]), flush=True)
            with open(path, "w") as f:
                json.dump(out, f, indent=1, sort_keys=True)
        return
    names = argv or ["icosphere", "torus128", "blobs256", "gyroid320"]
    path = os.path.join(ROOT, "profiles", "roofline.json")
    out = json.load(open(path)) if os.path.exists(path) else {}
    for n in names:
        out[n] = model(n)
        print(json.dumps(out[n]), flush=True)
        with open(path, "w") as f:
            json.dump(out, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    main(sys.argv[1:])
