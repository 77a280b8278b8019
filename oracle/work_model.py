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

    X, IEN, g, desc = bench.make_workload(name)
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


def main(argv):
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
