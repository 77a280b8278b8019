"""CPU restatement of RBFs_smoothing -- TEST INFRASTRUCTURE ONLY.

Follows src/SdfSmoothing/RBFs4Smoothing.jl:
  * process_vector (:15-22): Float32 values; |v| approx 1e10 (Julia isapprox, rtol sqrt(eps(Float32)))
    becomes sign(v) * max{|v| : |v| < 1e9};
  * create_grid (:35-45): coarse node coordinates range(Float32(min), Float32(max), length = N+1)
    per axis, taken here as the Float64 point lo + (hi - lo) * i / N between the Float32 end points,
    rounded to Float32;
  * create_smooth_grid (:58-70): dx = (xmax - xmin) / (nx - 1) in Float32 from the x axis,
    coordinate = min + (i - 1) * dx in Float32 on every axis, nx = N * smooth + 1;
  * LimitedRangeRBFKernel (:97-101): r = sqrt of the Float32 sum of squared Float32 differences,
    value = exp(-(r / sigma)^2) in Float64, kept when > threshold (stored as Float32, :159-174);
  * compute_rbf_weights (:193-203): IterativeSolvers.cg(K, b) -- x0 = 0, the recurrence
    u = r + (|r|^2 / |r_prev|^2) u, c = K u, alpha = |r|^2 / (u . c), until |r| <= sqrt(eps(Float32)) |b|
    or size(K, 2) iterations; Float32 vectors;
  * rbf_interpolation_kdtree (:220-250): for each fine point the 124 nearest coarse points, in
    increasing distance, terms weight * exp(-(dist / sigma)^2) for dist <= Float32(sqrt(-log(thr)
    sigma^2)) added to a Float32 accumulator;
  * approximation (Is_interpolation = false) uses the processed values as the weights (:297-299).

NearestNeighbors.jl (knn order among equal distances, its Float32 distance arithmetic) and
OpenBLAS (sdot / snrm2 summation order inside cg) are third-party arithmetic that is not
restated bit for bit, so parity with this restatement is within a tolerance, stated in the tests.
"""

from __future__ import annotations

import numpy as np


def process_vector(vec):
    v = np.asarray(vec, dtype=np.float64).astype(np.float32)
    small = np.abs(v)[np.abs(v) < np.float32(1.0e9)]
    if small.size == 0:
        return v
    mx = np.float32(small.max())
    big = np.float32(1.0e10)
    rtol = np.float32(np.sqrt(np.finfo(np.float32).eps))
    near = np.abs(np.abs(v) - big) <= rtol * np.maximum(np.abs(v), big)
    return np.where(near, np.sign(v) * mx, v).astype(np.float32)


def coarse_axes(aabb_min, aabb_max, N):
    out = []
    for a in range(3):
        lo, hi = float(np.float32(aabb_min[a])), float(np.float32(aabb_max[a]))  # Float32 end points
        out.append(np.array([np.float32(lo + (hi - lo) * i / int(N[a])) for i in range(int(N[a]) + 1)], np.float32))
    return out


def fine_axes(aabb_min, aabb_max, N, smooth):
    n = np.asarray(N, np.int64) * int(smooth) + 1
    xmin = np.float32(aabb_min[0])
    xmax = np.float32(aabb_max[0])
    dx = np.float32(np.float32(xmax - xmin) / np.float32(n[0] - 1))
    return [np.array([np.float32(np.float32(aabb_min[a]) + np.float32(np.float32(i) * dx)) for i in range(int(n[a]))],
                     dtype=np.float32) for a in range(3)], dx


def _points(axes):
    X, Y, Z = np.meshgrid(axes[0], axes[1], axes[2], indexing="ij")
    # x fastest (Julia column-major order of [.. for x in x, y in y, z in z])
    return np.stack([X.transpose(2, 1, 0).reshape(-1), Y.transpose(2, 1, 0).reshape(-1),
                     Z.transpose(2, 1, 0).reshape(-1)], axis=1).astype(np.float32)


def kernel_matrix(axes, sigma, threshold):
    from scipy import sparse
    from scipy.spatial import cKDTree

    P = _points(axes)
    rad = sigma * np.sqrt(-np.log(threshold))
    pairs = cKDTree(P.astype(np.float64)).query_pairs(r=rad * (1 + 1e-6), output_type="ndarray")
    i, j = pairs[:, 0], pairs[:, 1]
    d = (P[i] - P[j]).astype(np.float32)
    r = np.sqrt((d * d).sum(axis=1, dtype=np.float32)).astype(np.float32)
    val = np.exp(-(r.astype(np.float64) / sigma) ** 2)
    keep = val > threshold
    i, j, val = i[keep], j[keep], val[keep].astype(np.float32)
    n = P.shape[0]
    diag = np.arange(n)
    I = np.concatenate([i, j, diag])
    J = np.concatenate([j, i, diag])
    V = np.concatenate([val, val, np.ones(n, np.float32)])
    return sparse.csr_matrix((V, (I, J)), shape=(n, n), dtype=np.float32)


def cg(K, b):
    """IterativeSolvers.cg recurrence and stopping rule, Float32 vectors."""
    b = np.asarray(b, np.float32)
    x = np.zeros_like(b)
    r = b.copy()
    u = np.zeros_like(b)
    res = np.float32(np.linalg.norm(r))
    prev = np.float32(1.0)
    tol = np.float32(np.sqrt(np.finfo(np.float32).eps)) * res
    it = 0
    while not (it >= K.shape[1] or res <= tol):
        beta = np.float32(res * res / (prev * prev))
        u = (r + beta * u).astype(np.float32)
        c = (K @ u).astype(np.float32)
        alpha = np.float32(res * res / np.float32(np.dot(u, c)))
        x = (x + alpha * u).astype(np.float32)
        r = (r - alpha * c).astype(np.float32)
        prev = res
        res = np.float32(np.linalg.norm(r))
        it += 1
    return x, it, float(res)


def evaluate(fine_axes_, coarse_axes_, weights, sigma, threshold, k=124):
    from scipy.spatial import cKDTree

    C = _points(coarse_axes_)
    F = _points(fine_axes_)
    maxd = np.float32(np.sqrt(-np.log(threshold) * sigma ** 2))
    tree = cKDTree(C.astype(np.float64))
    out = np.zeros(F.shape[0], np.float32)
    kk = min(k, C.shape[0])
    for s in range(0, F.shape[0], 65536):
        f = F[s:s + 65536]
        _, idx = tree.query(f.astype(np.float64), k=kk)
        idx = idx.reshape(f.shape[0], kk)
        d = (f[:, None, :] - C[idx]).astype(np.float32)
        dist = np.sqrt((d * d).sum(axis=2, dtype=np.float32)).astype(np.float32)
        order = np.argsort(dist, axis=1, kind="stable")
        dist = np.take_along_axis(dist, order, 1)
        idx = np.take_along_axis(idx, order, 1)
        acc = np.zeros(f.shape[0], np.float32)
        for q in range(kk):
            term = weights[idx[:, q]].astype(np.float64) * np.exp(-(dist[:, q].astype(np.float64) / sigma) ** 2)
            acc = np.where(dist[:, q] <= maxd, (acc.astype(np.float64) + term).astype(np.float32), acc)
        out[s:s + f.shape[0]] = acc
    return out


def rbf_smoothing(dist, aabb_min, aabb_max, N, cell_size, interpolation: bool, smooth: int, threshold=1e-3):
    """Returns (fine values Float32 (x fastest), fine dims, weights, cg iterations)."""
    vals = process_vector(dist)
    ca = coarse_axes(aabb_min, aabb_max, N)
    sigma = float(cell_size)
    its = 0
    if interpolation:
        K = kernel_matrix(ca, sigma, threshold)
        w, its, _ = cg(K, vals)
    else:
        w = vals
    fa, _ = fine_axes(aabb_min, aabb_max, N, smooth)
    out = evaluate(fa, ca, w, sigma, threshold)
    return out, np.asarray(N, np.int64) * int(smooth) + 1, w, its
