"""CPU FP64 oracle for the SignedDistances hot path -- TEST INFRASTRUCTURE ONLY.

ctypes bindings to ``oracle/_build/liboracle.so`` (built from ``oracle/sdf_oracle.cpp`` by
``oracle/Makefile``).  Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` may use this module, and only as the checker or the timed CPU baseline.  The product
(``stl2sdf.jl_b200``) never imports it.

The restatement follows the reference file by file (see the header of ``sdf_oracle.cpp``):
``src/MeshGrid/Grid.jl:9-32,82-96``, ``src/MeshGrid/Grid_setup.jl:104-124``,
``src/SignedDistances/dfOnTriangularMesh.jl:19-392`` and
``src/SignedDistances/RaycastingSignDetection.jl:35-404``.

PARITY UNPINNED: the reference is Julia and cannot run here, and it ships no golden vectors.
The oracle is pinned against analytic known answers instead (tests/test_oracle.py).
"""

from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

MODE_REF_RULE = 0
MODE_EXACT = 1
MODE_UNBOUNDED = 2

_dp = ctypes.POINTER(ctypes.c_double)
_i64p = ctypes.POINTER(ctypes.c_int64)
_i32p = ctypes.POINTER(ctypes.c_int32)


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(
            os.path.join(_HERE, "sdf_oracle.cpp")
        ):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        L.oracle_grid.argtypes = [_dp, _dp, ctypes.c_int64, ctypes.c_int64, _dp, _dp, _i64p, _dp, _i64p]
        L.oracle_grid_from_cell_size.argtypes = [_dp, ctypes.c_int64, ctypes.c_double, _dp, _dp, _i64p, _dp, _i64p]
        L.oracle_distances.argtypes = [
            _dp, ctypes.c_int64, _i64p, ctypes.c_int64, _dp, ctypes.c_double, _i64p, ctypes.c_int,
            _i64p, ctypes.c_int64, _dp, _dp, _i32p, ctypes.c_int,
        ]
        L.oracle_signs.argtypes = [
            _dp, ctypes.c_int64, _i64p, ctypes.c_int64, _dp, ctypes.c_double, _i64p, ctypes.c_int,
            ctypes.c_int, ctypes.c_double, ctypes.c_int, _i64p, ctypes.c_int64, _dp, _dp, _i32p,
            _i32p, _dp, ctypes.c_int,
        ]
        L.oracle_ray_directions.argtypes = [_dp]
        L.oracle_ray_triangle.argtypes = [_dp, _dp, _dp, _dp, _dp, ctypes.c_double, _dp]
        L.oracle_barycentric.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp]
        L.oracle_winding.argtypes = [_dp, ctypes.c_int64, _i64p, ctypes.c_int64, _dp, ctypes.c_int64, _dp, _dp, ctypes.c_int]
        L.oracle_work_model.argtypes = [_dp, ctypes.c_int64, _i64p, ctypes.c_int64, _dp, ctypes.c_double, _i64p, _i64p,
                                        ctypes.c_int64, _i64p, _i64p, _i64p, _i32p, _i64p, ctypes.c_int]
        L.oracle_max_threads.restype = ctypes.c_int
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _mesh_arrays(X, IEN):
    """X: (nnp, 3) float64 vertex rows; IEN: (nel, 3) int64, 1-based."""
    X = np.ascontiguousarray(X, dtype=np.float64).reshape(-1, 3)
    IEN = np.ascontiguousarray(IEN, dtype=np.int64).reshape(-1, 3)
    return X, IEN


def grid(xmin, xmax, n_max, margin=3):
    o = np.zeros(3); amax = np.zeros(3); N = np.zeros(3, np.int64); h = ctypes.c_double(); ngp = ctypes.c_int64()
    rc = lib().oracle_grid(_d(np.asarray(xmin, np.float64)), _d(np.asarray(xmax, np.float64)), int(n_max), int(margin),
                           _d(o), _d(amax), N.ctypes.data_as(_i64p), ctypes.byref(h), ctypes.byref(ngp))
    if rc != 0:
        raise ValueError(f"oracle_grid failed ({rc})")
    return dict(origin=o, amax=amax, N=N, h=h.value, ngp=ngp.value)


def grid_from_cell_size(X, B):
    X = np.ascontiguousarray(X, dtype=np.float64).reshape(-1, 3)
    o = np.zeros(3); amax = np.zeros(3); N = np.zeros(3, np.int64); h = ctypes.c_double(); ngp = ctypes.c_int64()
    rc = lib().oracle_grid_from_cell_size(_d(X), X.shape[0], float(B), _d(o), _d(amax), N.ctypes.data_as(_i64p),
                                          ctypes.byref(h), ctypes.byref(ngp))
    if rc != 0:
        raise ValueError(f"oracle_grid_from_cell_size failed ({rc})")
    return dict(origin=o, amax=amax, N=N, h=h.value, ngp=ngp.value)


def distances(X, IEN, origin, h, N, mode=MODE_REF_RULE, nodes=None, want_xp=False, nthreads=0):
    """Returns (dist, xp or None, flags).  flags bit0: knn fallback used; bit1: order sensitive."""
    X, IEN = _mesh_arrays(X, IEN)
    N = np.asarray(N, dtype=np.int64)
    origin = np.asarray(origin, dtype=np.float64)
    if nodes is not None:
        nodes = np.ascontiguousarray(nodes, dtype=np.int64)
        count = nodes.shape[0]
    else:
        count = int(np.prod(N + 1))
    dist = np.empty(count)
    xp = np.empty((count, 3)) if want_xp else None
    flags = np.empty(count, np.int32)
    rc = lib().oracle_distances(
        _d(X), X.shape[0], IEN.ctypes.data_as(_i64p), IEN.shape[0], _d(origin), float(h), N.ctypes.data_as(_i64p),
        int(mode), nodes.ctypes.data_as(_i64p) if nodes is not None else None, count, _d(dist),
        _d(xp) if xp is not None else None, flags.ctypes.data_as(_i32p), int(nthreads))
    if rc != 0:
        raise ValueError(f"oracle_distances failed ({rc})")
    return dist, xp, flags


def signs(X, IEN, origin, h, N, min_rays=6, max_rays=30, confidence_threshold=0.6, use_winding_fallback=True,
          nodes=None, nthreads=0):
    """Returns dict(sign, conf, rays, fallback, winding)."""
    X, IEN = _mesh_arrays(X, IEN)
    N = np.asarray(N, dtype=np.int64)
    origin = np.asarray(origin, dtype=np.float64)
    if nodes is not None:
        nodes = np.ascontiguousarray(nodes, dtype=np.int64)
        count = nodes.shape[0]
    else:
        count = int(np.prod(N + 1))
    sign = np.empty(count); conf = np.empty(count)
    rays = np.empty(count, np.int32); fb = np.empty(count, np.int32); w = np.empty(count)
    rc = lib().oracle_signs(
        _d(X), X.shape[0], IEN.ctypes.data_as(_i64p), IEN.shape[0], _d(origin), float(h), N.ctypes.data_as(_i64p),
        int(min_rays), int(max_rays), float(confidence_threshold), int(bool(use_winding_fallback)),
        nodes.ctypes.data_as(_i64p) if nodes is not None else None, count, _d(sign), _d(conf),
        rays.ctypes.data_as(_i32p), fb.ctypes.data_as(_i32p), _d(w), int(nthreads))
    if rc != 0:
        raise ValueError(f"oracle_signs failed ({rc})")
    return dict(sign=sign, conf=conf, rays=rays, fallback=fb, winding=w)


def ray_directions():
    out = np.empty((36, 3))
    lib().oracle_ray_directions(_d(out))
    return out


def ray_triangle(o, d, v1, v2, v3, eps=1e-8):
    t = ctypes.c_double()
    a = [np.ascontiguousarray(x, np.float64) for x in (o, d, v1, v2, v3)]
    hit = lib().oracle_ray_triangle(*[_d(x) for x in a], float(eps), ctypes.byref(t))
    return (t.value if hit else None)


def barycentric(x1, x2, x3, n, x):
    lam = np.empty(3)
    a = [np.ascontiguousarray(v, np.float64) for v in (x1, x2, x3, n, x)]
    lib().oracle_barycentric(*[_d(v) for v in a], _d(lam))
    return lam


def winding(X, IEN, pts, nthreads=0):
    X, IEN = _mesh_arrays(X, IEN)
    pts = np.ascontiguousarray(pts, np.float64).reshape(-1, 3)
    s = np.empty(pts.shape[0]); w = np.empty(pts.shape[0])
    rc = lib().oracle_winding(_d(X), X.shape[0], IEN.ctypes.data_as(_i64p), IEN.shape[0], _d(pts), pts.shape[0],
                              _d(s), _d(w), int(nthreads))
    if rc != 0:
        raise ValueError("oracle_winding failed")
    return s, w


def work_model(X, IEN, origin, h, N, nodes, nthreads=0):
    """Per-node algorithmic work counts: dict(nD, nD_unb, nrow (k x 3), nextra, rays); see oracle_work_model."""
    X, IEN = _mesh_arrays(X, IEN)
    N = np.asarray(N, dtype=np.int64)
    origin = np.asarray(origin, dtype=np.float64)
    nodes = np.ascontiguousarray(nodes, dtype=np.int64)
    k = nodes.shape[0]
    nD = np.empty(k, np.int64); nrow = np.empty((k, 3), np.int64); nextra = np.empty(k, np.int64)
    rays = np.empty(k, np.int32)
    nDu = np.empty(k, np.int64)
    rc = lib().oracle_work_model(_d(X), X.shape[0], IEN.ctypes.data_as(_i64p), IEN.shape[0], _d(origin), float(h),
                                 N.ctypes.data_as(_i64p), nodes.ctypes.data_as(_i64p), k, nD.ctypes.data_as(_i64p),
                                 nrow.ctypes.data_as(_i64p), nextra.ctypes.data_as(_i64p), rays.ctypes.data_as(_i32p),
                                 nDu.ctypes.data_as(_i64p), int(nthreads))
    if rc != 0:
        raise ValueError("oracle_work_model failed")
    return dict(nD=nD, nD_unb=nDu, nrow=nrow, nextra=nextra, rays=rays)


def max_threads() -> int:
    return int(lib().oracle_max_threads())
