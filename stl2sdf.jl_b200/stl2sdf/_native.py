"""ctypes binding of libsdfgpu.so (the C ABI declared in include/sdfgpu.h).

The library is built in-tree into ``stl2sdf.jl_b200/lib/libsdfgpu.so`` (``make -C
stl2sdf.jl_b200/csrc``).  There is no CPU fallback: if the library is missing or no sm_100
device is present, every compute call raises :class:`SdfGpuError`.
"""

from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.abspath(os.path.join(_PKG, "..", "lib", "libsdfgpu.so"))

SDFGPU_OK = 0
STATUS_NAMES = {
    0: "OK", 1: "INVALID_ARGUMENT", 2: "NO_DEVICE", 3: "CUDA", 4: "OUT_OF_MEMORY", 5: "NO_MESH", 6: "CAPACITY", 7: "IO",
}
MODE_REF_RULE = 0
MODE_EXACT = 1
MODE_UNBOUNDED = 2
MODE_LEARNED = 3

_dp = ctypes.POINTER(ctypes.c_double)
_i64p = ctypes.POINTER(ctypes.c_int64)


class SdfGpuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"sdfgpu error {code} ({STATUS_NAMES.get(code, '?')}): {msg}")
        self.code = code


class Opts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("tile", ctypes.c_int32 * 3)]


class Stats(ctypes.Structure):
    _fields_ = [
        ("ngp", ctypes.c_int64), ("nel", ctypes.c_int64), ("tile_pairs", ctypes.c_int64),
        ("active_tiles", ctypes.c_int64), ("candidate_nodes", ctypes.c_int64), ("fp64_evals", ctypes.c_int64),
        ("knn_fallback_nodes", ctypes.c_int64), ("band_nodes", ctypes.c_int64), ("row_hits", ctypes.c_int64),
        ("undecided_nodes", ctypes.c_int64), ("extra_rays", ctypes.c_int64), ("winding_nodes", ctypes.c_int64),
        ("winding_ambiguous", ctypes.c_int64), ("unbounded_fallbacks", ctypes.c_int64), ("rho_max", ctypes.c_double),
        ("ms_distance", ctypes.c_double), ("ms_sign", ctypes.c_double), ("ms_mesh", ctypes.c_double),
        ("launches", ctypes.c_int64), ("mesh_launches", ctypes.c_int64), ("ms_tiles", ctypes.c_double),
        ("ms_fold", ctypes.c_double), ("ms_rows", ctypes.c_double), ("ms_parity", ctypes.c_double),
        ("ms_vote", ctypes.c_double), ("certified_nodes", ctypes.c_int64), ("radius_loss", ctypes.c_double),
        ("bvh_visits", ctypes.c_int64), ("ms_train", ctypes.c_double), ("train_launches", ctypes.c_int64),
        ("sign_band_reruns", ctypes.c_int64),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class BatchItem(ctypes.Structure):
    _fields_ = [
        ("X", _dp), ("nnp", ctypes.c_int64), ("IEN", _i64p), ("nel", ctypes.c_int64),
        ("origin", ctypes.c_double * 3), ("h", ctypes.c_double), ("N", ctypes.c_int64 * 3),
        ("sdf", _dp), ("dist", _dp), ("sign", _dp), ("conf", _dp),
    ]


# Every symbol include/sdfgpu.h declares, with its ctypes signature.
SIGNATURES = {
    "sdfgpu_abi_version": ([], ctypes.c_int),
    "sdfgpu_create": ([ctypes.POINTER(Opts), ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "sdfgpu_destroy": ([ctypes.c_void_p], ctypes.c_int),
    "sdfgpu_last_error": ([ctypes.c_void_p], ctypes.c_char_p),
    "sdfgpu_grid_setup": ([_dp, _dp, ctypes.c_int64, ctypes.c_int64, _dp, _dp, _i64p, _dp, _i64p], ctypes.c_int),
    "sdfgpu_grid_from_cell_size": ([_dp, ctypes.c_int64, ctypes.c_double, _dp, _dp, _i64p, _dp, _i64p], ctypes.c_int),
    "sdfgpu_set_mesh": ([ctypes.c_void_p, _dp, ctypes.c_int64, _i64p, ctypes.c_int64], ctypes.c_int),
    "sdfgpu_set_mesh_device": ([ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64],
                               ctypes.c_int),
    "sdfgpu_distances": ([ctypes.c_void_p, _dp, ctypes.c_double, _i64p, _dp, _dp, ctypes.c_int32, ctypes.c_int32],
                         ctypes.c_int),
    "sdfgpu_signs": ([ctypes.c_void_p, _dp, ctypes.c_double, _i64p, ctypes.c_int32, ctypes.c_int32, ctypes.c_double,
                      ctypes.c_int32, _dp, _dp], ctypes.c_int),
    "sdfgpu_sdf": ([ctypes.c_void_p, _dp, ctypes.c_double, _i64p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                    ctypes.c_double, ctypes.c_int32, _dp, _dp, _dp, _dp], ctypes.c_int),
    "sdfgpu_sdf_device": ([ctypes.c_void_p, _dp, ctypes.c_double, _i64p, ctypes.c_int32, ctypes.c_int32,
                           ctypes.c_int32, ctypes.c_double, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p,
                           ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "sdfgpu_sdf_slab": ([ctypes.c_void_p, _dp, ctypes.c_double, _i64p, ctypes.c_int64, ctypes.c_int64, ctypes.c_int32,
                         ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_int32, _dp, _dp, _dp, _dp],
                        ctypes.c_int),
    "sdfgpu_sdf_slab_device": ([ctypes.c_void_p, _dp, ctypes.c_double, _i64p, ctypes.c_int64, ctypes.c_int64,
                                ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_int32,
                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "sdfgpu_distances_noalloc": ([ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64, _dp,
                                  ctypes.c_double, _i64p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p], ctypes.c_int),
    "sdfgpu_train_radius": ([ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_float,
                             ctypes.c_uint64, ctypes.POINTER(ctypes.c_float)], ctypes.c_int),
    "sdfgpu_radius_param_count": ([], ctypes.c_int),
    "sdfgpu_radius_params": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_float), _dp], ctypes.c_int),
    "sdfgpu_set_radius_params": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_float), _dp], ctypes.c_int),
    "sdfgpu_radius_eval": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_float), ctypes.c_int64,
                            ctypes.POINTER(ctypes.c_float)], ctypes.c_int),
    "sdfgpu_mlp_train_eval": ([ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_float)] * 3 + [ctypes.c_int64]
                              + [ctypes.POINTER(ctypes.c_float)] * 3, ctypes.c_int),
    "sdfgpu_sdf_batch": ([ctypes.c_void_p, ctypes.POINTER(BatchItem), ctypes.c_int64, ctypes.c_int32, ctypes.c_int32,
                          ctypes.c_int32, ctypes.c_double, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32],
                         ctypes.c_int),
    "sdfgpu_sdf_batch_ex": ([ctypes.c_void_p, ctypes.POINTER(BatchItem), ctypes.c_int64, ctypes.c_int32, ctypes.c_int32,
                             ctypes.c_int32, ctypes.c_double, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                             ctypes.c_int32], ctypes.c_int),
    "sdfgpu_autotune": ([ctypes.c_void_p, _dp, ctypes.c_double, _i64p, ctypes.c_int32,
                         ctypes.POINTER(ctypes.c_int32), _dp], ctypes.c_int),
    "sdfgpu_set_brick": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)], ctypes.c_int),
    "sdfgpu_set_radius_margin": ([ctypes.c_void_p, ctypes.c_float, ctypes.c_float], ctypes.c_int),
    "sdfgpu_remove_artifacts": ([ctypes.c_void_p, _i64p, _dp, ctypes.c_double, ctypes.c_double, _i64p, _i64p, _i64p],
                                ctypes.c_int),
    "sdfgpu_remove_artifacts_device": ([ctypes.c_void_p, _i64p, ctypes.c_void_p, ctypes.c_double, ctypes.c_double,
                                        _i64p, _i64p, _i64p], ctypes.c_int),
    "sdfgpu_rbf_smoothing": ([ctypes.c_void_p, _dp, _dp, _i64p, ctypes.c_double, _dp, ctypes.c_int32, ctypes.c_int32,
                              ctypes.c_double, ctypes.POINTER(ctypes.c_float), ctypes.POINTER(ctypes.c_float),
                              ctypes.POINTER(ctypes.c_int32), _dp], ctypes.c_int),
    "sdfgpu_sdf_components": ([ctypes.c_void_p, _i64p, _dp, ctypes.c_double, ctypes.POINTER(ctypes.c_int32), _i64p,
                               _i64p], ctypes.c_int),
    "sdfgpu_mesh_edge_stats": ([ctypes.c_void_p, _dp, _i64p], ctypes.c_int),
    "sdfgpu_stl_dedupe": ([ctypes.c_void_p, _dp, ctypes.c_int64, _dp, _i64p, _i64p, _i64p], ctypes.c_int),
    "sdfgpu_get_stream": ([ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)], ctypes.c_int),
    "sdfgpu_get_stats": ([ctypes.c_void_p, ctypes.POINTER(Stats)], ctypes.c_int),
}

_lib = None
_lock = threading.Lock()


def lib():
    """Load libsdfgpu.so (raises if it has not been built)."""
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise SdfGpuError(7, f"{LIB_PATH} is missing; build it with `make -C stl2sdf.jl_b200/csrc`")
            L = ctypes.CDLL(LIB_PATH)
            for name, (args, res) in SIGNATURES.items():
                fn = getattr(L, name)
                fn.argtypes = args
                fn.restype = res
            _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(_dp)


def _i(a):
    return a.ctypes.data_as(_i64p)


def grid_setup(xmin, xmax, n_max, margin=3):
    o = np.zeros(3); amax = np.zeros(3); N = np.zeros(3, np.int64); h = ctypes.c_double(); ngp = ctypes.c_int64()
    rc = lib().sdfgpu_grid_setup(_d(np.ascontiguousarray(xmin, np.float64)), _d(np.ascontiguousarray(xmax, np.float64)),
                                 int(n_max), int(margin), _d(o), _d(amax), _i(N), ctypes.byref(h), ctypes.byref(ngp))
    if rc:
        raise SdfGpuError(rc, "grid setup rejected its arguments (need finite bounds, positive extent, N_max >= 1)")
    return o, amax, N, h.value, ngp.value


def grid_from_cell_size(X, B):
    X = np.ascontiguousarray(X, np.float64).reshape(-1, 3)
    o = np.zeros(3); amax = np.zeros(3); N = np.zeros(3, np.int64); h = ctypes.c_double(); ngp = ctypes.c_int64()
    rc = lib().sdfgpu_grid_from_cell_size(_d(X), X.shape[0], float(B), _d(o), _d(amax), _i(N), ctypes.byref(h),
                                          ctypes.byref(ngp))
    if rc:
        raise SdfGpuError(rc, "grid setup rejected its arguments (cell size must be > 0 and below the mesh extent)")
    return o, amax, N, h.value, ngp.value


class Context:
    """One libsdfgpu context (one CUDA device, one stream, resident mesh)."""

    def __init__(self, device: int = 0, tile=(0, 0, 0)):
        L = lib()
        opts = Opts(device, (ctypes.c_int32 * 3)(*tile))
        p = ctypes.c_void_p()
        rc = L.sdfgpu_create(ctypes.byref(opts), ctypes.byref(p))
        if rc:
            raise SdfGpuError(rc, L.sdfgpu_last_error(None).decode())
        self._p = p
        self._mesh_key = None

    def _check(self, rc):
        if rc:
            raise SdfGpuError(rc, lib().sdfgpu_last_error(self._p).decode())

    def close(self):
        if self._p:
            lib().sdfgpu_destroy(self._p)
            self._p = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._p

    def stream_ptr(self) -> int:
        s = ctypes.c_void_p()
        self._check(lib().sdfgpu_get_stream(self._p, ctypes.byref(s)))
        return int(s.value or 0)

    def set_mesh(self, X, IEN, key=None):
        """X: (nnp, 3) float64; IEN: (nel, 3) int64 1-based (vertex-major = 3 x n column-major)."""
        if key is not None and key == self._mesh_key:
            return
        X = np.ascontiguousarray(X, np.float64).reshape(-1, 3)
        IEN = np.ascontiguousarray(IEN, np.int64).reshape(-1, 3)
        self._check(lib().sdfgpu_set_mesh(self._p, _d(X), X.shape[0], _i(IEN), IEN.shape[0]))
        self._mesh_key = key

    def set_mesh_device(self, x_ptr: int, nnp: int, ien_ptr: int, nel: int):
        self._check(lib().sdfgpu_set_mesh_device(self._p, ctypes.c_void_p(x_ptr), nnp, ctypes.c_void_p(ien_ptr), nel))
        self._mesh_key = None

    def distances(self, origin, h, N, mode=MODE_REF_RULE, want_xp=False, learned=False, out=None):
        N = np.ascontiguousarray(N, np.int64)
        origin = np.ascontiguousarray(origin, np.float64)
        ngp = int(np.prod(N + 1))
        dist = np.empty(ngp) if out is None else out
        xp = np.empty((ngp, 3)) if want_xp else None
        self._check(lib().sdfgpu_distances(self._p, _d(origin), float(h), _i(N), _d(dist),
                                           _d(xp) if xp is not None else None, int(mode), int(bool(learned))))
        return dist, xp

    def signs(self, origin, h, N, min_rays=6, max_rays=30, confidence_threshold=0.6, use_winding_fallback=True):
        N = np.ascontiguousarray(N, np.int64)
        origin = np.ascontiguousarray(origin, np.float64)
        ngp = int(np.prod(N + 1))
        sign = np.empty(ngp); conf = np.empty(ngp)
        self._check(lib().sdfgpu_signs(self._p, _d(origin), float(h), _i(N), int(min_rays), int(max_rays),
                                       float(confidence_threshold), int(bool(use_winding_fallback)), _d(sign), _d(conf)))
        return sign, conf

    def sdf(self, origin, h, N, mode=MODE_REF_RULE, min_rays=6, max_rays=30, confidence_threshold=0.6,
            use_winding_fallback=True, want_parts=False):
        """sdf, or with want_parts (True, or a subset of ("dist", "sign", "conf")) the tuple
        (sdf, dist, sign, conf) with None for the parts not asked for (they are not copied back)."""
        N = np.ascontiguousarray(N, np.int64)
        origin = np.ascontiguousarray(origin, np.float64)
        ngp = int(np.prod(N + 1))
        sdf = np.empty(ngp)
        names = ("dist", "sign", "conf")
        wanted = names if want_parts is True else (tuple(want_parts) if want_parts else ())
        parts = [np.empty(ngp) if n in wanted else None for n in names]
        self._check(lib().sdfgpu_sdf(self._p, _d(origin), float(h), _i(N), int(mode), int(min_rays), int(max_rays),
                                     float(confidence_threshold), int(bool(use_winding_fallback)), _d(sdf),
                                     *[(_d(p) if p is not None else None) for p in parts]))
        return (sdf, *parts) if want_parts else sdf

    def sdf_device(self, origin, h, N, sdf_ptr, mode=MODE_REF_RULE, min_rays=6, max_rays=30,
                   confidence_threshold=0.6, use_winding_fallback=True, dist_ptr=0, sign_ptr=0, conf_ptr=0):
        N = np.ascontiguousarray(N, np.int64)
        origin = np.ascontiguousarray(origin, np.float64)
        self._check(lib().sdfgpu_sdf_device(self._p, _d(origin), float(h), _i(N), int(mode), int(min_rays),
                                            int(max_rays), float(confidence_threshold),
                                            int(bool(use_winding_fallback)), ctypes.c_void_p(sdf_ptr),
                                            ctypes.c_void_p(dist_ptr or None), ctypes.c_void_p(sign_ptr or None),
                                            ctypes.c_void_p(conf_ptr or None)))

    def sdf_slab(self, origin, h, N, k0, k1, mode=MODE_REF_RULE, min_rays=6, max_rays=30, confidence_threshold=0.6,
                 use_winding_fallback=True, want_parts=False):
        """z layers k0..k1 of the grid (origin, h, N): an (N0+1)(N1+1)(k1-k0+1) block, x fastest."""
        N = np.ascontiguousarray(N, np.int64)
        origin = np.ascontiguousarray(origin, np.float64)
        n = int((N[0] + 1) * (N[1] + 1) * (int(k1) - int(k0) + 1))
        sdf = np.empty(max(n, 0))
        parts = [np.empty(max(n, 0)) for _ in range(3)] if want_parts else [None, None, None]
        self._check(lib().sdfgpu_sdf_slab(self._p, _d(origin), float(h), _i(N), int(k0), int(k1), int(mode),
                                          int(min_rays), int(max_rays), float(confidence_threshold),
                                          int(bool(use_winding_fallback)), _d(sdf),
                                          *[(_d(p) if p is not None else None) for p in parts]))
        return (sdf, *parts) if want_parts else sdf

    def sdf_slab_device(self, origin, h, N, k0, k1, sdf_ptr, mode=MODE_REF_RULE, min_rays=6, max_rays=30,
                        confidence_threshold=0.6, use_winding_fallback=True, dist_ptr=0, sign_ptr=0, conf_ptr=0):
        N = np.ascontiguousarray(N, np.int64)
        origin = np.ascontiguousarray(origin, np.float64)
        self._check(lib().sdfgpu_sdf_slab_device(self._p, _d(origin), float(h), _i(N), int(k0), int(k1), int(mode),
                                                 int(min_rays), int(max_rays), float(confidence_threshold),
                                                 int(bool(use_winding_fallback)), ctypes.c_void_p(sdf_ptr),
                                                 ctypes.c_void_p(dist_ptr or None), ctypes.c_void_p(sign_ptr or None),
                                                 ctypes.c_void_p(conf_ptr or None)))

    def sdf_batch(self, meshes, mode=MODE_REF_RULE, min_rays=6, max_rays=30, confidence_threshold=0.6,
                  use_winding_fallback=True, streams=8, autotune=True, want_parts=False, out=None, persistent=False):
        """SDFs of many meshes, each on its own grid: meshes = [(X, IEN, origin, h, N), ...].
        Returns one sdf array per mesh (with want_parts, (sdf, dist, sign, conf) per mesh).  `out`
        may supply the sdf arrays (contiguous float64, prod(N+1) each), e.g. views of page-locked
        host memory, which the copies then reach by DMA."""
        keep, outs = [], []
        items = (BatchItem * max(1, len(meshes)))()
        for k, (X, IEN, origin, h, N) in enumerate(meshes):
            X = np.ascontiguousarray(X, np.float64).reshape(-1, 3)
            IEN = np.ascontiguousarray(IEN, np.int64).reshape(-1, 3)
            N = np.ascontiguousarray(N, np.int64)
            ngp = int(np.prod(N + 1))
            if out is not None:
                o = out[k]
                if o.dtype != np.float64 or not o.flags.c_contiguous or o.size != ngp:
                    raise ValueError(f"out[{k}] must be a contiguous float64 array of {ngp} values")
                first = o
            else:
                first = np.empty(ngp)
            out_k = [first] + ([np.empty(ngp) for _ in range(3)] if want_parts else [None] * 3)
            keep += [X, IEN]
            outs.append(out_k)
            it = items[k]
            it.X, it.nnp, it.IEN, it.nel = _d(X), X.shape[0], _i(IEN), IEN.shape[0]
            it.origin[:] = [float(v) for v in origin]
            it.h = float(h)
            it.N[:] = [int(v) for v in N]
            it.sdf, it.dist, it.sign, it.conf = [(_d(a) if a is not None else None) for a in out_k]
        self._check(lib().sdfgpu_sdf_batch_ex(self._p, items, len(meshes), int(mode), int(min_rays), int(max_rays),
                                              float(confidence_threshold), int(bool(use_winding_fallback)),
                                              int(streams), int(bool(autotune)), int(bool(persistent))))
        return [tuple(o) if want_parts else o[0] for o in outs]

    def autotune(self, origin, h, N, mode=MODE_REF_RULE):
        """Picks the fastest tile for the current mesh on this grid; returns (tile, ms)."""
        N = np.ascontiguousarray(N, np.int64)
        origin = np.ascontiguousarray(origin, np.float64)
        tile = (ctypes.c_int32 * 3)()
        ms = ctypes.c_double(0.0)
        self._check(lib().sdfgpu_autotune(self._p, _d(origin), float(h), _i(N), int(mode), tile, ctypes.byref(ms)))
        return tuple(tile), ms.value

    def set_brick(self, brick):
        """Nodes (x, y, z; product 32) one warp searches together in the unbounded mode."""
        b = (ctypes.c_int32 * 3)(*[int(v) for v in brick])
        self._check(lib().sdfgpu_set_brick(self._p, b))

    # ---- learned search radius ----
    def set_radius_margin(self, alpha=0.5, beta=4.0):
        """r = (dhat (1 + alpha) + beta * coarse spacing / s) * s; alpha = inf: every radius infinite
        (the learned mode's search without the network's bound)."""
        self._check(lib().sdfgpu_set_radius_margin(self._p, float(alpha), float(beta)))

    def train_radius(self, coarse_n=24, steps=50, batch=2048, lr=5e-3, seed=0):
        loss = ctypes.c_float()
        self._check(lib().sdfgpu_train_radius(self._p, int(coarse_n), int(steps), int(batch), float(lr), int(seed),
                                              ctypes.byref(loss)))
        return loss.value

    def radius_params(self):
        n = lib().sdfgpu_radius_param_count()
        P = np.empty(n, np.float32); norm = np.empty(4)
        self._check(lib().sdfgpu_radius_params(self._p, P.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), _d(norm)))
        return P, norm

    def set_radius_params(self, P, norm):
        P = np.ascontiguousarray(P, np.float32); norm = np.ascontiguousarray(norm, np.float64)
        self._check(lib().sdfgpu_set_radius_params(self._p, P.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), _d(norm)))

    def radius_eval(self, xn):
        xn = np.ascontiguousarray(xn, np.float32).reshape(-1, 3)
        out = np.empty(xn.shape[0], np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        self._check(lib().sdfgpu_radius_eval(self._p, xn.ctypes.data_as(fp), xn.shape[0], out.ctypes.data_as(fp)))
        return out

    def mlp_train_eval(self, P, xn, target):
        fp = ctypes.POINTER(ctypes.c_float)
        P = np.ascontiguousarray(P, np.float32); xn = np.ascontiguousarray(xn, np.float32).reshape(-1, 3)
        t = np.ascontiguousarray(target, np.float32)
        dh = np.empty(xn.shape[0], np.float32); loss = np.empty(1, np.float32); grad = np.empty(P.shape[0], np.float32)
        self._check(lib().sdfgpu_mlp_train_eval(self._p, P.ctypes.data_as(fp), xn.ctypes.data_as(fp), t.ctypes.data_as(fp),
                                                xn.shape[0], dh.ctypes.data_as(fp), loss.ctypes.data_as(fp),
                                                grad.ctypes.data_as(fp)))
        return dh, float(loss[0]), grad

    # ---- artifact removal (SdfArtifactRemoval.jl) ----
    def remove_artifacts(self, N, sdf, threshold=0.0, min_component_ratio=0.01):
        """In place on the float64 array sdf; returns (flipped, components, largest)."""
        N = np.ascontiguousarray(N, np.int64)
        if sdf.dtype != np.float64 or not sdf.flags.c_contiguous or sdf.size != int(np.prod(N + 1)):
            raise ValueError("sdf must be a contiguous float64 array of prod(N+1) values")
        f, c, l = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        self._check(lib().sdfgpu_remove_artifacts(self._p, _i(N), sdf.ctypes.data_as(_dp), float(threshold),
                                                  float(min_component_ratio), ctypes.byref(f), ctypes.byref(c),
                                                  ctypes.byref(l)))
        return f.value, c.value, l.value

    def components(self, N, sdf, threshold=0.0):
        """Per node the smallest linear index of its interior component (-1 exterior), count, largest."""
        N = np.ascontiguousarray(N, np.int64)
        sdf = np.ascontiguousarray(sdf, np.float64)
        if sdf.size != int(np.prod(N + 1)):
            raise ValueError("sdf must hold prod(N+1) values")
        roots = np.empty(sdf.size, np.int32)
        c, l = ctypes.c_int64(), ctypes.c_int64()
        self._check(lib().sdfgpu_sdf_components(self._p, _i(N), sdf.ctypes.data_as(_dp), float(threshold),
                                                roots.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), ctypes.byref(c),
                                                ctypes.byref(l)))
        return roots, c.value, l.value

    # ---- mesh analysis (Grid_setup.jl:28-102) ----
    def mesh_edge_stats(self):
        """Edge-length statistics of the resident mesh: dict with shortest, longest, mean, median,
        smallest_mean / largest_mean (mean edge of the triangle with the smallest / largest edge sum)
        and smallest_index / largest_index (0-based)."""
        out = np.empty(6, np.float64)
        idx = np.empty(2, np.int64)
        self._check(lib().sdfgpu_mesh_edge_stats(self._p, out.ctypes.data_as(_dp), idx.ctypes.data_as(_i64p)))
        return {"shortest": float(out[0]), "longest": float(out[1]), "mean": float(out[2]), "median": float(out[3]),
                "smallest_mean": float(out[4]), "largest_mean": float(out[5]), "smallest_index": int(idx[0]),
                "largest_index": int(idx[1])}

    # ---- STL import (ImportStlData.jl:198-309) ----
    def stl_dedupe(self, stream):
        """Deduplicate the (3 nel, 3) stream of STL vertices: (X (nnp, 3), IEN (nel, 3) 1-based, number
        of ordered pairs of distinct vertices closer than 1e-10)."""
        S = np.ascontiguousarray(stream, np.float64).reshape(-1, 3)
        X = np.empty_like(S)
        IEN = np.empty(S.shape[0], np.int64)
        nnp, near = ctypes.c_int64(), ctypes.c_int64()
        self._check(lib().sdfgpu_stl_dedupe(self._p, S.ctypes.data_as(_dp), S.shape[0], X.ctypes.data_as(_dp),
                                            IEN.ctypes.data_as(_i64p), ctypes.byref(nnp), ctypes.byref(near)))
        return X[:nnp.value].copy(), IEN.reshape(-1, 3), near.value

    # ---- RBF smoothing (RBFs4Smoothing.jl) ----
    def rbf_smoothing(self, aabb_min, aabb_max, N, cell_size, dist, interpolation=True, smooth=2, threshold=1e-3,
                      want_weights=False):
        """Returns (fine Float32 values, x fastest; weights or None; CG iterations; final |r|)."""
        N = np.ascontiguousarray(N, np.int64)
        lo = np.ascontiguousarray(aabb_min, np.float64)
        hi = np.ascontiguousarray(aabb_max, np.float64)
        dist = np.ascontiguousarray(dist, np.float64)
        if dist.size != int(np.prod(N + 1)):
            raise ValueError("dist must hold prod(N+1) values")
        fine = np.empty(int(np.prod(N * int(smooth) + 1)), np.float32)
        w = np.empty(dist.size, np.float32) if want_weights else None
        fp = ctypes.POINTER(ctypes.c_float)
        it, res = ctypes.c_int32(), ctypes.c_double()
        self._check(lib().sdfgpu_rbf_smoothing(self._p, _d(lo), _d(hi), _i(N), float(cell_size), _d(dist),
                                               int(bool(interpolation)), int(smooth), float(threshold),
                                               fine.ctypes.data_as(fp), w.ctypes.data_as(fp) if w is not None else None,
                                               ctypes.byref(it), ctypes.byref(res)))
        return fine, w, it.value, res.value

    def stats(self) -> dict:
        s = Stats()
        self._check(lib().sdfgpu_get_stats(self._p, ctypes.byref(s)))
        return s.as_dict()


_default_ctx = {}


def default_context(device: int = 0) -> Context:
    ctx = _default_ctx.get(device)
    if ctx is None:
        ctx = Context(device)
        _default_ctx[device] = ctx
    return ctx
