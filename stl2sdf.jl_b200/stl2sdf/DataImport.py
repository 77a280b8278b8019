"""STL import, mirroring ``stl2sdf.DataImport`` (src/DataImport/ImportStlData.jl).

``import_stl(filename) -> (X, IEN)`` returns the deduplicated vertices as an ``(nnp, 3)`` float64
array and the triangles as an ``(nel, 3)`` int64 array of 1-based indices (the reference returns
``Vector{Vector{Float64}}`` / ``Vector{Vector{Int}}``; rows here are those vectors).

* Binary STL vertices are float32 widened to float64 (ImportStlData.jl:127-161).
* ASCII STL vertices are parsed as float64 (ImportStlData.jl:163-196).
* ASCII vs binary: the file starts with ``solid`` (ImportStlData.jl:118-125).
* Deduplication follows ``process_stl_mesh`` (ImportStlData.jl:198-309): vertices are visited in
  stream order and merged into the first earlier unique vertex within ``norm < 1e-10`` found in
  the vertex's hash cell ``floor(v * 1e10)`` or, failing that, in one of its 26 neighbour cells
  (dx outermost, then dy, then dz).  The unique vertices keep their first-appearance order.
  When no two distinct vertices lie within 1e-10 of each other (always the case for meshes
  whose coordinates are separated by more than that), the result equals exact deduplication in
  first-appearance order, which runs on the GPU (``sdfgpu_stl_dedupe``: radix sorts, a scan and
  the reference's hash cells to detect distinct vertices closer than 1e-10).  Only when such
  vertices exist does the reference's order-dependent merge apply; it is then walked on the host
  (:func:`_dedupe_sequential`).
"""

from __future__ import annotations

import numpy as np

_STL_DTYPE = np.dtype([("n", "<f4", (3,)), ("v", "<f4", (3, 3)), ("attr", "<u2")])


def detect_stl_type(filename: str) -> bool:
    """True for ASCII (the first 5 bytes are ``solid``), as ImportStlData.jl:118-125."""
    with open(filename, "rb") as f:
        return f.read(5) == b"solid"


def read_binary_stl(filename: str):
    """Raw (non-deduplicated) float64 vertices, 3 per triangle, and 1-based triangles."""
    with open(filename, "rb") as f:
        head = f.read(84)
        if len(head) < 84:
            raise ValueError(f"{filename}: not a binary STL (shorter than its 84-byte header)")
        n = int(np.frombuffer(head[80:84], dtype="<u4")[0])
        body = f.read(n * 50)
    if len(body) < n * 50:
        # the reference's read loop hits end-of-file here (ImportStlData.jl:136-156)
        raise ValueError(f"{filename}: truncated binary STL: the header announces {n} triangles, "
                         f"the file holds {len(body) // 50}")
    rec = np.frombuffer(body, dtype=_STL_DTYPE, count=n)
    V = rec["v"].reshape(-1, 3).astype(np.float64)
    T = np.arange(1, 3 * n + 1, dtype=np.int64).reshape(n, 3)
    return V, T


def read_ascii_stl(filename: str):
    verts = []
    with open(filename, "r") as f:
        for line in f:
            s = line.strip()
            if s.startswith("vertex"):
                parts = s.split()
                if len(parts) >= 4:
                    verts.append((float(parts[1]), float(parts[2]), float(parts[3])))
    ntri = len(verts) // 3
    V = np.asarray(verts, dtype=np.float64).reshape(-1, 3)
    T = np.arange(1, 3 * ntri + 1, dtype=np.int64).reshape(ntri, 3)
    return V, T


def _dedupe_sequential(V: np.ndarray, T: np.ndarray):
    """process_stl_mesh (ImportStlData.jl:198-309) walked vertex by vertex, for the meshes whose
    distinct vertices come closer than 1e-10 (the GPU detects them), where the merge depends on the
    stream order."""
    tol = 1e-10
    sf = 10000000000  # floor(Int, 1/tol)
    vmap: dict = {}
    uniq: list = []
    newT = np.empty_like(T)
    for ti in range(T.shape[0]):
        for c in range(3):
            v = V[T[ti, c] - 1]
            key = (int(np.floor(v[0] * sf)), int(np.floor(v[1] * sf)), int(np.floor(v[2] * sf)))
            found = 0
            for idx in vmap.get(key, ()):
                if np.linalg.norm(v - uniq[idx - 1]) < tol:
                    found = idx
                    break
            if not found:
                pos = (v[0] * sf - np.floor(v[0] * sf), v[1] * sf - np.floor(v[1] * sf), v[2] * sf - np.floor(v[2] * sf))
                lim = tol * sf
                for dx in (-1, 0, 1):
                    for dy in (-1, 0, 1):
                        for dz in (-1, 0, 1):
                            if found or (dx == 0 and dy == 0 and dz == 0):
                                continue
                            if ((dx == -1 and pos[0] < lim) or (dx == 1 and pos[0] > 1 - lim) or
                                    (dy == -1 and pos[1] < lim) or (dy == 1 and pos[1] > 1 - lim) or
                                    (dz == -1 and pos[2] < lim) or (dz == 1 and pos[2] > 1 - lim)):
                                for idx in vmap.get((key[0] + dx, key[1] + dy, key[2] + dz), ()):
                                    if np.linalg.norm(v - uniq[idx - 1]) < tol:
                                        found = idx
                                        break
            if not found:
                uniq.append(v.copy())
                found = len(uniq)
                vmap.setdefault(key, []).append(found)
            newT[ti, c] = found
    return np.asarray(uniq, dtype=np.float64).reshape(-1, 3), newT


def process_stl_mesh(V: np.ndarray, T: np.ndarray, device: int = 0):
    """Deduplicate vertices (ImportStlData.jl:198-309) on the GPU.  Returns (X, IEN), IEN 1-based."""
    from . import _native

    V = np.ascontiguousarray(V, dtype=np.float64).reshape(-1, 3)
    T = np.ascontiguousarray(T, dtype=np.int64).reshape(-1, 3)
    if not np.all(np.isfinite(V)):
        raise ValueError("STL vertices must be finite")
    if T.shape[0] == 0:
        return np.zeros((0, 3)), np.zeros((0, 3), dtype=np.int64)
    X, IEN, near = _native.default_context(device).stl_dedupe(V[T.reshape(-1) - 1])
    if near:
        return _dedupe_sequential(V, T)
    return X, IEN


def import_stl(filename: str):
    """Import an STL file: (X, IEN) with X (nnp, 3) float64 and IEN (nel, 3) int64 1-based."""
    V, T = read_ascii_stl(filename) if detect_stl_type(filename) else read_binary_stl(filename)
    return process_stl_mesh(V, T)


def write_binary_stl(filename: str, X: np.ndarray, IEN: np.ndarray, header: bytes = b"stl2sdf.jl_b200 synthetic mesh"):
    """Write a binary STL (float32 vertices, per-face normals)."""
    X = np.asarray(X, dtype=np.float64).reshape(-1, 3)
    F = np.asarray(IEN, dtype=np.int64).reshape(-1, 3) - 1
    a, b, c = X[F[:, 0]], X[F[:, 1]], X[F[:, 2]]
    n = np.cross(b - a, c - a)
    ln = np.linalg.norm(n, axis=1, keepdims=True)
    n = np.divide(n, ln, out=np.zeros_like(n), where=ln > 0)
    rec = np.zeros(F.shape[0], dtype=_STL_DTYPE)
    rec["n"] = n.astype(np.float32)
    rec["v"] = np.stack([a, b, c], axis=1).astype(np.float32)
    hdr = header[:80].ljust(80, b" ")
    if hdr.startswith(b"solid"):
        raise ValueError("a binary STL header must not start with 'solid'")
    with open(filename, "wb") as f:
        f.write(hdr)
        f.write(np.uint32(F.shape[0]).tobytes())
        f.write(rec.tobytes())


def roundtrip_float32(X: np.ndarray, IEN: np.ndarray):
    """(X, IEN) as import_stl returns it after write_binary_stl, without touching disk: the vertices
    rounded to float32 and renumbered in order of first appearance in the triangle stream (unused
    ones dropped).  For building workload meshes from generated ones, whose distinct vertices stay
    distinct and farther apart than 1e-10 after the rounding (checked: an error otherwise)."""
    X = np.asarray(X, dtype=np.float64).reshape(-1, 3)
    F = np.asarray(IEN, dtype=np.int64).reshape(-1, 3) - 1
    ids, first = np.unique(F.reshape(-1), return_index=True)
    used = ids[np.argsort(first, kind="stable")]  # original ids in first-appearance order
    new = np.empty(X.shape[0], np.int64)
    new[used] = np.arange(1, used.shape[0] + 1)
    X32 = X[used].astype(np.float32).astype(np.float64)
    if X32.shape[0] > 1:
        from scipy.spatial import cKDTree

        if cKDTree(X32).query_pairs(r=1e-10, output_type="ndarray").shape[0] > 0:
            raise ValueError("mesh vertices coincide (within 1e-10) after rounding to float32")
    return X32, new[F]
