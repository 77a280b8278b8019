"""Mesh and grid containers, mirroring ``stl2sdf.MeshGrid`` (src/MeshGrid/).

* :class:`TriangularMesh` -- MeshInformations.jl:57-84.  ``X`` is exposed as the reference's
  3 x nnp matrix and ``IEN`` as 3 x nel (1-based); both are views of vertex-major row arrays,
  which is also the memory layout of the Julia column-major matrices passed through the C ABI.
* :class:`Grid` -- Grid.jl:9-32, computed by ``sdfgpu_grid_setup`` (the same host arithmetic the
  C ABI uses, so the Python object and the library always agree on the grid).
* :func:`generateGridPoints` -- Grid.jl:82-96: node = AABB_min + cell_size * [i, j, k], x fastest.
* :func:`noninteractive_sdf_grid_setup` / :func:`interactive_sdf_grid_setup` -- Grid_setup.jl,
  including the mesh analysis they print first (:func:`mesh_edge_statistics`, computed on the GPU
  by ``sdfgpu_mesh_edge_stats``).
"""

from __future__ import annotations

import numpy as np

from . import _native


class TriangularMesh:
    """TriangularMesh(X, IEN): X vertices (nnp x 3 rows or 3 x nnp), IEN triangles 1-based."""

    def __init__(self, X, IEN):
        X = np.asarray(X, dtype=np.float64)
        IEN = np.asarray(IEN, dtype=np.int64)
        if X.ndim != 2 or IEN.ndim != 2:
            raise ValueError("X and IEN must be 2-D")
        if X.shape[1] != 3 and X.shape[0] == 3:
            X = X.T
        if IEN.shape[1] != 3 and IEN.shape[0] == 3:
            IEN = IEN.T
        self._Xrows = np.ascontiguousarray(X)
        self._IENrows = np.ascontiguousarray(IEN)
        self.nsd = 3
        self.nnp = self._Xrows.shape[0]
        self.nen = 3
        self.nel = self._IENrows.shape[0]
        self._INE = None
        self._key = (id(self), self.nnp, self.nel)

    @property
    def X(self):
        """3 x nnp view (the reference's layout)."""
        return self._Xrows.T

    @property
    def IEN(self):
        """3 x nel view, 1-based."""
        return self._IENrows.T

    @property
    def INE(self):
        """Node-to-element lists (MeshInformations.jl:39-54), 1-based element ids."""
        if self._INE is None:
            INE = [[] for _ in range(self.nnp)]
            for el in range(self.nel):
                for k in range(3):
                    INE[self._IENrows[el, k] - 1].append(el + 1)
            self._INE = INE
        return self._INE

    def vertex_rows(self):
        return self._Xrows

    def triangle_rows(self):
        return self._IENrows


def nodeToElementConnectivity(X, IEN):
    return TriangularMesh(X, IEN).INE


class Grid:
    """Grid(AABB_min, AABB_max, N_max, margineCells=3) (Grid.jl:9-32)."""

    def __init__(self, AABB_min, AABB_max, N_max: int, margineCells: int = 3):
        o, amax, N, h, ngp = _native.grid_setup(AABB_min, AABB_max, int(N_max), int(margineCells))
        self.AABB_min = o
        self.AABB_max = amax
        self.N = N
        self.cell_size = h
        self.ngp = ngp

    @classmethod
    def from_parts(cls, AABB_min, N, cell_size):
        g = cls.__new__(cls)
        g.AABB_min = np.asarray(AABB_min, dtype=np.float64).copy()
        g.N = np.asarray(N, dtype=np.int64).copy()
        g.cell_size = float(cell_size)
        g.AABB_max = g.AABB_min + g.N.astype(np.float64) * g.cell_size
        g.ngp = int(np.prod(g.N + 1))
        return g

    def __eq__(self, other):
        return (isinstance(other, Grid) and np.array_equal(self.AABB_min, other.AABB_min)
                and np.array_equal(self.N, other.N) and self.cell_size == other.cell_size)

    def __repr__(self):
        return f"Grid(AABB_min={self.AABB_min.tolist()}, N={self.N.tolist()}, cell_size={self.cell_size!r}, ngp={self.ngp})"


def getMesh_AABB(X):
    """(X_min, X_max) of a 3 x nnp vertex matrix (Grid.jl:74-78)."""
    X = np.asarray(X)
    if X.shape[0] != 3 and X.shape[1] == 3:
        X = X.T
    return X.min(axis=1), X.max(axis=1)


class GridPoints(np.ndarray):
    """3 x ngp node matrix that remembers the grid it was generated from."""

    grid = None

    def __array_finalize__(self, obj):
        self.grid = getattr(obj, "grid", None)


def generateGridPoints(grid: Grid) -> GridPoints:
    """Grid.jl:82-96: node a = AABB_min + cell_size * [i, j, k], x fastest, as a 3 x ngp matrix."""
    n = grid.N + 1
    h = grid.cell_size
    o = grid.AABB_min
    x = o[0] + h * np.arange(n[0], dtype=np.float64)
    y = o[1] + h * np.arange(n[1], dtype=np.float64)
    z = o[2] + h * np.arange(n[2], dtype=np.float64)
    P = np.empty((grid.ngp, 3))
    P[:, 0] = np.tile(x, n[1] * n[2])
    P[:, 1] = np.tile(np.repeat(y, n[0]), n[2])
    P[:, 2] = np.repeat(z, n[0] * n[1])
    out = P.T.view(GridPoints)
    out.grid = grid
    return out


_RED, _BOLD, _RESET = "\x1b[31m", "\x1b[1m", "\x1b[0m"


def mesh_edge_statistics(mesh: TriangularMesh, device: int = 0) -> dict:
    """Edge-length statistics of the mesh (calculate_edge_distances + analyze_mesh,
    Grid_setup.jl:28-102), computed on the GPU: shortest, longest, mean and median edge, and the mean
    edge of the triangles with the smallest / largest edge sum (smallest_index / largest_index,
    0-based, the first on ties).  Uploads the mesh to the device's default context, where the
    distance and sign calls that follow find it."""
    ctx = _native.default_context(device)
    ctx.set_mesh(mesh.vertex_rows(), mesh.triangle_rows(), key=mesh._key)
    return ctx.mesh_edge_stats()


def analyze_mesh(mesh: TriangularMesh, device: int = 0) -> dict:
    """Prints the mesh analysis of Grid_setup.jl:64-102 and returns its statistics."""
    st = mesh_edge_statistics(mesh, device)
    print("Mesh Statistics:")
    print("----------------")
    print(f"Number of elements: {mesh.nel}")
    print(f"Shortest edge in the mesh: {_RED}{_BOLD}{round(st['shortest'], 4)}{_RESET}")
    print(f"Longest edge in the mesh: {round(st['longest'], 4)}")
    print(f"Average edge length: {round(st['mean'], 4)}")
    print(f"Median edge length: {round(st['median'], 4)}")
    print(f"Average edge length of the smallest element: {_RED}{_BOLD}{round(st['smallest_mean'], 4)}{_RESET}")
    print(f"Average edge length of the largest element: {round(st['largest_mean'], 4)}")
    return st


def noninteractive_sdf_grid_setup(mesh: TriangularMesh, B: float, analyze: bool = True) -> Grid:
    """Grid_setup.jl:104-124: N_new = floor(max extent / B), 3 padding cells.

    analyze: print the mesh analysis first, as the reference does (needs the GPU)."""
    if analyze:
        analyze_mesh(mesh)
    o, amax, N, h, ngp = _native.grid_from_cell_size(mesh.vertex_rows(), float(B))
    g = Grid.from_parts(o, N, h)
    g.AABB_max = amax
    print(f"Number of all grid points: {g.ngp}")
    return g


def interactive_sdf_grid_setup(mesh: TriangularMesh, analyze: bool = True) -> Grid:
    """Grid_setup.jl:126-173: prints the mesh analysis (analyze=True, needs the GPU), then prompts for
    the cell size on stdin until the user accepts."""
    if analyze:
        analyze_mesh(mesh)
    while True:
        while True:
            try:
                B = float(input("Write a grid step based on grid analysis: "))
                g = noninteractive_sdf_grid_setup(mesh, B, analyze=False)
                break
            except ValueError:
                print("Error: Please enter a valid floating-point number.")
        if input("Do you want to continue? (y/n): ").strip().lower() == "y":
            return g
        print("You can write a grid step.")
