"""Data formats either side of the hot path: STL import/dedupe (ImportStlData.jl), VTI export
(ExportToVTI.jl), the synthetic workload meshes and the Python mirror of MeshGrid."""

from __future__ import annotations

import os

import numpy as np
import pytest

import oracle
from conftest import GOLDEN


def test_reference_fixture_import():
    """The reference's own test input: 3,712 triangles, 1,890 unique vertices, closed (the reader
    and the oracle's deduplication; the GPU deduplication is checked against it in the gpu tests)."""
    from oracle import stl_dedupe
    from stl2sdf import DataImport
    from workloads import synthetic

    V, T = DataImport.read_binary_stl(os.path.join(GOLDEN, "artifacts.stl"))
    X, IEN = stl_dedupe.exact(V, T)
    assert stl_dedupe.near_pairs(X) == 0
    assert IEN.shape == (3712, 3) and X.shape == (1890, 3)
    assert synthetic.is_closed(IEN)
    assert IEN.min() == 1 and IEN.max() == X.shape[0]


def test_binary_roundtrip_and_first_appearance_order(tmp_path):
    from oracle import stl_dedupe
    from stl2sdf import DataImport
    from workloads import synthetic

    V, F = synthetic.icosphere(2, jitter=0.01, seed=3)
    path = str(tmp_path / "s.stl")
    DataImport.write_binary_stl(path, V, F)
    X, IEN = stl_dedupe.exact(*DataImport.read_binary_stl(path))
    X2, IEN2 = DataImport.roundtrip_float32(V, F)
    assert np.array_equal(X, X2) and np.array_equal(IEN, IEN2)
    # vertices appear in the order the triangle stream first mentions them
    first = np.unique(IEN.reshape(-1), return_index=True)[1]
    assert np.all(np.diff(first) > 0)
    assert np.array_equal(X, V[F.reshape(-1)[np.sort(np.unique(F.reshape(-1), return_index=True)[1])] - 1]
                          .astype(np.float32).astype(np.float64))


def test_ascii_reader(tmp_path):
    from stl2sdf import DataImport

    path = str(tmp_path / "a.stl")
    with open(path, "w") as f:
        f.write("solid t\n facet normal 0 0 1\n  outer loop\n   vertex 0 0 0\n   vertex 1 0 0\n   vertex 0 1 0\n"
                "  endloop\n endfacet\n facet normal 0 0 1\n  outer loop\n   vertex 1 0 0\n   vertex 1 1 0\n"
                "   vertex 0 1 0\n  endloop\n endfacet\nendsolid t\n")
    from oracle import stl_dedupe

    assert DataImport.detect_stl_type(path)
    X, IEN = stl_dedupe.exact(*DataImport.read_ascii_stl(path))
    assert X.shape == (4, 3) and IEN.tolist() == [[1, 2, 3], [2, 4, 3]]


def test_dedupe_tolerance_restatements():
    """The reference's walk merges a vertex 1e-11 from the origin into it; exact deduplication does
    not, and the near-pair count tells the two cases apart.  The product's host walk for that case
    agrees with the oracle's."""
    from oracle import stl_dedupe
    from stl2sdf import DataImport

    V = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [1e-11, 0, 0], [1, 1, 0], [0, 1, 0]], dtype=np.float64)
    T = np.array([[1, 2, 3], [4, 5, 6]])
    Xs, IENs = stl_dedupe.sequential(V, T)
    assert Xs.shape[0] == 4 and IENs.tolist() == [[1, 2, 3], [1, 4, 3]]  # 1e-11 merged into the origin
    Xe, IENe = stl_dedupe.exact(V, T)
    assert Xe.shape[0] == 5 and stl_dedupe.near_pairs(Xe) == 2
    Xp, IENp = DataImport._dedupe_sequential(V, T)
    assert np.array_equal(Xp, Xs) and np.array_equal(IENp, IENs)
    # without near pairs the walk is exact deduplication
    V2 = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [-0.0, 0, 0], [1, 1, 0], [0, 1, 0]], dtype=np.float64)
    a, b = stl_dedupe.sequential(V2, T), stl_dedupe.exact(V2, T)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[1].tolist() == [[1, 2, 3], [1, 4, 3]]


def test_vti_roundtrip(tmp_path):
    from stl2sdf import DataExport, MeshGrid

    g = MeshGrid.Grid([0.0, 0.0, 0.0], [1.0, 0.5, 0.25], 8, 3)
    vals = np.random.default_rng(0).normal(size=g.ngp)
    for comp in (True, False):
        path = DataExport.exportSdfToVTI(str(tmp_path / f"x{comp}_sdf"), g, vals, "distance", compress=comp)
        assert path.endswith(".vti")
        v, dims, o, sp, label = DataExport.read_vti(path)
        assert np.array_equal(v, vals) and dims.tolist() == (g.N + 1).tolist()
        assert np.array_equal(o, g.AABB_min) and sp.tolist() == [g.cell_size] * 3 and label == "distance"
    with pytest.raises(ValueError):
        DataExport.exportSdfToVTI(str(tmp_path / "bad"), g, vals[:-1], "distance")


def _decode_vti_from_spec(path):
    """A decoder written from the VTK XML file-format description, independent of DataExport:
    the XML header is parsed as XML (the raw appended block cut out), and the appended data is
    decoded by its rules -- an '_' marker, then at the array's offset either a UInt64 byte count and
    the raw bytes, or (vtkZLibDataCompressor) a UInt64 header [number of blocks, uncompressed block
    size, uncompressed size of the last block (0: a full block), compressed size of each block]
    followed by the zlib streams."""
    import struct
    import xml.etree.ElementTree as ET
    import zlib

    data = open(path, "rb").read()
    a = data.index(b"<AppendedData")
    marker = data.index(b"_", a) + 1
    end = data.rindex(b"</AppendedData>")
    root = ET.fromstring(data[:marker - 1] + data[end:])
    assert root.tag == "VTKFile" and root.get("type") == "ImageData"
    assert root.get("byte_order") == "LittleEndian" and root.get("header_type") == "UInt64"
    img = root.find("ImageData")
    ext = [int(v) for v in img.get("WholeExtent").split()]
    assert img.find("Piece").get("Extent") == img.get("WholeExtent")
    arr = img.find("Piece").find("PointData").find("DataArray")
    assert arr.get("format") == "appended" and root.find("AppendedData").get("encoding") == "raw"
    size = {"Float64": 8, "Float32": 4}[arr.get("type")]
    blob = data[marker + int(arr.get("offset")):]
    if root.get("compressor") == "vtkZLibDataCompressor":
        nb, bs, last = struct.unpack("<3Q", blob[:24])
        csz = struct.unpack(f"<{nb}Q", blob[24:24 + 8 * nb])
        pos, raw = 24 + 8 * nb, b""
        for q in range(nb):
            part = zlib.decompress(blob[pos:pos + csz[q]])
            want = (last if last else bs) if q == nb - 1 else bs
            assert len(part) == want
            raw += part
            pos += csz[q]
    else:
        assert root.get("compressor") is None
        (n,) = struct.unpack("<Q", blob[:8])
        raw = blob[8:8 + n]
    dims = [ext[1] - ext[0] + 1, ext[3] - ext[2] + 1, ext[5] - ext[4] + 1]
    assert len(raw) == size * dims[0] * dims[1] * dims[2]
    vals = np.frombuffer(raw, dtype="<f8" if size == 8 else "<f4")
    return (vals, dims, [float(v) for v in img.get("Origin").split()], [float(v) for v in img.get("Spacing").split()],
            arr.get("Name"), img.get("Direction"))


def test_vti_layout_by_an_independent_decoder(tmp_path):
    """The writer's files decoded by the spec-based decoder above: uncompressed, one zlib block,
    several zlib blocks (a field over 4 MiB), Float64 and the Float32 smoothed field, values x
    fastest (ExportToVTI.jl:55-64 reshapes the field to N+1 per axis, x first)."""
    from stl2sdf import DataExport, MeshGrid

    rng = np.random.default_rng(4)
    for hi, n_max, comp, smooth in (((1.0, 0.5, 2.25), 8, False, None), ((1.0, 0.5, 2.25), 8, True, None),
                                    ((1.0, 2.0, 4.0), 74, True, None), ((1.0, 0.5, 2.25), 8, True, 2)):
        g = MeshGrid.Grid([-1.0, 0.0, 2.0], list(hi), n_max, 3)
        dims = (g.N + 1) if smooth is None else g.N * smooth + 1
        n = int(np.prod(dims))
        vals = rng.normal(size=n).astype(np.float32 if smooth else np.float64)
        path = DataExport.exportSdfToVTI(str(tmp_path / f"f{n_max}{comp}{smooth}"), g, vals, "distance",
                                         smooth=smooth, compress=comp)
        got, gdims, origin, spacing, label, direction = _decode_vti_from_spec(path)
        assert np.array_equal(got, vals) and gdims == [int(v) for v in dims]
        assert origin == [float(v) for v in g.AABB_min]
        h = g.cell_size / (smooth or 1)
        assert spacing == [h, h, h] and label == "distance" and direction == "1 0 0 0 1 0 0 0 1"
        # x fastest: the value at (i, j, k) sits at i + nx (j + ny k)
        i, j, k = dims[0] - 1, 1, 1
        assert got[i + dims[0] * (j + dims[1] * k)] == vals.reshape(dims[2], dims[1], dims[0])[k, j, i]
        if n_max == 74:  # this field spans more than one 4 MiB zlib block
            assert 8 * n > (1 << 22)


def test_workload_meshes():
    from workloads import synthetic

    V, F = synthetic.icosphere(4)
    assert V.shape == (2562, 3) and F.shape == (5120, 3) and synthetic.is_closed(F)
    V, F = synthetic.torus()
    assert V.shape == (65536, 3) and F.shape == (131072, 3) and synthetic.is_closed(F)
    V, F = synthetic.box()
    assert F.shape == (12, 3) and synthetic.is_closed(F)


def test_grid_points_match_oracle_nodes(icosphere_mesh):
    from stl2sdf import MeshGrid

    X, IEN = icosphere_mesh
    mesh = MeshGrid.TriangularMesh(X, IEN)
    g = MeshGrid.noninteractive_sdf_grid_setup(mesh, 0.05, analyze=False)  # the analysis needs the GPU
    P = MeshGrid.generateGridPoints(g)
    assert P.shape == (3, g.ngp)
    n = g.N + 1
    for lin in (0, 1, n[0], n[0] * n[1] + 5, g.ngp - 1):
        i, j, k = lin % n[0], (lin // n[0]) % n[1], lin // (n[0] * n[1])
        assert P[:, lin].tolist() == [g.AABB_min[0] + g.cell_size * i, g.AABB_min[1] + g.cell_size * j,
                                      g.AABB_min[2] + g.cell_size * k]
    xmin, xmax = MeshGrid.getMesh_AABB(mesh.X)
    assert np.array_equal(xmin, X.min(0)) and np.array_equal(xmax, X.max(0))
    assert len(mesh.INE) == mesh.nnp and sum(len(v) for v in mesh.INE) == 3 * mesh.nel


def _two_blobs():
    N = np.array([19, 19, 19])
    n = N + 1
    sdf = -np.ones(int(np.prod(n)))
    vol = sdf.reshape(n[2], n[1], n[0])
    vol[2:12, 2:12, 2:12] = 1.0   # large interior component (1000 nodes)
    vol[15:17, 15:17, 15:16] = 1.0  # small one (4 nodes)
    return N, sdf


def test_artifact_removal_oracle_known_answer():
    from oracle import artifacts

    N, sdf = _two_blobs()
    out, flipped, comps, largest = artifacts.remove_sdf_artifacts(sdf, N, min_component_ratio=0.01)
    assert (flipped, comps, largest) == (4, 2, 1000)
    assert np.count_nonzero(out > 0) == 1000 and np.count_nonzero(sdf > 0) == 1004
    # ratio 0.004 -> min size round(4.0) = 4: the 4-node component stays
    _, flipped, _, _ = artifacts.remove_sdf_artifacts(sdf, N, min_component_ratio=0.004)
    assert flipped == 0
    # round half to even, as Julia's round(Int, x): 0.0045 * 1000 = 4.5 -> 4, the 4-node component stays
    _, flipped, _, _ = artifacts.remove_sdf_artifacts(sdf, N, min_component_ratio=0.0045)
    assert flipped == 0
    _, flipped, _, _ = artifacts.remove_sdf_artifacts(sdf, N, min_component_ratio=0.0055)
    assert flipped == 4


def test_artifact_labelling_matches_union_find():
    from oracle import artifacts

    rng = np.random.default_rng(5)
    for shape in ([6, 5, 4], [9, 1, 7], [0, 0, 0], [3, 3, 3]):
        n = np.asarray(shape) + 1
        mask = rng.random(int(np.prod(n))) < 0.45
        assert np.array_equal(artifacts.labels(mask, n), artifacts.union_find_labels(mask, n))


def test_malformed_stl_is_reported(tmp_path):
    from stl2sdf import DataImport
    from workloads import synthetic

    V, F = synthetic.icosphere(1)
    good = tmp_path / "good.stl"
    DataImport.write_binary_stl(str(good), V, F)
    data = good.read_bytes()
    short = tmp_path / "short.stl"
    short.write_bytes(data[:84 + 50 * 3 + 7])
    with pytest.raises(ValueError, match="truncated binary STL"):
        DataImport.import_stl(str(short))
    tiny = tmp_path / "tiny.stl"
    tiny.write_bytes(b"\x00" * 40)
    with pytest.raises(ValueError, match="84-byte header"):
        DataImport.import_stl(str(tiny))
    nan = tmp_path / "nan.stl"
    arr = bytearray(data)
    arr[84 + 12:84 + 16] = np.float32(np.nan).tobytes()
    nan.write_bytes(bytes(arr))
    with pytest.raises(ValueError, match="finite"):
        DataImport.import_stl(str(nan))


def test_options_validation():
    import stl2sdf

    with pytest.raises(AssertionError):
        stl2sdf.stl_to_sdf("x.stl", stl2sdf.Options(grid_refinement=3))
    with pytest.raises(AssertionError):
        stl2sdf.stl_to_sdf("x.stl", stl2sdf.Options(artifact_ratio=1.5))
