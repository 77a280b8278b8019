"""VTK ImageData export, mirroring ``exportSdfToVTI`` (src/DataExport/ExportToVTI.jl:22-67).

The file holds one point field (``value_label``) over an ImageData with extent 0..N per axis,
origin ``grid.AABB_min`` and spacing ``cell_size`` (``cell_size/smooth`` with ``N*smooth`` cells
when ``smooth`` is given), values in the grid's x-fastest order.  The layout is the one WriteVTK
writes for ``vtk_grid(filename, x, y, z)``: appended raw binary, UInt64 block headers, and (by
default, like WriteVTK) a single zlib-compressed block.
"""

from __future__ import annotations

import os
import re
import zlib

import numpy as np


def _vti_name(filename: str) -> str:
    return filename if filename.endswith(".vti") else filename + ".vti"


def exportSdfToVTI(filename: str, grid, values, value_label: str, smooth=None, compress: bool = True) -> str:
    """Write values on grid to a .vti file; returns the path written."""
    N = np.asarray(grid.N, dtype=np.int64)
    dims = N + 1 if smooth is None else N * int(smooth) + 1
    h = grid.cell_size if smooth is None else grid.cell_size / int(smooth)
    # WriteVTK writes the array's own element type: Float32 for the smoothed field, else Float64
    vt = np.float32 if np.asarray(values).dtype == np.float32 else np.float64
    values = np.ascontiguousarray(values, dtype=vt).reshape(-1)
    if values.shape[0] != int(np.prod(dims)):
        raise ValueError(f"Values vector length ({values.shape[0]}) doesn't match grid dimensions ({int(np.prod(dims))}).")
    o = [float(v) for v in np.asarray(grid.AABB_min, dtype=np.float64)]
    h = float(h)
    ext = f"0 {dims[0] - 1} 0 {dims[1] - 1} 0 {dims[2] - 1}"
    raw = values.astype("<f4" if vt == np.float32 else "<f8").tobytes()
    if compress:
        comp = zlib.compress(raw, 6)
        payload = np.array([1, len(raw), len(raw), len(comp)], dtype="<u8").tobytes() + comp
        comp_attr = ' compressor="vtkZLibDataCompressor"'
    else:
        payload = np.array([len(raw)], dtype="<u8").tobytes() + raw
        comp_attr = ""
    head = (
        '<?xml version="1.0" encoding="utf-8"?>\n'
        f'<VTKFile type="ImageData" version="1.0" byte_order="LittleEndian" header_type="UInt64"{comp_attr}>\n'
        f'  <ImageData WholeExtent="{ext}" Origin="{o[0]!r} {o[1]!r} {o[2]!r}" Spacing="{h!r} {h!r} {h!r}" '
        'Direction="1 0 0 0 1 0 0 0 1">\n'
        f'    <Piece Extent="{ext}">\n'
        "      <PointData>\n"
        f'        <DataArray type="{"Float32" if vt == np.float32 else "Float64"}" Name="{value_label}" format="appended" offset="0"/>\n'
        "      </PointData>\n"
        "    </Piece>\n"
        "  </ImageData>\n"
        '  <AppendedData encoding="raw">\n_'
    )
    path = _vti_name(filename)
    with open(path, "wb") as f:
        f.write(head.encode())
        f.write(payload)
        f.write(b"\n  </AppendedData>\n</VTKFile>\n")
    return path


def read_vti(path: str):
    """Read back a file written by :func:`exportSdfToVTI`: (values, dims, origin, spacing, label)."""
    with open(path, "rb") as f:
        data = f.read()
    start = data.index(b'<AppendedData encoding="raw">')
    body = data[start:]
    us = body.index(b"_") + 1
    head = data[:start].decode()
    m = re.search(r'WholeExtent="0 (\d+) 0 (\d+) 0 (\d+)" Origin="([^"]+)" Spacing="([^"]+)"', head)
    dims = np.array([int(m.group(i)) + 1 for i in (1, 2, 3)])
    origin = np.array([float(x) for x in m.group(4).split()])
    spacing = np.array([float(x) for x in m.group(5).split()])
    label = re.search(r'Name="([^"]+)"', head).group(1)
    blob = body[us:]
    if "vtkZLibDataCompressor" in head:
        hdr = np.frombuffer(blob[:32], dtype="<u8")
        clen = int(hdr[3])
        raw = zlib.decompress(blob[32:32 + clen])
    else:
        n = int(np.frombuffer(blob[:8], dtype="<u8")[0])
        raw = blob[8:8 + n]
    dt = "<f4" if 'type="Float32"' in head else "<f8"
    return np.frombuffer(raw, dtype=dt).copy(), dims, origin, spacing, label


def export_path(filename: str) -> str:
    return os.path.abspath(_vti_name(filename))
