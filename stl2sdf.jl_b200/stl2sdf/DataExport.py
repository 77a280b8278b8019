"""VTK ImageData export, mirroring ``exportSdfToVTI`` (src/DataExport/ExportToVTI.jl:22-67).

The file holds one point field (``value_label``) over an ImageData with extent 0..N per axis,
origin ``grid.AABB_min`` and spacing ``cell_size`` (``cell_size/smooth`` with ``N*smooth`` cells
when ``smooth`` is given), values in the grid's x-fastest order.  The layout is the one WriteVTK
writes for ``vtk_grid(filename, x, y, z)``: appended raw binary, UInt64 block headers and zlib
compression (one block up to 4 MiB, as WriteVTK; larger fields in 4 MiB blocks compressed in
parallel).
"""

from __future__ import annotations

import os
import re
import zlib

import numpy as np


_BLOCK = 1 << 22  # 4 MiB uncompressed per zlib block


def _zlib_blocks(raw: bytes) -> bytes:
    """vtkZLibDataCompressor payload: UInt64 header [nblocks, block size, last block size,
    compressed sizes...] and the zlib streams of the blocks.  A field of one block is what WriteVTK
    writes; larger fields are cut into 4 MiB blocks compressed on all host cores (zlib releases the
    GIL), which every VTK reader accepts."""
    blocks = [raw[i:i + _BLOCK] for i in range(0, len(raw), _BLOCK)] or [b""]
    if len(blocks) == 1:
        comp = [zlib.compress(blocks[0], 6)]
    else:
        from concurrent.futures import ThreadPoolExecutor

        with ThreadPoolExecutor(max_workers=min(len(blocks), os.cpu_count() or 1)) as ex:
            comp = list(ex.map(lambda b: zlib.compress(b, 6), blocks))
    last = len(blocks[-1])
    hdr = np.array([len(blocks), len(blocks[0]) if len(blocks) > 1 else last, last] + [len(c) for c in comp], dtype="<u8")
    return hdr.tobytes() + b"".join(comp)


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
        payload = _zlib_blocks(raw)
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
        nb = int(np.frombuffer(blob[:8], dtype="<u8")[0])
        hdr = np.frombuffer(blob[:8 * (3 + nb)], dtype="<u8")
        pos, parts = 8 * (3 + nb), []
        for c in hdr[3:]:
            parts.append(zlib.decompress(blob[pos:pos + int(c)]))
            pos += int(c)
        raw = b"".join(parts)
    else:
        n = int(np.frombuffer(blob[:8], dtype="<u8")[0])
        raw = blob[8:8 + n]
    dt = "<f4" if 'type="Float32"' in head else "<f8"
    return np.frombuffer(raw, dtype=dt).copy(), dims, origin, spacing, label


def export_path(filename: str) -> str:
    return os.path.abspath(_vti_name(filename))
