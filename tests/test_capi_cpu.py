"""The C-ABI library without a GPU: it loads, exports every symbol include/sdfgpu.h declares,
and its host-only grid functions agree with the oracle.  No compute call is made here."""

from __future__ import annotations

import os
import re

import numpy as np
import pytest

import oracle
from conftest import ROOT


def declared_symbols():
    hdr = open(os.path.join(ROOT, "include", "sdfgpu.h")).read()
    hdr = re.sub(r"/\*.*?\*/", "", hdr, flags=re.S)
    return sorted(set(re.findall(r"\b(sdfgpu_[a-z_]+)\s*\(", hdr)))


def test_library_exports_every_declared_symbol():
    from stl2sdf import _native

    L = _native.lib()
    syms = declared_symbols()
    assert len(syms) >= 14
    for s in syms:
        assert hasattr(L, s), f"{s} declared in include/sdfgpu.h but not exported"
        assert s in _native.SIGNATURES, f"{s} has no ctypes signature"


def test_abi_version():
    from stl2sdf import _native

    assert _native.lib().sdfgpu_abi_version() == 1


@pytest.mark.parametrize("seed", range(8))
def test_grid_setup_matches_oracle(seed):
    from stl2sdf import _native

    rng = np.random.default_rng(seed)
    lo = rng.normal(size=3) * 10
    hi = lo + rng.uniform(0.1, 20, size=3)
    n = int(rng.integers(1, 300))
    o, amax, N, h, ngp = _native.grid_setup(lo, hi, n, 3)
    g = oracle.grid(lo, hi, n, 3)
    assert h == g["h"] and np.array_equal(o, g["origin"]) and np.array_equal(N, g["N"])
    assert np.array_equal(amax, g["amax"]) and ngp == g["ngp"]


def test_grid_from_cell_size_matches_oracle(icosphere_mesh):
    from stl2sdf import _native

    X, _ = icosphere_mesh
    for B in (0.05, 0.1, 0.33):
        o, amax, N, h, ngp = _native.grid_from_cell_size(X, B)
        g = oracle.grid_from_cell_size(X, B)
        assert h == g["h"] and np.array_equal(o, g["origin"]) and np.array_equal(N, g["N"]) and ngp == g["ngp"]


def test_grid_rejects_bad_input():
    from stl2sdf import _native

    with pytest.raises(_native.SdfGpuError):
        _native.grid_setup([0, 0, 0], [1, 1, 1], 0, 3)
    with pytest.raises(_native.SdfGpuError):
        _native.grid_setup([0, 0, 0], [0, 0, 0], 10, 3)
    with pytest.raises(_native.SdfGpuError):
        _native.grid_from_cell_size(np.zeros((3, 3)) + [[0, 0, 0], [1, 0, 0], [0, 1, 0]], -1.0)


def test_create_reports_missing_device():
    import torch

    from stl2sdf import _native

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(_native.SdfGpuError) as e:
        _native.Context(0)
    assert e.value.code == 2 and "device" in str(e.value)


def test_product_never_imports_the_oracle():
    pkg = os.path.join(ROOT, "stl2sdf.jl_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h", ".cpp")):
                text = open(os.path.join(dirpath, f), errors="ignore").read()
                assert "import oracle" not in text and "liboracle" not in text, f
