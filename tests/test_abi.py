"""The C-ABI library loads without a GPU and exports every declared entry point."""

import ctypes
import pathlib
import re

import pytest
import torch

import pygrog_b200
from pygrog_b200 import _ext, _lib

HEADER = pathlib.Path(__file__).resolve().parent.parent / "include" / "pygrog_b200.h"


def declared_symbols():
    txt = HEADER.read_text()
    return sorted(set(re.findall(r"PGB_API\s+[\w\s\*]+?\b(pgb_\w+)\s*\(", txt)))


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "pgb_grog_grid" in names and "pgb_scatter_add" in names
    assert len(names) >= 16


def test_library_exports_every_declared_symbol():
    lib = pygrog_b200.load_library()
    for name in declared_symbols():
        assert hasattr(lib, name), f"{name} declared in include/pygrog_b200.h but not exported"
    # and the ctypes binding knows every exported entry point it declares
    for name in _lib.exported_names():
        assert name in declared_symbols(), f"binding expects undeclared symbol {name}"


def test_version_and_error_string():
    lib = pygrog_b200.load_library()
    assert b"sm_100a" in lib.pgb_version()
    assert isinstance(lib.pgb_last_error(), bytes)


def test_invalid_arguments_are_rejected_without_touching_the_gpu():
    lib = pygrog_b200.load_library()
    # negative sizes and a bad dtype code come back as status codes, no launch
    st = lib.pgb_scatter_add(None, -1, None, None, None, 5, 0, None)
    assert st == 1
    assert b"negative" in lib.pgb_last_error()
    st = lib.pgb_grog_interpolate(None, None, None, None, 4, 1, 2000, 3, 0, None)
    assert st == 4  # C above the limit
    st = lib.pgb_scatter_add_binned(None, 10, None, None, None, 3, None, 1, 0, 0, None)
    assert st == 1 and b"bin_size" in lib.pgb_last_error()


def test_shim_raises_reference_messages_on_bad_shapes():
    d = torch.zeros(4, 2, dtype=torch.complex64)
    with pytest.raises(RuntimeError, match="data must be 3-D"):
        _ext.grog_interpolate(d, torch.zeros(4, dtype=torch.int64), torch.zeros(3, 2, 2, dtype=torch.complex64))
    with pytest.raises(RuntimeError, match="indices must be int64"):
        _ext.scatter_add(torch.zeros(8, dtype=torch.complex64), torch.zeros(3, dtype=torch.complex64),
                         torch.zeros(3, dtype=torch.int32), torch.zeros(3))
    with pytest.raises(RuntimeError, match="data/weights size mismatch"):
        _ext.scatter_add(torch.zeros(8, dtype=torch.complex64), torch.zeros(3, dtype=torch.complex64),
                         torch.zeros(3, dtype=torch.int64), torch.zeros(2))
    with pytest.raises(RuntimeError, match="psf/w_sq dtype mismatch"):
        _ext.psf_scatter_scalar(torch.zeros(8), torch.zeros(3, dtype=torch.int64), torch.zeros(3, dtype=torch.float64))


def test_cpu_tensors_fail_loudly():
    """No CPU fallback: valid CPU inputs raise instead of silently computing."""
    with pytest.raises(RuntimeError, match="CUDA"):
        _ext.gather(torch.zeros(8, dtype=torch.complex64), torch.zeros(3, dtype=torch.int64), torch.zeros(3))
