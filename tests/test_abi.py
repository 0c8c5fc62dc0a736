"""C-ABI library checks that need no GPU: it loads, exports every symbol the
header declares, and validates grid descriptors."""
import ctypes
import os
import re

import numpy as np
import pytest

from torchannel_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "torchannel_b200.h")


def header_symbols():
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(tc_[a-z0-9_]+)\s*\(", txt)))


def test_library_loads_and_exports_header_symbols():
    lib = L.load()
    syms = header_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(lib, s), s
    assert sorted(n for n, _, _ in L.SIGNATURES) == syms
    assert b"sm_100a" in lib.tc_version()


def _desc(nx=16, ny=12, nz=10, precision=L.TC_FP64):
    from torchannel_b200.grid import generate_grid
    _, _, dzf, dzc = generate_grid(2.6, nz, 2.0)
    d = L.GridDesc()
    d.nx, d.ny, d.nz = nx, ny, nz
    d.Lx, d.Ly, d.Lz, d.nu, d.U_bulk = 4 * np.pi, 4 * np.pi / 3, 2.0, 1 / 2870.0, 1.0
    d.top_wall, d.precision, d.rhs_path = 0, precision, 0
    keep = (np.ascontiguousarray(dzf), np.ascontiguousarray(dzc))
    d.dz_f = keep[0].ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    d.dz_c = keep[1].ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    return d, keep


def test_workspace_bytes():
    lib = L.load()
    d, keep = _desc(192, 192, 128)
    n = ctypes.c_size_t()
    assert lib.tc_workspace_bytes(ctypes.byref(d), ctypes.byref(n)) == L.TC_OK
    fields = 10 * 192 * 192 * 129 * 8
    assert fields < n.value < 1.6 * fields
    d2, keep2 = _desc(192, 192, 128, L.TC_MIXED)
    n2 = ctypes.c_size_t()
    assert lib.tc_workspace_bytes(ctypes.byref(d2), ctypes.byref(n2)) == L.TC_OK
    assert n2.value < n.value


@pytest.mark.parametrize("nx,ny,code", [(15, 12, L.TC_ERR_SIZE), (20, 12, L.TC_ERR_SIZE),
                                        (14, 12, L.TC_ERR_SIZE), (16, 12, L.TC_OK)])
def test_size_validation(nx, ny, code):
    lib = L.load()
    d, keep = _desc(nx, ny)
    n = ctypes.c_size_t()
    assert lib.tc_workspace_bytes(ctypes.byref(d), ctypes.byref(n)) == code
    if code:
        assert lib.tc_last_error()


def test_null_arguments():
    lib = L.load()
    assert lib.tc_workspace_bytes(None, None) == L.TC_ERR_ARG
    assert lib.tc_step(None, 0, 0.1, 1, None) == L.TC_ERR_ARG
