"""The allocation-free Poisson entry point, tc_poisson_solve_noalloc.

It exists for callers that cannot give the library device memory: programs
whose device memory is handed out by their own pool manager (a raw cudaMalloc
would be refused or would fight that pool) and loops that must not take the
device-wide synchronisation a cudaMalloc / cudaFree can cause.  Its scratch is
a fixed 64 MiB array in device memory, so a grid may need at most 67108864
bytes of it (nx*ny*nz*8 + (nx/2+1)*ny*nz*16 + small tables).  These tests call
it through the C ABI and check it against the workspace-based entry point
tc_poisson_solve, including a grid whose scratch ends close to the array's
end.

This file is named to be collected last.
"""
import ctypes

import numpy as np
import pytest

from torchannel_b200 import _lib as L
from torchannel_b200.grid import generate_grid


def _noalloc(lib, nx, ny, nz, Lx, Ly, dzf_dev, dzc_dev, rhs_dev, p_dev, stream):
    return lib.tc_poisson_solve_noalloc(nx, ny, nz, Lx, Ly, ctypes.c_void_p(dzf_dev.data_ptr()),
                                        ctypes.c_void_p(dzc_dev.data_ptr()), ctypes.c_void_p(rhs_dev.data_ptr()),
                                        ctypes.c_void_p(p_dev.data_ptr()), stream)


def _compatible_rhs(rng, nx, ny, nz, dz_f, Lz):
    r = rng.random((nx, ny, nz)) - 0.5
    return r - np.sum(r * dz_f) / (nx * ny * Lz)


LIMIT = 64 << 20


def _scratch_bytes(nx, ny, nz):
    """The entry point's scratch layout: rhs/p field, spectrum, k2x, k2y,
    cl, cr and the two twiddle tables, each region 256-byte aligned."""
    nxh = nx // 2 + 1
    o = 0
    for s in (nx * ny * nz * 8, nxh * nz * ny * 16, nxh * 8, ny * 8, nz * 8, nz * 8, nx * 16, ny * 16):
        o = (o + 255) & ~255
        o += s
    return o


@pytest.mark.parametrize("nx,ny,nz", [(192, 192, 128), (128, 128, 256), (162, 162, 162), (162, 128, 202)])
def test_noalloc_rejects_oversize_grid(nx, ny, nz):
    """Grids whose scratch exceeds the static array get TC_ERR_SIZE (no GPU
    work is attempted before the size check); (162, 128, 202) is one plane
    more than a grid that needs exactly the whole array."""
    assert _scratch_bytes(nx, ny, nz) > LIMIT
    lib = L.load()
    rc = lib.tc_poisson_solve_noalloc(nx, ny, nz, 1.0, 1.0, ctypes.c_void_p(8), ctypes.c_void_p(8),
                                      ctypes.c_void_p(8), ctypes.c_void_p(8), None)
    assert rc == L.TC_ERR_SIZE
    assert b"static maximum" in lib.tc_last_error()


def test_noalloc_limit_examples():
    """The documented examples: 144x144x192 fits, 162x128x201 needs exactly
    the whole array."""
    assert _scratch_bytes(144, 144, 192) == 64153088 <= LIMIT
    assert _scratch_bytes(162, 128, 201) == LIMIT


@pytest.mark.gpu
@pytest.mark.parametrize("nx,ny,nz", [(32, 24, 16), (96, 96, 64), (162, 128, 201)])
def test_noalloc_matches_workspace_solve(nx, ny, nz):
    """(162, 128, 201) needs exactly the 67108864 bytes of the static array:
    its last table ends at the array's last byte (162 takes the shared-memory
    Stockham transforms along x, 128 and 96 the register ones)."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from torchannel_b200.core import Channel
    Lx, Ly, Lz = 4 * np.pi, 4 * np.pi / 3, 2.0
    _, _, dz_f, dz_c = generate_grid(2.6, nz, Lz)
    ch = Channel(nx, ny, nz, Lx, Ly, Lz, 1 / 2870.0, dz_f, dz_c)
    lib = ch.lib
    dzf = torch.as_tensor(dz_f, device="cuda")
    dzc = torch.as_tensor(dz_c, device="cuda")
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(nx + nz)
    # two calls in a row (different right-hand sides): the shared scratch
    # keeps the first call's contents, which must not leak into the second
    for call in range(2):
        rhs = _compatible_rhs(rng, nx, ny, nz, dz_f, Lz)
        want = ch.poisson_solve(rhs).cpu().numpy()
        rhs_dev = torch.as_tensor(rhs, device="cuda").contiguous()
        p_dev = torch.empty((nx + 2, ny + 2, nz + 2), dtype=torch.float64, device="cuda")
        assert _noalloc(lib, nx, ny, nz, Lx, Ly, dzf, dzc, rhs_dev, p_dev, stream) == L.TC_OK, \
            lib.tc_last_error()
        torch.cuda.synchronize()
        got = p_dev.cpu().numpy()
        scale = np.max(np.abs(want))
        assert np.max(np.abs(got - want)) / scale < 1e-11, call
        gi, wi = got[1:-1, 1:-1, 1:-1], want[1:-1, 1:-1, 1:-1]
        assert np.max(np.abs((gi - gi.mean()) - (wi - wi.mean()))) / scale < 1e-11, call


@pytest.mark.gpu
def test_noalloc_rejects_host_arrays():
    """Host arrays are refused with TC_ERR_ARG before any launch (they would
    make the kernels fault)."""
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    lib = L.load()
    nx, ny, nz = 32, 24, 16
    _, _, dz_f, dz_c = generate_grid(2.6, nz, 2.0)
    dzf = torch.as_tensor(dz_f, device="cuda")
    dzc = torch.as_tensor(dz_c, device="cuda")
    rhs = torch.zeros((nx, ny, nz), dtype=torch.float64, device="cuda")
    p = torch.empty((nx + 2, ny + 2, nz + 2), dtype=torch.float64, device="cuda")
    host_dzf = np.ascontiguousarray(dz_f)
    rc = lib.tc_poisson_solve_noalloc(nx, ny, nz, 1.0, 1.0, ctypes.c_void_p(host_dzf.ctypes.data),
                                      ctypes.c_void_p(dzc.data_ptr()), ctypes.c_void_p(rhs.data_ptr()),
                                      ctypes.c_void_p(p.data_ptr()), None)
    assert rc == L.TC_ERR_ARG and b"dz_f" in lib.tc_last_error()
    host_p = torch.empty((nx + 2, ny + 2, nz + 2), dtype=torch.float64)
    rc = lib.tc_poisson_solve_noalloc(nx, ny, nz, 1.0, 1.0, ctypes.c_void_p(dzf.data_ptr()),
                                      ctypes.c_void_p(dzc.data_ptr()), ctypes.c_void_p(rhs.data_ptr()),
                                      ctypes.c_void_p(host_p.data_ptr()), None)
    assert rc == L.TC_ERR_ARG and lib.tc_last_error().startswith(b"p must be device memory")
