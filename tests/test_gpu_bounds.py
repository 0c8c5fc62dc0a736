"""Bounds-checked build of the library (-DTC_BOUNDS_CHECK).

The checked library compares the index of every checked global access of the
step kernels (explicit RHS with both stagings, CN, x / y transforms in both
stagings, z solve, the streamed y / z passes, projection) with its buffer's
extent and records a violation instead of making the access.  These tests
run steps of several grids, precisions, schemes and kernel forms on that
library, in a child process that loads it in place of the normal one, and
check that no access was out of range.  A GPU fault is never provoked: a
violation is only recorded.
"""
import ctypes
import os
import subprocess
import sys

import pytest

from torchannel_b200 import _lib as L

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_normal_build_has_no_checks():
    """The normal library reports that no checks are compiled in (-1) without
    touching the device."""
    lib = L.load()
    flag, where = ctypes.c_int(7), ctypes.c_int(7)
    assert lib.tc_bounds_error(ctypes.byref(flag), ctypes.byref(where)) == L.TC_OK
    assert flag.value == -1 and where.value == 0


CHILD = r"""
import ctypes, sys
import numpy as np
import torch
sys.path.insert(0, ROOT)
from tests._util import make_oracle, make_gpu
from torchannel_b200 import _lib as L

lib = L.lib()
flag, where = ctypes.c_int(), ctypes.c_int()
assert lib.tc_bounds_error(ctypes.byref(flag), ctypes.byref(where)) == 0
assert flag.value == 0, ("checks not compiled in", flag.value)
cases = [
    # nx, ny, nz, precision, top, Poisson middle, bulk y, tensor-copy RHS
    (64, 64, 48, "mixed", "dirichlet", 0, True, True),
    (64, 64, 48, "fp64", "neumann", 2, False, True),
    (96, 48, 13, "mixed", "neumann", 0, True, False),
    (144, 36, 13, "fp64", "dirichlet", 0, True, True),
    (48, 96, 17, "mixed", "dirichlet", 2, True, True),
    (192, 192, 128, "mixed", "dirichlet", 0, True, True),
    (192, 192, 128, "fp64", "dirichlet", 2, True, True),
    (32, 24, 16, "fp64", "dirichlet", 0, False, False),
]
for nx, ny, nz, prec, top, middle, bulk, tma in cases:
    oc = make_oracle(nx, ny, nz, seed=5, top=top)
    ch = make_gpu(oc, prec)
    for opt, call in ((middle, ch.use_fused_poisson), (bulk, ch.use_bulk_ffty), (tma, ch.use_tma_rhs)):
        try:
            call(opt)
        except L.TCError:
            pass  # the form is not available for this grid: the default runs
    ch.set_state(oc.u, oc.v, oc.w)
    for scheme, dt, n in (("IMEX", 0.002, 5), ("AB2", 0.0004, 2), ("FE", 0.0004, 1), ("IMEX", 0.002, 4)):
        ch.step(scheme, dt, n)
    ch.get_state()
    ch.diagnostics()
    torch.cuda.synchronize()
    assert lib.tc_bounds_error(ctypes.byref(flag), ctypes.byref(where)) == 0
    print(nx, ny, nz, prec, top, middle, bulk, tma, "flag", flag.value, "where", where.value, flush=True)
    assert flag.value == 0, (nx, ny, nz, prec, "out-of-range access at", where.value)
# ensemble launches (the tensor-copy RHS of several members in one launch)
from torchannel_b200.ensemble import Ensemble, make_members
for prec in ("mixed", "fp64"):
    e = Ensemble(make_members(3, seed=2, sizes_xy=(64, 96), sizes_z=(16, 24)), precision=prec)
    e.batch()
    e.step_batch(5)
    torch.cuda.synchronize()
    assert lib.tc_bounds_error(ctypes.byref(flag), ctypes.byref(where)) == 0
    print("ensemble", prec, "flag", flag.value, "where", where.value, flush=True)
    assert flag.value == 0, ("ensemble", prec, "out-of-range access at", where.value)
print("bounds ok")
"""


@pytest.mark.gpu
def test_checked_build_steps_stay_in_bounds():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    if not os.path.exists(L.CHECKED_LIB_PATH):
        pytest.fail("bounds-checked library not built (torchannel_b200.build.build_checked)")
    env = dict(os.environ, TORCHANNEL_B200_LIB=L.CHECKED_LIB_PATH)
    r = subprocess.run([sys.executable, "-c", "ROOT = %r\n" % ROOT + CHILD], env=env, cwd=ROOT,
                       capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert "bounds ok" in r.stdout
