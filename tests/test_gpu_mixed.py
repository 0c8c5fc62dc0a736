"""Mixed precision (FP32 velocity fields and AB2 history, FP64 Poisson
spectrum / pressure / tridiagonal arithmetic / bulk forcing / statistics sums)
against the FP64 oracle.  Tolerances are stated per quantity:

* u, v, w after 20 IMEX steps: <= 2e-5 relative (FP32 storage, ~1e-7 per step)
* post-projection max|div| <= 1e-6 (the bound the mixed step is built to)
* u_bulk <= 1e-9 absolute; U(z) <= 1e-6 relative (0.5% allowed)
* statistics sums <= 1e-5 relative
"""
import numpy as np
import pytest

from oracle.stats import TurbulenceStats
from tests._util import dof, make_gpu, make_oracle, np_, rel

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def test_mixed_state_roundtrip(torch_cuda):
    nx, ny, nz = 32, 24, 16
    oc = make_oracle(nx, ny, nz, seed=1)
    ch = make_gpu(oc, precision="mixed")
    ch.set_state(oc.u, oc.v, oc.w)
    gu, gv, gw, _ = ch.get_state()
    # u is stored as u - U0(z) in FP32: error below one FP32 ulp of the deviation
    ud = oc.u[1:nx + 1, 1:ny + 1, 1:nz + 1]
    dev = np.max(np.abs(ud - ud.mean(axis=(0, 1))))
    assert np.max(np.abs(np_(gu) - oc.u)) <= 1.2e-7 * dev + 1e-15
    assert np.max(np.abs(np_(gv) - oc.v)) <= 1.2e-7 * np.max(np.abs(oc.v))
    assert np.max(np.abs(np_(gw) - oc.w)) <= 1.2e-7 * np.max(np.abs(oc.w))


@pytest.mark.parametrize("top", ["dirichlet", "neumann"])
def test_mixed_imex_vs_fp64_oracle(torch_cuda, top):
    nx, ny, nz = 48, 32, 24
    oc = make_oracle(nx, ny, nz, seed=21, top=top)
    ch = make_gpu(oc, precision="mixed")
    ch.set_state(oc.u, oc.v, oc.w)
    dt = 0.004
    for s in range(20):
        ub, f = oc.step_imex(dt)
        ch.step("IMEX", dt)
    gu, gv, gw, gp = ch.get_state()
    for name, g, r in zip("uvw", (gu, gv, gw), (oc.u, oc.v, oc.w)):
        assert rel(dof(name, np_(g), nx, ny, nz), dof(name, r, nx, ny, nz)) < 2e-5, name
    d = ch.diagnostics()
    assert d["max_div"] <= 1e-6, d
    assert abs(d["u_bulk"] - ub) < 1e-9
    assert abs(d["forcing"] - f) < 1e-6 * max(1.0, abs(f))
    Ug = np_(gu)[1:nx + 1, 1:ny + 1, 1:nz + 1].mean(axis=(0, 1))
    Ur = oc.u[1:nx + 1, 1:ny + 1, 1:nz + 1].mean(axis=(0, 1))
    assert np.max(np.abs(Ug - Ur)) / np.max(np.abs(Ur)) < 1e-6


def test_mixed_poisson_is_fp64(torch_cuda):
    """The Poisson solve keeps its FP64 path in the mixed form."""
    from oracle import poisson
    nx, ny, nz = 48, 32, 24
    oc = make_oracle(nx, ny, nz)
    rng = np.random.default_rng(3)
    rhs = rng.random((nx, ny, nz)) - 0.5
    rhs -= np.sum(rhs * oc.dz_f) / (nx * ny * oc.Lz)
    ref = poisson.solve_poisson_fft(rhs, oc.fd)
    ch = make_gpu(oc, precision="mixed")
    p = np_(ch.poisson_solve(rhs))
    assert rel(dof("p", p, nx, ny, nz), dof("p", ref, nx, ny, nz)) < 1e-11


def test_mixed_stats(torch_cuda):
    nx, ny, nz = 32, 24, 16
    oc = make_oracle(nx, ny, nz, seed=4)
    ch = make_gpu(oc, precision="mixed")
    ts = TurbulenceStats(nx, ny, nz, oc.Lx, oc.Ly, oc.Lz, oc.z_c, oc.dx, oc.dy, oc.nu, 180.0, 15.0)
    ch.stats_init(oc.z_c, 180.0, 15.0)
    ch.set_state(oc.u, oc.v, oc.w)
    for s in range(3):
        oc.step_imex(0.002)
        ch.step("IMEX", 0.002)
        ts.accumulate_statistics(oc.u, oc.v, oc.w)
        ch.stats_accumulate()
    got = ch.stats_read()
    for k in ("U_sum", "uu_sum", "vv_sum", "ww_sum", "uw_sum",
              "E_uu_2d_sum", "E_vv_2d_sum", "E_ww_2d_sum", "E_uw_2d_sum"):
        assert rel(got[k], getattr(ts, k)) < 1e-5, k


@pytest.mark.parametrize("scheme", ["AB2", "FE"])
def test_mixed_other_schemes(torch_cuda, scheme):
    nx, ny, nz = 24, 36, 20
    oc = make_oracle(nx, ny, nz, seed=8)
    ch = make_gpu(oc, precision="mixed")
    ch.set_state(oc.u, oc.v, oc.w)
    step = oc.step_ab2 if scheme == "AB2" else oc.step_fe
    for s in range(5):
        step(0.0005)
        ch.step(scheme, 0.0005)
    gu, gv, gw, _ = ch.get_state()
    for name, g, r in zip("uvw", (gu, gv, gw), (oc.u, oc.v, oc.w)):
        assert rel(dof(name, np_(g), nx, ny, nz), dof(name, r, nx, ny, nz)) < 2e-5, name
    assert ch.diagnostics()["max_div"] <= 1e-6


# ---- single-precision Poisson step (FP32 spectrum, FP64 low modes, increment
# over the previous pressure) -------------------------------------------------
FP32P_SIZES = [(64, 64, 48), (96, 64, 40), (128, 96, 24), (192, 192, 16)]


@pytest.mark.parametrize("nx,ny,nz", FP32P_SIZES)
def test_fp32_poisson_steps_vs_fp64_oracle(torch_cuda, nx, ny, nz):
    """20 IMEX steps with the single-precision Poisson solve from step 3 on,
    against the FP64 oracle: u, v, w <= 2e-5 relative (as the mixed form),
    u_bulk <= 1e-9, U(z) <= 1e-6 relative; the post-projection divergence is
    printed (FP32 rounding of the increment) and bounded by 1e-5."""
    oc = make_oracle(nx, ny, nz, seed=41)
    ch = make_gpu(oc, precision="mixed")
    ch.set_state(oc.u, oc.v, oc.w)
    ch.use_fp32_poisson(True, warm_steps=2)
    dt = 0.004
    divs = []
    for s in range(20):
        ub, f = oc.step_imex(dt)
        ch.step("IMEX", dt)
        divs.append(ch.diagnostics()["max_div"])
    gu, gv, gw, gp = ch.get_state()
    for name, g, r in zip("uvw", (gu, gv, gw), (oc.u, oc.v, oc.w)):
        assert rel(dof(name, np_(g), nx, ny, nz), dof(name, r, nx, ny, nz)) < 2e-5, name
    assert rel(dof("p", np_(gp), nx, ny, nz), dof("p", oc.p, nx, ny, nz)) < 1e-3
    d = ch.diagnostics()
    print(f"{nx}x{ny}x{nz} FP32 Poisson: max|div| per step {['%.1e' % x for x in divs]}")
    assert max(divs) <= 1e-5 and not d["nonfinite"], divs
    assert abs(d["u_bulk"] - ub) < 1e-9
    Ug = np_(gu)[1:nx + 1, 1:ny + 1, 1:nz + 1].mean(axis=(0, 1))
    Ur = oc.u[1:nx + 1, 1:ny + 1, 1:nz + 1].mean(axis=(0, 1))
    assert np.max(np.abs(Ug - Ur)) / np.max(np.abs(Ur)) < 1e-6
    assert ch.error_word() == 0


def test_fp32_poisson_graph_replay_is_bitwise_identical(torch_cuda):
    nx, ny, nz = 64, 64, 24
    oc = make_oracle(nx, ny, nz, seed=42)
    a, b = make_gpu(oc, "mixed"), make_gpu(oc, "mixed")
    a.use_graphs(False)
    for ch in (a, b):
        ch.set_state(oc.u, oc.v, oc.w)
        ch.use_fp32_poisson(True, warm_steps=3)
        ch.step("IMEX", 0.003, 9)       # 3 FP64 warm-up steps, then graph pairs + remainder
        ch.step("IMEX", 0.002, 7)
    for x, y in zip(a.get_state(), b.get_state()):
        assert np.array_equal(np_(x), np_(y))
    assert np.array_equal(np_(a.scalars), np_(b.scalars))


def test_fp32_poisson_refused_where_unavailable(torch_cuda):
    from torchannel_b200._lib import TCError
    oc = make_oracle(32, 48, 16)                    # ny = 48: no register transform of the fused kernel
    with pytest.raises(TCError):
        make_gpu(oc, "mixed").use_fp32_poisson(True)
    with pytest.raises(TCError):
        make_gpu(make_oracle(64, 64, 16), "fp64").use_fp32_poisson(True)
