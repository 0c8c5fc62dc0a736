"""The benchmark configurations of the time step, run on the GPU through the C
ABI against the CPU oracle at their own sizes:

* the small plain-method case exactly: 64x64x48, seeded laminar + 0.1 noise,
  initial projection on the GPU, then 100 FP64 IMEX steps at dt 0.002,
  checked after every step (u, v, w <= 1e-12 relative, max|div| <= 1e-12,
  u_bulk <= 1e-13 absolute, forcing <= 1e-9 relative);
* the production grid 192x192x128: three FP64 steps against the oracle with
  the same bars, and mixed-precision steps against the FP64 oracle with the
  error of every derived quantity printed (post-projection divergence,
  u_bulk, u_tau, U(z), the Reynolds stresses): U(z) <= 0.5% after 10 and
  after 30 steps; max|div| <= 1e-6 after 30 steps, and <= 2e-6 after 10,
  while the seeded grid-scale noise (amplitude 0.1) still decays and FP32
  rounding of the stored w near the walls, divided by dz_f ~ 1e-3, sets the
  divergence;
* the one-sided (`bottom`) and `hybrid` stretched grids (utils.py:24-30,
  47-113), both top walls, against the oracle;
* one member of an ensemble advanced by the ensemble launches against the
  oracle directly.
"""
import numpy as np
import pytest

from oracle.grid import generate_hybrid_grid
from oracle.step import OracleChannel, initial_fields
from tests._util import dof, make_gpu, make_oracle, np_, rel

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _check_step(ch, oc, ub, f, s, tol=TOL, div_tol=1e-12):
    gu, gv, gw, _ = ch.get_state()
    for name, g, r in zip("uvw", (gu, gv, gw), (oc.u, oc.v, oc.w)):
        e = rel(np_(g), r)
        assert e < tol, (s, name, e)
    sc = np_(ch.scalars)
    assert abs(sc[1] - ub) < 1e-13, (s, sc[1], ub)
    assert abs(sc[0] - f) < 1e-9 * max(1.0, abs(f)), (s, sc[0], f)
    d = ch.diagnostics()
    assert d["max_div"] < div_tol and not d["nonfinite"], (s, d)


def test_small_config_100_steps(torch_cuda):
    """64x64x48, Lx 4 pi, Ly 4 pi / 3, Lz 2, gamma 2.6, Re 2870, dt 0.002,
    FP64, 100 IMEX steps; the GPU takes the raw seeded field, rescales it to
    U_bulk and projects it itself (solver.py:271-276, 345-370)."""
    nx, ny, nz = 64, 64, 48
    oc = make_oracle(nx, ny, nz, seed=0)
    u0, v0, w0, _ = initial_fields(nx, ny, nz, oc.z_c, oc.Lz, seed=0)
    ch = make_gpu(oc)
    ch.set_state(u0, v0, w0)
    ub = ch.bulk_velocity()
    ch.set_state(u0 * (1.0 / ub), v0, w0)
    ch.project_initial()
    gu, gv, gw, _ = ch.get_state()
    for name, g, r in zip("uvw", (gu, gv, gw), (oc.u, oc.v, oc.w)):
        assert rel(np_(g), r) < 1e-11, name        # after the initial projection (div 1e2 -> 1e-12)
    # continue from the oracle's projected state so every step starts equal
    ch.set_state(oc.u, oc.v, oc.w, forcing=0.0)
    dt = 0.002
    worst = 0.0
    for s in range(1, 101):
        ub, f = oc.step_imex(dt)
        ch.step("IMEX", dt)
        _check_step(ch, oc, ub, f, s)
        gu = np_(ch.get_field("u"))
        worst = max(worst, rel(gu, oc.u))
    print(f"64x64x48, 100 FP64 IMEX steps: worst relative u error {worst:.2e}")


@pytest.fixture(scope="module")
def production_run():
    """The oracle on 192x192x128 (seeded laminar + 0.1 noise, projected), dt
    from the CFL rule at CFL 0.25 (solver.py:465-496), 30 FP64 IMEX steps;
    states kept after steps 1, 2, 3, 10 and 30."""
    nx, ny, nz = 192, 192, 128
    oc = make_oracle(nx, ny, nz, seed=0)
    start = (oc.u.copy(), oc.v.copy(), oc.w.copy())
    dt = oc.cfl_dt(0.25, 3e-4, 0.011)
    keep = {}
    for s in range(1, 31):
        ub, f = oc.step_imex(dt)
        if s in (1, 2, 3, 10, 30):
            keep[s] = dict(u=oc.u.copy(), v=oc.v.copy(), w=oc.w.copy(), ub=ub, f=f)
    return oc, start, dt, keep


def test_production_grid_fp64_steps(torch_cuda, production_run):
    oc, (u0, v0, w0), dt, keep = production_run
    ch = make_gpu(oc)
    ch.set_state(u0, v0, w0, forcing=0.0)
    for s in (1, 2, 3):
        ch.step("IMEX", dt)
        gu, gv, gw, _ = ch.get_state()
        k = keep[s]
        for name, g in zip("uvw", (gu, gv, gw)):
            e = rel(np_(g), k[name])
            assert e < TOL, (s, name, e)
        sc = np_(ch.scalars)
        assert abs(sc[1] - k["ub"]) < 1e-13 and abs(sc[0] - k["f"]) < 1e-9 * max(1.0, abs(k["f"]))
        assert ch.diagnostics()["max_div"] < 1e-12


def _profiles(u, v, w, nx, ny, nz):
    """U(z) and the Reynolds stresses on cell centres (turbstats.py:101-150)."""
    uc = 0.5 * (u[0:nx, 1:ny + 1, 1:nz + 1] + u[1:nx + 1, 1:ny + 1, 1:nz + 1])
    vc = 0.5 * (v[1:nx + 1, 0:ny, 1:nz + 1] + v[1:nx + 1, 1:ny + 1, 1:nz + 1])
    wc = 0.5 * (w[1:nx + 1, 1:ny + 1, 0:nz] + w[1:nx + 1, 1:ny + 1, 1:nz + 1])
    U = uc.mean(axis=(0, 1))
    up, vp, wp = uc - U, vc - vc.mean(axis=(0, 1)), wc - wc.mean(axis=(0, 1))
    return dict(U=U, uu=(up * up).mean(axis=(0, 1)), vv=(vp * vp).mean(axis=(0, 1)),
                ww=(wp * wp).mean(axis=(0, 1)), uw=(up * wp).mean(axis=(0, 1)))


def _mixed_report(ch, oc, k, label):
    from oracle import ops
    nx, ny, nz = oc.nx, oc.ny, oc.nz
    gu, gv, gw, _ = ch.get_state()
    gu, gv, gw = np_(gu), np_(gv), np_(gw)
    d = ch.diagnostics()
    pg, pr = _profiles(gu, gv, gw, nx, ny, nz), _profiles(k["u"], k["v"], k["w"], nx, ny, nz)
    err = {q: float(np.max(np.abs(pg[q] - pr[q])) / np.max(np.abs(pr[q]))) for q in pg}
    ut_r = ops.compute_u_tau(k["u"], oc.z_c, oc.nu)
    report = dict(max_div=d["max_div"], u_bulk_abs=abs(d["u_bulk"] - k["ub"]),
                  u_tau_rel=abs(d["u_tau"] - ut_r) / ut_r,
                  u_rel=rel(dof("u", gu, nx, ny, nz), dof("u", k["u"], nx, ny, nz)),
                  w_rel=rel(dof("w", gw, nx, ny, nz), dof("w", k["w"], nx, ny, nz)), **err)
    print(f"192x192x128 {label} vs FP64 oracle: " + ", ".join(f"{q} {v:.2e}" for q, v in report.items()))
    assert not d["nonfinite"]
    assert report["u_bulk_abs"] < 1e-9
    return report


@pytest.mark.parametrize("fp32_poisson", [False, True])
def test_production_grid_mixed_vs_fp64_oracle(torch_cuda, production_run, fp32_poisson):
    """Mixed precision (FP32 fields; FP64 Poisson, or the single-precision
    Poisson step after 10 FP64 warm-up steps) against the FP64 oracle."""
    oc, (u0, v0, w0), dt, keep = production_run
    ch = make_gpu(oc, precision="mixed")
    ch.set_state(u0, v0, w0, forcing=0.0)
    if fp32_poisson:
        ch.use_fp32_poisson(True, warm_steps=10)
    label = "mixed, FP32 Poisson" if fp32_poisson else "mixed"
    ch.step("IMEX", dt, 10)
    r10 = _mixed_report(ch, oc, keep[10], label + ", 10 steps")
    assert r10["U"] <= 5e-3
    assert r10["max_div"] <= 2e-6
    ch.step("IMEX", dt, 20)
    r30 = _mixed_report(ch, oc, keep[30], label + ", 30 steps")
    assert r30["U"] <= 5e-3
    assert r30["max_div"] <= 1e-6
    assert ch.error_word() == 0


@pytest.mark.parametrize("top", ["dirichlet", "neumann"])
def test_bottom_stretched_grid(torch_cuda, top):
    nx, ny, nz = 32, 24, 20
    oc = make_oracle(nx, ny, nz, seed=31, top=top, stretching="bottom")
    assert oc.dz_f[0] < oc.dz_f[-1] / 10            # one-sided: fine at the bottom wall only
    ch = make_gpu(oc)
    ch.set_state(oc.u, oc.v, oc.w, forcing=0.0)
    for s in range(1, 5):
        ub, f = oc.step_imex(0.002)
        ch.step("IMEX", 0.002)
        _check_step(ch, oc, ub, f, s)


@pytest.mark.parametrize("top", ["dirichlet", "neumann"])
def test_hybrid_grid(torch_cuda, top):
    """Uniform layer of 12 cells up to z = 0.25, one-sided tanh above (gamma 1.8)."""
    nx, ny = 32, 24
    grid = generate_hybrid_grid(12, 18, 0.25, 2.0, 1.8)
    nz = len(grid[2])
    oc = OracleChannel(nx, ny, nz, 4 * np.pi, 4 * np.pi / 3, 2.0, 2870.0, top_wall_bc_type=top, grid=grid)
    oc.init_fresh(seed=32)
    ch = make_gpu(oc)
    ch.set_state(oc.u, oc.v, oc.w, forcing=0.0)
    for s in range(1, 5):
        ub, f = oc.step_imex(0.002)
        ch.step("IMEX", 0.002)
        _check_step(ch, oc, ub, f, s)


def test_ensemble_member_vs_oracle(torch_cuda):
    """Three uneven FP64 members advanced together by the ensemble launches;
    every member against its own oracle channel (same Re, gamma, dt)."""
    from torchannel_b200.ensemble import Ensemble, make_members
    members = make_members(3, seed=5, sizes_xy=(64, 96, 128), sizes_z=(16, 24, 40))
    e = Ensemble(members, precision="fp64")
    oracles = []
    for m, ch in zip(members, e.channels):
        oc = OracleChannel(m["nx"], m["ny"], m["nz"], 4 * np.pi, 4 * np.pi / 3, 2.0, m["Re"], gamma=m["gamma"])
        u, v, w, _ = ch.get_state()
        oc.set_state(np_(u), np_(v), np_(w))
        oracles.append(oc)
    b = e.batch()
    for s in range(1, 5):
        b.step("IMEX", e.dts, 1)
        torch_cuda.cuda.synchronize()
        for oc, ch, dt in zip(oracles, e.channels, e.dts):
            ub, f = oc.step_imex(dt)
            _check_step(ch, oc, ub, f, s)
