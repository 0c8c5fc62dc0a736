"""Generate golden vectors by running the reference TorChannel code itself.

Run once in a container that has the reference checked out (it cannot run on
a machine without it):

    python tests/golden/make_golden.py [--ref /root/reference]

The reference imports ``matplotlib.pyplot`` at module level (``utils.py:3``)
and matplotlib is not installed here, so a no-op stub package is written to a
temporary directory and put on ``sys.path`` first.  Everything runs on the CPU
in FP64 with ``PYTORCH_JIT=0`` (the TorchScript decorators become plain
Python, which computes the same arithmetic).

Outputs (small ``.npz`` files next to this script):
  ops_16x12x10.npz     operator-level vectors (advection, diffusion, fused
                       RHS, CN solves, divergence, Poisson, projection, bulk,
                       u_tau, CFL, BC fill, grids)
  step_imex_*.npz      whole IMEX steps of ``ChannelFlow.step_imex`` (CPU path)
  step_fe_16x12x10.npz one ``step_forward_euler`` (state captured after the
                       NameError its return raises)
  stats_16x12x10.npz   ``TurbulenceStats`` running sums after two samples
  run_16x12x10.npz     a short ``run_simulation`` with adaptive dt, stats and
                       saves: the files it writes, loaded back
"""
import argparse
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

STUB = '''
class _Any:
    def __getattr__(self, name):
        return _Any()
    def __call__(self, *a, **k):
        return _Any()
    def __iter__(self):
        return iter((_Any(), _Any()))
import sys as _s
_s.modules[__name__ + ".pyplot"] = _Any()
def use(*a, **k):
    pass
'''


def _setup(ref):
    stub = tempfile.mkdtemp(prefix="mplstub_")
    os.makedirs(os.path.join(stub, "matplotlib"))
    with open(os.path.join(stub, "matplotlib", "__init__.py"), "w") as f:
        f.write(STUB)
    with open(os.path.join(stub, "matplotlib", "pyplot.py"), "w") as f:
        f.write("def __getattr__(n):\n    from matplotlib import _Any\n    return _Any()\n")
    os.environ["PYTORCH_JIT"] = "0"
    sys.path.insert(0, ref)
    sys.path.insert(0, stub)


def _yaml(path, nx, ny, nz, *, top="dirichlet", dt=0.002, n_steps=3, scheme="IMEX",
          results="res", dt_update_interval=0, n_out=10, n_save=100, n_stats=0,
          t_stats=10.0, stretching="symmetric", Re=2870.0):
    import yaml
    cfg = {
        "grid": {"nx": nx, "ny": ny, "nz": nz},
        "domain": {"Lx": float(4 * np.pi), "Ly": float(4 * np.pi / 3), "Lz": 2.0,
                   "stretching_type": stretching},
        "flow": {"Re": Re, "Re_tau": 180.0, "U_bulk": 1.0, "gamma": 2.6},
        "boundary_conditions": {"top_wall": {"type": top}},
        "initialization": {"type": "parabolic", "perturbation_intensity": 0.1},
        "solver": {"type": "fft"},
        "time": {"dt": dt, "n_steps": n_steps, "CFL_target": 0.25,
                 "dt_update_interval": dt_update_interval, "dt_max": 0.011,
                 "dt_min": 0.0003, "scheme": scheme},
        "compute": {"device": "cpu"},
        "output": {"results_folder": results, "n_out": n_out, "n_save": n_save},
        "statistics": {"n_stats": n_stats, "t_stats": t_stats, "z_plus_target": 15.0},
    }
    with open(path, "w") as f:
        yaml.safe_dump(cfg, f)


def _np(t):
    return t.detach().cpu().numpy().copy() if hasattr(t, "detach") else np.asarray(t)


def make_ops(out):
    import torch
    import operators as O
    import projection_fft as PF
    import projection as PR
    import utils as U
    from solver import apply_bc_all
    torch.set_default_dtype(torch.float64)
    nx, ny, nz = 16, 12, 10
    Lx, Ly, Lz = 4 * np.pi, 4 * np.pi / 3, 2.0
    dx, dy, nu = Lx / nx, Ly / ny, 1.0 / 2870.0
    z_f, z_c, dz_f, dz_c = U.generate_grid(2.6, nz, Lz)
    g = torch.Generator().manual_seed(42)
    u = torch.randn(nx + 1, ny + 2, nz + 2, generator=g) * 0.1 + 1.0
    v = torch.randn(nx + 2, ny + 1, nz + 2, generator=g) * 0.1
    w = torch.randn(nx + 2, ny + 2, nz + 1, generator=g) * 0.1
    d = dict(nx=nx, ny=ny, nz=nz, Lx=Lx, Ly=Ly, Lz=Lz, nu=nu,
             z_f=_np(z_f), z_c=_np(z_c), dz_f=_np(dz_f), dz_c=_np(dz_c),
             u=_np(u), v=_np(v), w=_np(w))
    for top in ("dirichlet", "neumann"):
        uu, vv, ww = u.clone(), v.clone(), w.clone()
        apply_bc_all(uu, vv, ww, top)
        d[f"bc_{top}_u"], d[f"bc_{top}_v"], d[f"bc_{top}_w"] = _np(uu), _np(vv), _np(ww)
    d["adv_u"] = _np(O.advection_u(u, v, w, nx, ny, nz, dx, dy, dz_f))
    d["adv_v"] = _np(O.advection_v(u, v, w, nx, ny, nz, dx, dy, dz_f))
    d["adv_w"] = _np(O.advection_w(u, v, w, nx, ny, nz, dx, dy, dz_c))
    d["dxy_u"] = _np(O.diffusion_xy_u(u, nx, ny, nz, dx, dy, nu))
    d["dxy_v"] = _np(O.diffusion_xy_v(v, nx, ny, nz, dx, dy, nu))
    d["dxy_w"] = _np(O.diffusion_xy_w(w, nx, ny, nz, dx, dy, nu))
    d["dif_u"] = _np(O.diffusion_u(u, nx, ny, nz, dx, dy, dz_c, dz_f, nu))
    d["dif_v"] = _np(O.diffusion_v(v, nx, ny, nz, dx, dy, dz_c, dz_f, nu))
    d["dif_w"] = _np(O.diffusion_w(w, nx, ny, nz, dx, dy, dz_c, dz_f, nu))
    for name, f in (("imex", O.compute_momentum_rhs_fused_imex), ("v2", O.compute_momentum_rhs_fused_v2)):
        r = f(u, v, w, nx, ny, nz, dx, dy, dz_c, dz_f, nu)
        d[f"fused_{name}_u"], d[f"fused_{name}_v"], d[f"fused_{name}_w"] = map(_np, r)
    dt = torch.as_tensor(0.002)
    for top in ("dirichlet", "neumann"):
        d[f"cn_{top}_u"] = _np(O.solve_implicit_diffusion_u(u, dt, nx, ny, nz, dz_c, dz_f, nu, top_wall_bc_type=top))
        d[f"cn_{top}_v"] = _np(O.solve_implicit_diffusion_v(v, dt, nx, ny, nz, dz_c, dz_f, nu, top_wall_bc_type=top))
    d["cn_w"] = _np(O.solve_implicit_diffusion_w(w, dt, nx, ny, nz, dz_c, dz_f, nu))
    # PCR on a generic diagonally dominant batch
    a = torch.rand(nz, generator=g); b = 3 + torch.rand(nz, generator=g); c = torch.rand(nz, generator=g)
    rhs = torch.randn(7, nz, generator=g)
    d["pcr_a"], d["pcr_b"], d["pcr_c"], d["pcr_d"] = map(_np, (a, b, c, rhs))
    d["pcr_x"] = _np(O.solve_tridiagonal_batch(a, b, c, rhs))
    div = U.compute_divergence(u, v, w, nx, ny, nz, dx, dy, dz_f)
    d["div"] = _np(div)
    # Poisson on a compatible (dz_f-weighted zero-mean) right-hand side
    rhs = torch.rand(nx, ny, nz, generator=g) - 0.5
    rhs = rhs - (rhs * dz_f).sum() / (nx * ny * Lz)
    fd = PF.initialize_fft_solver(nx, ny, nz, dx, dy, dz_c, dz_f)
    d["poisson_rhs"] = _np(rhs)
    d["poisson_p"] = _np(PF.solve_poisson_fft(rhs, fd)).copy()
    d["tri_a"], d["tri_b"], d["tri_c"] = _np(fd["tri_a"]), _np(fd["tri_b"]), _np(fd["tri_c"])
    p = torch.randn(nx + 2, ny + 2, nz + 2, generator=g)
    d["proj_p"] = _np(p)
    pu, pv, pw = PR.project_velocity(u.clone(), v.clone(), w.clone(), p, nx, ny, nz, dx, dy, dz_c, dz_f, 0.002)
    d["proj_u"], d["proj_v"], d["proj_w"] = _np(pu), _np(pv), _np(pw)
    cell_vol = (dx * dy * dz_f.view(1, 1, -1)).expand(nx, ny, nz)
    d["bulk"] = float(U.compute_bulk_velocity(u, cell_vol, Lx * Ly * Lz))
    d["u_tau_dirichlet"] = float(U.compute_u_tau(u, z_c, nu))
    d["u_tau_neumann"] = float(U.compute_u_tau(u, z_c, nu, top_wall_bc_type="neumann"))
    d["cfl_dti"] = float(O.compute_cfl_fused(u, v, w, nx, ny, nz, dx, dy, dz_f, dz_c))
    for st in ("symmetric", "bottom"):
        zf, zc, dzf, dzc = U.generate_grid(2.6, 48, 2.0, stretching_type=st)
        d[f"grid_{st}_z_f"], d[f"grid_{st}_z_c"] = _np(zf), _np(zc)
        d[f"grid_{st}_dz_f"], d[f"grid_{st}_dz_c"] = _np(dzf), _np(dzc)
    zf, zc, dzf, dzc = U.generate_hybrid_grid(20, 30, 0.25, 2.0, 1.8)
    d["grid_hybrid_z_f"], d["grid_hybrid_z_c"] = _np(zf), _np(zc)
    d["grid_hybrid_dz_f"], d["grid_hybrid_dz_c"] = _np(zf[1:] - zf[:-1]), _np(dzc)
    np.savez(out, **d)


def _channel(tmp, nx, ny, nz, seed=0, **kw):
    import torch
    from solver import ChannelFlow
    cfgp = os.path.join(tmp, f"cfg_{nx}_{ny}_{nz}.yaml")
    _yaml(cfgp, nx, ny, nz, results=os.path.join(tmp, "res"), **kw)
    torch.manual_seed(seed)
    cwd = os.getcwd()
    os.chdir(tmp)
    try:
        cf = ChannelFlow(cfgp)
    finally:
        os.chdir(cwd)
    return cf


def make_step(tmp, out, nx, ny, nz, n_steps=3, top="dirichlet", dt=0.002, seed=0):
    cf = _channel(tmp, nx, ny, nz, seed=seed, top=top, dt=dt)
    d = dict(nx=nx, ny=ny, nz=nz, Lx=cf.Lx, Ly=cf.Ly, Lz=cf.Lz, nu=cf.nu, dt=dt,
             U_bulk=cf.U_bulk, top=top,
             z_f=_np(cf.z_f), z_c=_np(cf.z_c), dz_f=_np(cf.dz_f), dz_c=_np(cf.dz_c),
             u0=_np(cf.u), v0=_np(cf.v), w0=_np(cf.w), p0=_np(cf.p))
    # the reference's singular (0,0) Poisson mode can divide by an exact zero
    # pivot (e.g. at 24x16x12) and return NaN: only keep sizes where it does not
    assert np.isfinite(d["u0"]).all(), "reference returned non-finite fields"
    for s in range(1, n_steps + 1):
        cf.current_step = s
        ub, f = cf.step_imex(dt)
        d[f"u{s}"], d[f"v{s}"], d[f"w{s}"], d[f"p{s}"] = _np(cf.u), _np(cf.v), _np(cf.w), _np(cf.p)
        d[f"ubulk{s}"], d[f"forcing{s}"] = float(ub), float(f)
    np.savez(out, **d)


def make_fe(tmp, out, nx, ny, nz, dt=0.001):
    cf = _channel(tmp, nx, ny, nz, seed=3, scheme="FE", dt=dt)
    d = dict(nx=nx, ny=ny, nz=nz, dt=dt, u0=_np(cf.u), v0=_np(cf.v), w0=_np(cf.w))
    try:
        cf.step_forward_euler(dt)
        raise RuntimeError("reference FE step was expected to raise NameError")
    except NameError:
        pass
    d["u1"], d["v1"], d["w1"], d["p1"] = _np(cf.u), _np(cf.v), _np(cf.w), _np(cf.p)
    np.savez(out, **d)


def make_stats(tmp, out, nx, ny, nz):
    import torch
    from turbstats import TurbulenceStats
    import utils as U
    cf = _channel(tmp, nx, ny, nz, seed=5)
    ts = TurbulenceStats(nx, ny, nz, cf.Lx, cf.Ly, cf.Lz, cf.z_c, cf.z_f, cf.dz_c, cf.dz_f,
                         cf.dx, cf.dy, cf.nu, 180.0, z_plus_target=15.0)
    d = dict(nx=nx, ny=ny, nz=nz, k_bot=ts.k_bot, k_top=ts.k_top)
    for s in range(2):
        cf.current_step = s + 1
        cf.step_imex(0.002)
        d[f"u{s}"], d[f"v{s}"], d[f"w{s}"] = _np(cf.u), _np(cf.v), _np(cf.w)
        ts.accumulate_statistics(cf.u, cf.v, cf.w, U.compute_u_tau(cf.u, cf.z_c, cf.nu))
    for k in ("U_sum", "uu_sum", "vv_sum", "ww_sum", "uw_sum",
              "E_uu_2d_sum", "E_vv_2d_sum", "E_ww_2d_sum", "E_uw_2d_sum"):
        d[k] = _np(getattr(ts, k))
    d["n_samples"] = ts.n_samples
    np.savez(out, **d)


def make_run(tmp, out, nx, ny, nz):
    res = os.path.join(tmp, "res_run")
    cf = _channel(tmp, nx, ny, nz, seed=7, n_steps=20, dt=0.002, dt_update_interval=5,
                  n_out=5, n_save=10, n_stats=5, t_stats=0.0)
    cf.results_folder = res
    os.makedirs(res, exist_ok=True)
    cf.stats_output_path = os.path.join(res, "turbulence_stats.npz")
    cf.stats_state_path = os.path.join(res, "turbulence_stats_state.npz")
    d = dict(nx=nx, ny=ny, nz=nz, u0=_np(cf.u), v0=_np(cf.v), w0=_np(cf.w))
    cf.run_simulation()
    for fn, pre in (("fields_final.npz", "final_"), ("fields.npz", "save_"),
                    ("timeseries.npz", "ts_"), ("turbulence_stats.npz", "stats_"),
                    ("turbulence_stats_state.npz", "state_")):
        z = np.load(os.path.join(res, fn))
        for k in z.files:
            d[pre + k] = z[k]
    d["final_dt"] = cf.dt
    np.savez(out, **d)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    a = ap.parse_args()
    _setup(a.ref)
    tmp = tempfile.mkdtemp(prefix="golden_")
    make_ops(os.path.join(HERE, "ops_16x12x10.npz"))
    make_step(tmp, os.path.join(HERE, "step_imex_16x12x10.npz"), 16, 12, 10, n_steps=3)
    make_step(tmp, os.path.join(HERE, "step_imex_neumann_16x12x10.npz"), 16, 12, 10,
              n_steps=2, top="neumann", seed=1)
    make_step(tmp, os.path.join(HERE, "step_imex_32x24x16.npz"), 32, 24, 16, n_steps=2, seed=2)
    make_fe(tmp, os.path.join(HERE, "step_fe_16x12x10.npz"), 16, 12, 10)
    make_stats(tmp, os.path.join(HERE, "stats_16x12x10.npz"), 16, 12, 10)
    make_run(tmp, os.path.join(HERE, "run_16x12x10.npz"), 16, 12, 10)
    print("golden vectors written to", HERE)


if __name__ == "__main__":
    main()
