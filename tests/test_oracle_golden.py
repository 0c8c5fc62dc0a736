"""Pin the CPU oracle to golden vectors produced by the reference itself
(``tests/golden/make_golden.py``).  CPU only."""
import numpy as np
import pytest

from oracle import ops, poisson, grid as ogrid, stats as ostats
from oracle.step import OracleChannel


def rel(a, b):
    d = np.max(np.abs(np.asarray(a) - np.asarray(b)))
    s = np.max(np.abs(np.asarray(b)))
    return d / (s if s > 0 else 1.0)


@pytest.fixture(scope="module")
def G(golden):
    return golden("ops_16x12x10.npz")


def _args(G):
    nx, ny, nz = int(G["nx"]), int(G["ny"]), int(G["nz"])
    return nx, ny, nz, float(G["Lx"]) / nx, float(G["Ly"]) / ny, float(G["nu"])


@pytest.mark.parametrize("st", ["symmetric", "bottom"])
def test_grid(G, st):
    z_f, z_c, dz_f, dz_c = ogrid.generate_grid(2.6, 48, 2.0, st)
    for k, a in (("z_f", z_f), ("z_c", z_c), ("dz_f", dz_f), ("dz_c", dz_c)):
        assert rel(a, G[f"grid_{st}_{k}"]) < 1e-14


def test_hybrid_grid(G):
    z_f, z_c, dz_f, dz_c = ogrid.generate_hybrid_grid(20, 30, 0.25, 2.0, 1.8)
    assert rel(z_f, G["grid_hybrid_z_f"]) < 1e-14
    assert rel(z_c, G["grid_hybrid_z_c"]) < 1e-14
    assert rel(dz_c, G["grid_hybrid_dz_c"]) < 1e-13


@pytest.mark.parametrize("top", ["dirichlet", "neumann"])
def test_bc(G, top):
    u, v, w = G["u"].copy(), G["v"].copy(), G["w"].copy()
    ops.apply_bc_all(u, v, w, top)
    assert np.array_equal(u, G[f"bc_{top}_u"])
    assert np.array_equal(v, G[f"bc_{top}_v"])
    assert np.array_equal(w, G[f"bc_{top}_w"])


def test_advection_diffusion(G):
    nx, ny, nz, dx, dy, nu = _args(G)
    u, v, w, dz_f, dz_c = G["u"], G["v"], G["w"], G["dz_f"], G["dz_c"]
    assert rel(ops.advection_u(u, v, w, nx, ny, nz, dx, dy, dz_f), G["adv_u"]) < 1e-13
    assert rel(ops.advection_v(u, v, w, nx, ny, nz, dx, dy, dz_f), G["adv_v"]) < 1e-13
    assert rel(ops.advection_w(u, v, w, nx, ny, nz, dx, dy, dz_c), G["adv_w"]) < 1e-13
    assert rel(ops.diffusion_xy_u(u, nx, ny, nz, dx, dy, nu), G["dxy_u"]) < 1e-13
    assert rel(ops.diffusion_xy_v(v, nx, ny, nz, dx, dy, nu), G["dxy_v"]) < 1e-13
    assert rel(ops.diffusion_xy_w(w, nx, ny, nz, dx, dy, nu), G["dxy_w"]) < 1e-13
    assert rel(ops.diffusion_u(u, nx, ny, nz, dx, dy, dz_c, dz_f, nu), G["dif_u"]) < 1e-13
    assert rel(ops.diffusion_v(v, nx, ny, nz, dx, dy, dz_c, dz_f, nu), G["dif_v"]) < 1e-13
    assert rel(ops.diffusion_w(w, nx, ny, nz, dx, dy, dz_c, dz_f, nu), G["dif_w"]) < 1e-13


@pytest.mark.parametrize("name,f", [("imex", ops.rhs_imex_fused), ("v2", ops.rhs_full_fused)])
def test_fused_paths(G, name, f):
    nx, ny, nz, dx, dy, nu = _args(G)
    r = f(G["u"], G["v"], G["w"], nx, ny, nz, dx, dy, G["dz_c"], G["dz_f"], nu)
    for c, a in zip("uvw", r):
        assert rel(a, G[f"fused_{name}_{c}"]) < 1e-12, c


def test_separate_vs_fused_quirk(G):
    """The CPU path adds x/y diffusion on u[nx] and v[:, ny]; the CUDA path does not."""
    nx, ny, nz, dx, dy, nu = _args(G)
    a = ops.rhs_imex_separate(G["u"], G["v"], G["w"], nx, ny, nz, dx, dy, G["dz_c"], G["dz_f"], nu)
    assert np.max(np.abs(a[0][nx] - G["fused_imex_u"][nx])) > 1e-6
    assert rel(a[0][:nx], G["fused_imex_u"][:nx]) < 1e-12
    assert rel(a[2], G["fused_imex_w"]) < 1e-12


def test_pcr(G):
    x = ops.pcr_solve(G["pcr_a"], G["pcr_b"], G["pcr_c"], G["pcr_d"])
    assert rel(x, G["pcr_x"]) < 1e-14


@pytest.mark.parametrize("top", ["dirichlet", "neumann"])
def test_cn(G, top):
    nx, ny, nz, dx, dy, nu = _args(G)
    dz_c, dz_f = G["dz_c"], G["dz_f"]
    assert rel(ops.solve_implicit_diffusion_uv(G["u"], 0.002, nx, ny, nz, dz_c, dz_f, nu,
                                               top_wall_bc_type=top), G[f"cn_{top}_u"]) < 1e-14
    assert rel(ops.solve_implicit_diffusion_uv(G["v"], 0.002, nx, ny, nz, dz_c, dz_f, nu,
                                               top_wall_bc_type=top), G[f"cn_{top}_v"]) < 1e-14
    assert rel(ops.solve_implicit_diffusion_w(G["w"], 0.002, nx, ny, nz, dz_c, dz_f, nu), G["cn_w"]) < 1e-14


def test_div_proj_bulk_utau_cfl(G):
    nx, ny, nz, dx, dy, nu = _args(G)
    u, v, w, dz_f, dz_c = G["u"], G["v"], G["w"], G["dz_f"], G["dz_c"]
    assert rel(ops.compute_divergence(u, v, w, nx, ny, nz, dx, dy, dz_f), G["div"]) < 1e-13
    pu, pv, pw = ops.project_velocity(u.copy(), v.copy(), w.copy(), G["proj_p"], nx, ny, nz,
                                      dx, dy, dz_c, dz_f, 0.002)
    assert rel(pu, G["proj_u"]) < 1e-15 and rel(pv, G["proj_v"]) < 1e-15 and rel(pw, G["proj_w"]) < 1e-15
    vol = float(G["Lx"]) * float(G["Ly"]) * float(G["Lz"])
    assert abs(ops.compute_bulk_velocity(u, nx, ny, nz, dx, dy, dz_f, vol) - G["bulk"]) < 1e-14
    zc = G["z_c"]
    assert abs(ops.compute_u_tau(u, zc, nu) - G["u_tau_dirichlet"]) < 1e-15
    assert abs(ops.compute_u_tau(u, zc, nu, "neumann") - G["u_tau_neumann"]) < 1e-15
    dti = ops.compute_cfl_inverse(u, v, w, nx, ny, nz, dx, dy, dz_f, dz_c)
    assert abs(dti - G["cfl_dti"]) / G["cfl_dti"] < 1e-14


def test_poisson(G):
    nx, ny, nz, dx, dy, nu = _args(G)
    fd = poisson.initialize_fft_solver(nx, ny, nz, dx, dy, G["dz_c"], G["dz_f"])
    for k in ("tri_a", "tri_b", "tri_c"):
        assert rel(fd[k], G[k]) < 1e-14
    p = poisson.solve_poisson_fft(G["poisson_rhs"], fd)
    ref = G["poisson_p"]
    # the (0,0) mode is singular: compare modulo the interior mean
    pi = p[1:-1, 1:-1, 1:-1] - p[1:-1, 1:-1, 1:-1].mean()
    ri = ref[1:-1, 1:-1, 1:-1] - ref[1:-1, 1:-1, 1:-1].mean()
    assert rel(pi, ri) < 1e-10
    res = poisson.poisson_residual(p, G["poisson_rhs"], nx, ny, nz, dx, dy, G["dz_c"], G["dz_f"])
    assert np.max(np.abs(res)) < 1e-9 * np.max(np.abs(G["poisson_rhs"])) * 1e3


def _oracle_from(S, **kw):
    nx, ny, nz = int(S["nx"]), int(S["ny"]), int(S["nz"])
    oc = OracleChannel(nx, ny, nz, float(S["Lx"]), float(S["Ly"]), float(S["Lz"]),
                       1.0 / float(S["nu"]), grid=(S["z_f"], S["z_c"], S["dz_f"], S["dz_c"]), **kw)
    oc.set_state(S["u0"], S["v0"], S["w0"], S["p0"])
    return oc


@pytest.mark.parametrize("name", ["step_imex_16x12x10.npz", "step_imex_32x24x16.npz",
                                  "step_imex_neumann_16x12x10.npz"])
def test_step_imex(golden, name):
    S = golden(name)
    oc = _oracle_from(S, top_wall_bc_type=str(S["top"]))
    dt = float(S["dt"])
    s = 1
    while f"u{s}" in S:
        ub, f = oc.step_imex(dt)
        for c, a in (("u", oc.u), ("v", oc.v), ("w", oc.w)):
            assert rel(a, S[f"{c}{s}"]) < 1e-12, (name, s, c, rel(a, S[f"{c}{s}"]))
        pr = S[f"p{s}"][1:-1, 1:-1, 1:-1]
        po = oc.p[1:-1, 1:-1, 1:-1]
        assert rel(po - po.mean(), pr - pr.mean()) < 1e-9
        assert abs(ub - S[f"ubulk{s}"]) < 1e-13
        assert abs(f - S[f"forcing{s}"]) < 1e-9 * max(1.0, abs(S[f"forcing{s}"]))
        s += 1
    assert s > 2


def test_step_fe(golden):
    S = golden("step_fe_16x12x10.npz")
    G = golden("step_imex_16x12x10.npz")   # same grid and domain
    nx, ny, nz = int(S["nx"]), int(S["ny"]), int(S["nz"])
    oc = OracleChannel(nx, ny, nz, float(G["Lx"]), float(G["Ly"]), float(G["Lz"]),
                       1.0 / float(G["nu"]), grid=(G["z_f"], G["z_c"], G["dz_f"], G["dz_c"]))
    oc.set_state(S["u0"], S["v0"], S["w0"])
    oc.step_fe(float(S["dt"]))
    for c, a in (("u", oc.u), ("v", oc.v), ("w", oc.w)):
        assert rel(a, S[f"{c}1"]) < 1e-12


def test_stats(golden):
    S = golden("stats_16x12x10.npz")
    G = golden("step_imex_16x12x10.npz")
    nx, ny, nz = int(S["nx"]), int(S["ny"]), int(S["nz"])
    ts = ostats.TurbulenceStats(nx, ny, nz, float(G["Lx"]), float(G["Ly"]), float(G["Lz"]),
                                G["z_c"], float(G["Lx"]) / nx, float(G["Ly"]) / ny,
                                float(G["nu"]), 180.0, 15.0)
    assert (ts.k_bot, ts.k_top) == (int(S["k_bot"]), int(S["k_top"]))
    for s in range(2):
        ts.accumulate_statistics(S[f"u{s}"], S[f"v{s}"], S[f"w{s}"])
    for k in ("U_sum", "uu_sum", "vv_sum", "ww_sum", "uw_sum",
              "E_uu_2d_sum", "E_vv_2d_sum", "E_ww_2d_sum", "E_uw_2d_sum"):
        assert rel(getattr(ts, k), S[k]) < 1e-12, k
