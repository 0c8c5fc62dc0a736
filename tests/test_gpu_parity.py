"""Parity of the CUDA path (through the C ABI) with the CPU oracle and the
reference's golden vectors.  FP64 plain form: <= 1e-12 relative per step."""
import numpy as np
import pytest

from oracle import ops, poisson
from oracle.stats import TurbulenceStats
from tests._util import dof, make_gpu, make_oracle, np_, rel

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _bc_random(oc, seed, top):
    rng = np.random.default_rng(seed)
    nx, ny, nz = oc.nx, oc.ny, oc.nz
    u = 1.0 + 0.1 * rng.standard_normal((nx + 1, ny + 2, nz + 2))
    v = 0.1 * rng.standard_normal((nx + 2, ny + 1, nz + 2))
    w = 0.1 * rng.standard_normal((nx + 2, ny + 2, nz + 1))
    ops.apply_bc_all(u, v, w, top)
    return u, v, w


SIZES = [(16, 12, 10), (24, 36, 20), (48, 32, 24)]


@pytest.mark.parametrize("nx,ny,nz", SIZES)
@pytest.mark.parametrize("path", ["separate", "fused"])
@pytest.mark.parametrize("full", [False, True])
@pytest.mark.parametrize("top", ["dirichlet", "neumann"])
def test_explicit_rhs(torch_cuda, nx, ny, nz, path, full, top):
    oc = make_oracle(nx, ny, nz, top=top, rhs_path=path)
    u, v, w = _bc_random(oc, 3, top)
    oc.set_state(u, v, w)
    ref = oc.explicit_rhs_full() if full else oc.explicit_rhs_imex()
    ch = make_gpu(oc)
    ch.set_state(u, v, w)
    got = ch.explicit_rhs(full=full)
    for name, g, r in zip("uvw", got, ref):
        assert rel(dof(name, np_(g), nx, ny, nz), dof(name, r, nx, ny, nz)) < TOL, name


# nz past one 32-row chunk of the CN solve: ragged last chunks (70, 33 -> w has
# 32 rows), 8 chunks (256) and the deep-channel form (300, 512 rows)
CN_SIZES = SIZES + [(16, 12, 70), (8, 16, 33), (8, 8, 256), (8, 8, 300), (8, 8, 512)]


@pytest.mark.parametrize("nx,ny,nz", CN_SIZES)
@pytest.mark.parametrize("top", ["dirichlet", "neumann"])
def test_implicit_diffusion(torch_cuda, nx, ny, nz, top):
    oc = make_oracle(nx, ny, nz, top=top)
    u, v, w = _bc_random(oc, 4, top)
    dt = 0.002
    ru = ops.solve_implicit_diffusion_uv(u, dt, nx, ny, nz, oc.dz_c, oc.dz_f, oc.nu, top_wall_bc_type=top)
    rv = ops.solve_implicit_diffusion_uv(v, dt, nx, ny, nz, oc.dz_c, oc.dz_f, oc.nu, top_wall_bc_type=top)
    rw = ops.solve_implicit_diffusion_w(w, dt, nx, ny, nz, oc.dz_c, oc.dz_f, oc.nu)
    ch = make_gpu(oc)
    ch.set_state(u, v, w)
    ch.implicit_diffusion(dt)
    gu, gv, gw, _ = ch.get_state()
    for name, g, r in zip("uvw", (gu, gv, gw), (ru, rv, rw)):
        assert rel(dof(name, np_(g), nx, ny, nz), dof(name, r, nx, ny, nz)) < TOL, name


REG_Y = (64, 96, 128, 144, 192, 256)   # y lengths of the streamed y / z passes


def _fused(ch, fused, nz):
    """Select the Poisson middle (0 three kernels, 1 fused cluster kernel, 2
    streamed y / z passes); the fused cluster kernel must be available for
    portable cluster sizes (nz <= 128: at most 8 CTAs of 16 planes) and y
    rows of at most 384 points (it holds whole rows of its planes in shared
    memory), the streamed passes for register y lengths up to 256."""
    try:
        ch.use_fused_poisson(fused)
    except Exception:
        if fused == 1 and nz <= 128 and ch.ny <= 384:
            raise
        if fused == 2 and ch.ny in REG_Y:
            raise
        pytest.skip("Poisson middle not available for this shape")


# (32,24,128): 8 CTAs of 16 planes; (16,12,100): 8 CTAs, ragged last chunk;
# (16,12,200): 16-CTA cluster
POISSON_SIZES = SIZES + [(64, 64, 48), (96, 48, 32), (32, 24, 128), (16, 12, 100), (16, 12, 200),
                         (768, 32, 8), (32, 768, 8), (512, 48, 6), (48, 512, 6),  # 768 = 24 x 32, 512 = 32 x 16
                         (144, 288, 6), (1024, 16, 4), (16, 576, 4)]               # 9 x 16, 18 x 16, 32 x 32, 18 x 32


@pytest.mark.parametrize("nx,ny,nz", POISSON_SIZES)
@pytest.mark.parametrize("fused", [0, 1, 2])
def test_poisson(torch_cuda, nx, ny, nz, fused):
    oc = make_oracle(nx, ny, nz)
    rng = np.random.default_rng(1)
    rhs = rng.random((nx, ny, nz)) - 0.5
    rhs -= np.sum(rhs * oc.dz_f) / (nx * ny * oc.Lz)     # dz_f-weighted zero mean
    ref = poisson.solve_poisson_fft(rhs, oc.fd)
    ch = make_gpu(oc)
    _fused(ch, fused, nz)
    p = np_(ch.poisson_solve(rhs))
    assert rel(dof("p", p, nx, ny, nz), dof("p", ref, nx, ny, nz)) < 1e-11
    res = poisson.poisson_residual(p, rhs, nx, ny, nz, oc.dx, oc.dy, oc.dz_c, oc.dz_f)
    assert np.max(np.abs(res)) < 1e-8 * np.max(np.abs(rhs)) * np.max(1 / oc.dz_f) ** 2 * 1e-3
    # ghosts: periodic in x/y, Neumann in z
    assert np.array_equal(p[0], p[nx]) and np.array_equal(p[nx + 1], p[1])
    assert np.array_equal(p[:, :, 0], p[:, :, 1]) and np.array_equal(p[:, :, nz + 1], p[:, :, nz])


@pytest.mark.parametrize("nx,ny,nz", SIZES)
def test_projection_divergence_reductions(torch_cuda, nx, ny, nz):
    oc = make_oracle(nx, ny, nz)
    u, v, w = _bc_random(oc, 5, "dirichlet")
    ch = make_gpu(oc)
    ch.set_state(u, v, w)
    div = np_(ch.divergence())
    assert rel(div, ops.compute_divergence(u, v, w, nx, ny, nz, oc.dx, oc.dy, oc.dz_f)) < TOL
    assert abs(ch.bulk_velocity() - oc.bulk(u)) < 1e-14
    dti = ch.cfl_inverse()
    ref = ops.compute_cfl_inverse(u, v, w, nx, ny, nz, oc.dx, oc.dy, oc.dz_f, oc.dz_c)
    assert abs(dti - ref) / ref < 1e-14
    d = ch.diagnostics()
    assert abs(d["u_tau"] - ops.compute_u_tau(u, oc.z_c, oc.nu)) < 1e-14
    rng = np.random.default_rng(6)
    p = rng.standard_normal((nx + 2, ny + 2, nz + 2))
    # the projection reads p through its periodic / Neumann ghosts
    p[0] = p[nx]; p[nx + 1] = p[1]; p[:, 0] = p[:, ny]; p[:, ny + 1] = p[:, 1]
    p[:, :, 0] = p[:, :, 1]; p[:, :, nz + 1] = p[:, :, nz]
    ch.project(p, 0.002)
    gu, gv, gw, _ = ch.get_state()
    ru, rv, rw = ops.project_velocity(u.copy(), v.copy(), w.copy(), p, nx, ny, nz, oc.dx, oc.dy, oc.dz_c,
                                      oc.dz_f, 0.002)
    for name, g, r in zip("uvw", (gu, gv, gw), (ru, rv, rw)):
        assert rel(dof(name, np_(g), nx, ny, nz), dof(name, r, nx, ny, nz)) < TOL, name


def test_state_roundtrip_ghosts(torch_cuda):
    nx, ny, nz = 16, 12, 10
    for top in ("dirichlet", "neumann"):
        oc = make_oracle(nx, ny, nz, top=top)
        u, v, w = _bc_random(oc, 7, top)
        ch = make_gpu(oc)
        ch.set_state(u, v, w)
        gu, gv, gw, _ = ch.get_state()
        assert np.array_equal(np_(gu), u) and np.array_equal(np_(gv), v) and np.array_equal(np_(gw), w)


def test_initial_projection(torch_cuda):
    nx, ny, nz = 32, 24, 16
    oc = make_oracle(nx, ny, nz)                 # fresh start, already projected
    from oracle.step import initial_fields
    u, v, w, _ = initial_fields(nx, ny, nz, oc.z_c, oc.Lz, seed=0)
    ch = make_gpu(oc)
    ch.set_state(u, v, w)
    ub = ch.bulk_velocity()
    u = u * (1.0 / ub)
    ch.set_state(u, v, w)
    ch.project_initial()
    gu, gv, gw, gp = ch.get_state()
    for name, g, r in zip("uvwp", (gu, gv, gw, gp), (oc.u, oc.v, oc.w, oc.p)):
        assert rel(dof(name, np_(g), nx, ny, nz), dof(name, r, nx, ny, nz)) < 1e-11, name
    assert ch.diagnostics()["max_div"] < 1e-12


@pytest.mark.parametrize("name", ["step_imex_16x12x10.npz", "step_imex_32x24x16.npz",
                                  "step_imex_neumann_16x12x10.npz"])
def test_steps_vs_reference_golden(torch_cuda, golden, name):
    from torchannel_b200.core import Channel
    S = golden(name)
    nx, ny, nz = int(S["nx"]), int(S["ny"]), int(S["nz"])
    ch = Channel(nx, ny, nz, float(S["Lx"]), float(S["Ly"]), float(S["Lz"]), float(S["nu"]),
                 S["dz_f"], S["dz_c"], U_bulk=float(S["U_bulk"]), top_wall_bc_type=str(S["top"]))
    ch.set_state(S["u0"], S["v0"], S["w0"])
    dt = float(S["dt"])
    s = 1
    while f"u{s}" in S:
        ch.step("IMEX", dt)
        gu, gv, gw, gp = ch.get_state()
        for c, g in (("u", gu), ("v", gv), ("w", gw)):
            assert rel(np_(g), S[f"{c}{s}"]) < TOL, (s, c)
        assert rel(dof("p", np_(gp), nx, ny, nz), dof("p", S[f"p{s}"], nx, ny, nz)) < 1e-9
        sc = np_(ch.scalars)
        assert abs(sc[1] - S[f"ubulk{s}"]) < 1e-13
        assert abs(sc[0] - S[f"forcing{s}"]) < 1e-9 * max(1.0, abs(S[f"forcing{s}"]))
        s += 1


def test_fe_vs_reference_golden(torch_cuda, golden):
    from torchannel_b200.core import Channel
    S = golden("step_fe_16x12x10.npz")
    G = golden("step_imex_16x12x10.npz")
    nx, ny, nz = int(S["nx"]), int(S["ny"]), int(S["nz"])
    ch = Channel(nx, ny, nz, float(G["Lx"]), float(G["Ly"]), float(G["Lz"]), float(G["nu"]), G["dz_f"], G["dz_c"])
    ch.set_state(S["u0"], S["v0"], S["w0"])
    ch.step("FE", float(S["dt"]))
    gu, gv, gw, _ = ch.get_state()
    for c, g in (("u", gu), ("v", gv), ("w", gw)):
        assert rel(np_(g), S[f"{c}1"]) < TOL, c


@pytest.mark.parametrize("scheme", ["IMEX", "AB2", "FE"])
@pytest.mark.parametrize("path", ["separate", "fused"])
@pytest.mark.parametrize("top", ["dirichlet", "neumann"])
@pytest.mark.parametrize("nx,ny,nz", [(24, 36, 20), (64, 64, 40)])
def test_steps_vs_oracle(torch_cuda, scheme, path, top, nx, ny, nz):
    """(64, 64, 40) takes the register-resident x and y transforms and the
    chunked z solve (3 chunks of 16 levels, the last ragged)."""
    oc = make_oracle(nx, ny, nz, seed=11, top=top, rhs_path=path)
    ch = make_gpu(oc)
    ch.set_state(oc.u, oc.v, oc.w, forcing=0.0)
    dt = 0.002 if scheme == "IMEX" else 0.0005
    step = {"IMEX": oc.step_imex, "AB2": oc.step_ab2, "FE": oc.step_fe}[scheme]
    for s in range(4):
        ub, f = step(dt)
        ch.step(scheme, dt)
        gu, gv, gw, gp = ch.get_state()
        for name, g, r in zip("uvw", (gu, gv, gw), (oc.u, oc.v, oc.w)):
            assert rel(np_(g), r) < TOL, (s, name, rel(np_(g), r))
        sc = np_(ch.scalars)
        assert abs(sc[1] - ub) < 1e-13
        if scheme != "FE":
            assert abs(sc[0] - f) < 1e-9 * max(1.0, abs(f))
        assert ch.diagnostics()["max_div"] < 1e-12


@pytest.mark.parametrize("nx,ny,nz", [(768, 32, 8), (32, 768, 8), (512, 48, 6), (48, 512, 6),
                                      (144, 288, 6), (288, 144, 6), (1024, 16, 4), (16, 1024, 4), (576, 32, 4),
                                      (32, 576, 4)])
def test_steps_vs_oracle_long_rows(torch_cuda, nx, ny, nz):
    """Register transforms of every supported split beyond 384 points (512 =
    32 x 16, 576 = 18 x 32, 768 = 24 x 32, 1024 = 32 x 32) and of the odd
    radix-3 lengths 144 = 9 x 16 and 288 = 18 x 16, in x and in y, through full
    IMEX steps."""
    oc = make_oracle(nx, ny, nz, seed=12)
    ch = make_gpu(oc)
    ch.set_state(oc.u, oc.v, oc.w, forcing=0.0)
    for s in range(3):
        ub, f = oc.step_imex(0.002)
        ch.step("IMEX", 0.002)
        gu, gv, gw, gp = ch.get_state()
        for name, g, r in zip("uvw", (gu, gv, gw), (oc.u, oc.v, oc.w)):
            assert rel(np_(g), r) < TOL, (s, name, rel(np_(g), r))
        assert ch.diagnostics()["max_div"] < 1e-12


def test_stats_vs_golden(torch_cuda, golden):
    from torchannel_b200.core import Channel
    S = golden("stats_16x12x10.npz")
    G = golden("step_imex_16x12x10.npz")
    nx, ny, nz = int(S["nx"]), int(S["ny"]), int(S["nz"])
    ch = Channel(nx, ny, nz, float(G["Lx"]), float(G["Ly"]), float(G["Lz"]), float(G["nu"]), G["dz_f"], G["dz_c"])
    kb, kt = ch.stats_init(G["z_c"], 180.0, 15.0)
    assert (kb, kt) == (int(S["k_bot"]), int(S["k_top"]))
    for s in range(2):
        ch.set_state(S[f"u{s}"], S[f"v{s}"], S[f"w{s}"])
        ch.stats_accumulate()
    got = ch.stats_read()
    assert got["n_samples"] == 2
    for k in ("U_sum", "uu_sum", "vv_sum", "ww_sum", "uw_sum",
              "E_uu_2d_sum", "E_vv_2d_sum", "E_ww_2d_sum", "E_uw_2d_sum"):
        assert rel(got[k], S[k]) < 1e-12, k


@pytest.mark.parametrize("nx,ny,nz", [(32, 24, 16), (48, 96, 24)])
def test_stats_vs_oracle(torch_cuda, nx, ny, nz):
    oc = make_oracle(nx, ny, nz, seed=2)
    ch = make_gpu(oc)
    ts = TurbulenceStats(nx, ny, nz, oc.Lx, oc.Ly, oc.Lz, oc.z_c, oc.dx, oc.dy, oc.nu, 180.0, 15.0)
    ch.stats_init(oc.z_c, 180.0, 15.0)
    assert (ch.k_bot, ch.k_top) == (ts.k_bot, ts.k_top)
    ch.set_state(oc.u, oc.v, oc.w)
    for s in range(3):
        oc.step_imex(0.002)
        ch.step("IMEX", 0.002)
        ts.accumulate_statistics(oc.u, oc.v, oc.w)
        ch.stats_accumulate()
    got = ch.stats_read()
    for k in ("U_sum", "uu_sum", "vv_sum", "ww_sum", "uw_sum",
              "E_uu_2d_sum", "E_vv_2d_sum", "E_ww_2d_sum", "E_uw_2d_sum"):
        assert rel(got[k], getattr(ts, k)) < 1e-11, k


def test_history_roundtrip(torch_cuda):
    """Saving and restoring the AB2 history gives a bit-continuous restart."""
    nx, ny, nz = 24, 36, 20
    oc = make_oracle(nx, ny, nz, seed=12)
    a = make_gpu(oc)
    a.set_state(oc.u, oc.v, oc.w)
    a.step("IMEX", 0.002, 3)
    u, v, w, _ = a.get_state()
    hist = a.get_history()
    f = float(np_(a.scalars)[0])
    b = make_gpu(oc)
    b.set_state(u, v, w, forcing=f)
    b.set_history(*hist)
    a.step("IMEX", 0.002, 2)
    b.step("IMEX", 0.002, 2)
    for x, y in zip(a.get_state()[:3], b.get_state()[:3]):
        assert np.array_equal(np_(x), np_(y))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_graph_replay_is_bitwise_identical(torch_cuda, precision):
    nx, ny, nz = 32, 24, 16
    oc = make_oracle(nx, ny, nz, seed=13)
    a, b = make_gpu(oc, precision), make_gpu(oc, precision)
    a.use_graphs(False)
    for ch in (a, b):
        ch.set_state(oc.u, oc.v, oc.w)
        ch.step("IMEX", 0.003, 9)      # 1 plain + graph pairs + remainder
        ch.step("IMEX", 0.002, 6)      # dt change: new tables, new graph
        ch.step("AB2", 0.0005, 5)
    for x, y in zip(a.get_state(), b.get_state()):
        assert np.array_equal(np_(x), np_(y))
    assert np.array_equal(np_(a.scalars), np_(b.scalars))


@pytest.mark.parametrize("nx,ny,nz", [(192, 192, 128), (384, 384, 256)])
@pytest.mark.parametrize("fused", [0, 1, 2])
def test_poisson_full_size_residual(torch_cuda, nx, ny, nz, fused):
    """Full-size Poisson microbench grids: the discrete residual of the
    returned p (size-independent property; FP64 roundoff scale)."""
    from oracle.grid import generate_grid
    from torchannel_b200.core import Channel
    Lx, Ly, Lz = 4 * np.pi, 4 * np.pi / 3, 2.0
    z_f, z_c, dz_f, dz_c = generate_grid(2.6, nz, Lz)
    rng = np.random.default_rng(1)
    rhs = rng.random((nx, ny, nz)) - 0.5
    rhs -= np.sum(rhs * dz_f) / (nx * ny * Lz)
    ch = Channel(nx, ny, nz, Lx, Ly, Lz, 1 / 2870.0, dz_f, dz_c)
    _fused(ch, fused, nz)
    p = np_(ch.poisson_solve(rhs))
    r = poisson.poisson_residual(p, rhs, nx, ny, nz, Lx / nx, Ly / ny, dz_c, dz_f)
    # the operator's largest coefficients are ~1/dz_min^2; roundoff relative to them
    scale = np.max(np.abs(p)) * np.max(1.0 / (dz_c[:-1] * dz_f))
    assert np.max(np.abs(r)) < 1e-12 * scale + 1e-9


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_fused_poisson_steps_match_three_kernel_path(torch_cuda, precision):
    """IMEX steps with the fused y/z Poisson kernel and with the three-kernel
    path: same state up to the rounding of the chunked sweep."""
    nx, ny, nz = 48, 32, 64
    oc = make_oracle(nx, ny, nz, seed=21)
    a, b = make_gpu(oc, precision), make_gpu(oc, precision)
    a.use_fused_poisson(True)
    b.use_fused_poisson(False)
    for ch in (a, b):
        ch.set_state(oc.u, oc.v, oc.w)
        ch.step("IMEX", 0.003, 8)
    for x, y in zip(a.get_state()[:3], b.get_state()[:3]):
        assert rel(np_(x), np_(y)) < (1e-12 if precision == "fp64" else 1e-6)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("nx,ny,nz,top", [(48, 64, 48, "dirichlet"), (32, 96, 13, "neumann"), (64, 128, 40, "dirichlet"),
                                          (16, 144, 17, "neumann"), (192, 192, 128, "dirichlet"),
                                          (32, 256, 33, "neumann")])
def test_streamed_poisson_passes_are_bitwise_identical(torch_cuda, precision, nx, ny, nz, top):
    """IMEX steps with the Poisson middle as two streaming passes (y transform
    + forward elimination, back substitution + inverse y transform; whole
    and partial groups of levels, the gauged (0,0) mode) and with the three
    kernels: the same arithmetic, identical states and scalars."""
    oc = make_oracle(nx, ny, nz, seed=33, top=top)
    a, b = make_gpu(oc, precision), make_gpu(oc, precision)
    a.use_fused_poisson(2)
    b.use_fused_poisson(0)
    for ch in (a, b):
        ch.set_state(oc.u, oc.v, oc.w)
        ch.step("IMEX", 0.003, 6)
    for x, y in zip(a.get_state(), b.get_state()):
        assert np.array_equal(np_(x), np_(y))
    assert np.array_equal(np_(a.scalars)[:2], np_(b.scalars)[:2])


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("scheme", ["IMEX", "AB2", "FE"])
@pytest.mark.parametrize("nx,ny,nz,top", [(64, 64, 48, "dirichlet"), (144, 36, 13, "neumann"), (96, 16, 4, "dirichlet"),
                                          (192, 24, 9, "neumann")])
def test_tma_rhs_is_bitwise_identical(torch_cuda, precision, scheme, nx, ny, nz, top):
    """The explicit-RHS kernel with tensor-copy staging, every tile shape
    (partial x / y / z tiles, periodic wraps at both ends, both z ghosts, base
    profile in mixed precision), against the kernel with per-thread staging:
    identical states."""
    oc = make_oracle(nx, ny, nz, seed=51, top=top)
    b = make_gpu(oc, precision)
    b.use_tma_rhs(False)
    dt = 0.002 if scheme == "IMEX" else 0.0004
    b.set_state(oc.u, oc.v, oc.w)
    b.step(scheme, dt, 7)
    ref = [np_(x) for x in b.get_state()[:3]]
    for mode in range(1, 7):
        a = make_gpu(oc, precision)
        a.use_tma_rhs(mode)
        a.set_state(oc.u, oc.v, oc.w)
        a.step(scheme, dt, 7)
        for x, y in zip(a.get_state()[:3], ref):
            assert np.array_equal(np_(x), y), mode
        assert np.array_equal(np_(a.scalars)[:2], np_(b.scalars)[:2]), mode
        assert a.error_word() == 0


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("nx,ny,nz", [(48, 64, 48), (32, 96, 13), (64, 128, 40), (16, 144, 17), (192, 192, 128),
                                      (32, 256, 33), (16, 288, 6), (48, 512, 6), (32, 768, 8)])
def test_bulk_staged_y_transforms_are_bitwise_identical(torch_cuda, precision, nx, ny, nz):
    """IMEX steps with the y transforms staged by bulk copies (partial last
    tiles, every register length class) and by per-lane loads: the same
    arithmetic, identical states and scalars."""
    oc = make_oracle(nx, ny, nz, seed=34)
    a, b = make_gpu(oc, precision), make_gpu(oc, precision)
    a.use_bulk_ffty(True)
    b.use_bulk_ffty(False)
    for ch in (a, b):
        ch.set_state(oc.u, oc.v, oc.w)
        ch.step("IMEX", 0.003, 5)
    for x, y in zip(a.get_state(), b.get_state()):
        assert np.array_equal(np_(x), np_(y))
    assert np.array_equal(np_(a.scalars)[:2], np_(b.scalars)[:2])
    assert a.error_word() == 0
