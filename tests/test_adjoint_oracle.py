"""The reference-autograd adjoint golden vectors (tests/golden/
make_adjoint_golden.py) against the CPU oracle's forward operators, and the
identity the projection adjoint is built on.  No GPU."""
import numpy as np
import pytest

from oracle import ops, poisson


def _ghost(ud, vd, wd, nx, ny, nz, top):
    u = np.zeros((nx + 1, ny + 2, nz + 2)); v = np.zeros((nx + 2, ny + 1, nz + 2))
    w = np.zeros((nx + 2, ny + 2, nz + 1))
    u[1:nx + 1, 1:ny + 1, 1:nz + 1] = ud
    v[1:nx + 1, 1:ny + 1, 1:nz + 1] = vd
    w[1:nx + 1, 1:ny + 1, 1:nz] = wd
    ops.apply_bc_all(u, v, w, top)
    return u, v, w


@pytest.fixture(scope="module")
def G(golden):
    return golden("adjoint_16x12x10.npz")


def _dims(G):
    return int(G["nx"]), int(G["ny"]), int(G["nz"])


def test_rhs_vjp_matches_oracle_jvp(G):
    """lam . (J d) = (J^T lam) . d with J d by central differences of the
    oracle's (quadratic) right-hand side, exact up to rounding."""
    nx, ny, nz = _dims(G)
    dx, dy = float(G["Lx"]) / nx, float(G["Ly"]) / ny
    dz_f, dz_c, nu = G["dz_f"], G["dz_c"], float(G["nu"])
    q = (G["u"], G["v"], G["w"])

    def R(qu, qv, qw):
        u, v, w = _ghost(qu, qv, qw, nx, ny, nz, "dirichlet")
        ru, rv, rw = ops.rhs_imex_separate(u, v, w, nx, ny, nz, dx, dy, dz_c, dz_f, nu)
        return ru[1:nx + 1, 1:ny + 1, 1:nz + 1], rv[1:nx + 1, 1:ny + 1, 1:nz + 1], rw[1:nx + 1, 1:ny + 1, 1:nz]

    r0 = R(*q)
    for a, b in zip(r0, (G["rhs_ru"], G["rhs_rv"], G["rhs_rw"])):
        assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b))
    rng = np.random.default_rng(3)
    for _ in range(3):
        d = [rng.standard_normal(x.shape) for x in q]
        eps = 1e-3
        rp = R(*[x + eps * y for x, y in zip(q, d)])
        rm = R(*[x - eps * y for x, y in zip(q, d)])
        jd = [(p - m) / (2 * eps) for p, m in zip(rp, rm)]
        lhs = sum(np.sum(l * j) for l, j in zip((G["rhs_lu"], G["rhs_lv"], G["rhs_lw"]), jd))
        rhs = sum(np.sum(g * y) for g, y in zip((G["rhs_gu"], G["rhs_gv"], G["rhs_gw"]), d))
        assert abs(lhs - rhs) <= 1e-10 * abs(rhs), (lhs, rhs)


@pytest.mark.parametrize("top", ["dirichlet", "neumann"])
def test_cn_vjp_matches_oracle(G, top):
    nx, ny, nz = _dims(G)
    dz_f, dz_c, nu, dt = G["dz_f"], G["dz_c"], float(G["nu"]), float(G["cn_dt"])
    t = "cn_" + top + "_"

    def CN(qu, qv, qw):
        u, v, w = _ghost(qu, qv, qw, nx, ny, nz, top)
        un = ops.solve_implicit_diffusion_uv(u, dt, nx, ny, nz, dz_c, dz_f, nu, top_wall_bc_type=top)
        vn = ops.solve_implicit_diffusion_uv(v, dt, nx, ny, nz, dz_c, dz_f, nu, top_wall_bc_type=top)
        wn = ops.solve_implicit_diffusion_w(w, dt, nx, ny, nz, dz_c, dz_f, nu)
        return un[1:nx + 1, 1:ny + 1, 1:nz + 1], vn[1:nx + 1, 1:ny + 1, 1:nz + 1], wn[1:nx + 1, 1:ny + 1, 1:nz]

    o = CN(G["u"], G["v"], G["w"])
    for a, name in zip(o, "uvw"):
        b = G[t + "o" + name]
        assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(b)), name
    rng = np.random.default_rng(4)
    d = [rng.standard_normal(x.shape) for x in o]
    jd = CN(*d)  # linear map
    lhs = sum(np.sum(G[t + "l" + n] * j) for n, j in zip("uvw", jd))
    rhs = sum(np.sum(G[t + "g" + n] * y) for n, y in zip("uvw", d))
    assert abs(lhs - rhs) <= 1e-11 * abs(rhs)


def test_bulk_gradient(G):
    nx, ny, nz = _dims(G)
    dx, dy = float(G["Lx"]) / nx, float(G["Ly"]) / ny
    V = float(G["Lx"]) * float(G["Ly"]) * float(G["Lz"])
    want = np.broadcast_to(dx * dy * G["dz_f"][None, None, :] / V, (nx, ny, nz))
    assert np.max(np.abs(G["bulk_gu"] - want)) <= 1e-15 * np.max(want)


def test_projection_is_self_adjoint_in_volume_weights():
    """<D q, phi>_Wp = -<q, G phi>_Wq (W = cell / face volumes) for the
    oracle's divergence (utils.py:226-240) and projection gradient
    (projection.py:143-165), and hence P^T = W P W^-1 for P = I - G L^-1 D:
    the identity the CUDA projection adjoint applies."""
    from oracle.grid import generate_grid
    nx, ny, nz = 16, 12, 10
    Lx, Ly, Lz = 4 * np.pi, 4 * np.pi / 3, 2.0
    dx, dy = Lx / nx, Ly / ny
    _, _, dz_f, dz_c = generate_grid(2.6, nz, Lz)
    rng = np.random.default_rng(5)
    qd = (rng.standard_normal((nx, ny, nz)), rng.standard_normal((nx, ny, nz)),
          rng.standard_normal((nx, ny, nz - 1)))
    u, v, w = _ghost(*qd, nx, ny, nz, "dirichlet")
    phi = np.zeros((nx + 2, ny + 2, nz + 2))
    phi[1:nx + 1, 1:ny + 1, 1:nz + 1] = rng.standard_normal((nx, ny, nz))
    phi[0] = phi[nx]; phi[nx + 1] = phi[1]; phi[:, 0] = phi[:, ny]; phi[:, ny + 1] = phi[:, 1]
    phi[:, :, 0] = phi[:, :, 1]; phi[:, :, nz + 1] = phi[:, :, nz]
    div = ops.compute_divergence(u, v, w, nx, ny, nz, dx, dy, dz_f)
    lhs = np.sum(div * phi[1:nx + 1, 1:ny + 1, 1:nz + 1] * dz_f[None, None, :])
    g = [a.copy() for a in (u, v, w)]
    zero = [np.zeros_like(a) for a in g]
    ops.project_velocity(*zero, phi, nx, ny, nz, dx, dy, dz_c, dz_f, 1.0)  # zero - grad phi
    gu, gv, gw = (-zero[0][1:nx + 1, 1:ny + 1, 1:nz + 1], -zero[1][1:nx + 1, 1:ny + 1, 1:nz + 1],
                  -zero[2][1:nx + 1, 1:ny + 1, 1:nz])
    rhs = -(np.sum(qd[0] * gu * dz_f) + np.sum(qd[1] * gv * dz_f) + np.sum(qd[2] * gw * dz_c[1:nz]))
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), 1.0)
    # P^T = W P W^-1 on the whole projection (FFT Poisson, gauged)
    fd = poisson.initialize_fft_solver(nx, ny, nz, dx, dy, dz_c, dz_f)

    def P(qu, qv, qw):
        a, b, c = _ghost(qu, qv, qw, nx, ny, nz, "dirichlet")
        p = poisson.solve_poisson_fft(ops.compute_divergence(a, b, c, nx, ny, nz, dx, dy, dz_f), fd)
        ops.project_velocity(a, b, c, p, nx, ny, nz, dx, dy, dz_c, dz_f, 1.0)
        return a[1:nx + 1, 1:ny + 1, 1:nz + 1], b[1:nx + 1, 1:ny + 1, 1:nz + 1], c[1:nx + 1, 1:ny + 1, 1:nz]

    W = (dz_f[None, None, :], dz_f[None, None, :], dz_c[None, None, 1:nz])
    x = [rng.standard_normal(t.shape) for t in qd]
    y = [rng.standard_normal(t.shape) for t in qd]
    Px = P(*x)
    PTy = [wt * t for wt, t in zip(W, P(*[t / wt for wt, t in zip(W, y)]))]
    lhs = sum(np.sum(a * b) for a, b in zip(y, Px))
    rhs = sum(np.sum(a * b) for a, b in zip(PTy, x))
    assert abs(lhs - rhs) <= 1e-11 * abs(lhs)
