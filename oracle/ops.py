"""Staggered-grid operators (oracle restatement, test infrastructure only).

Each function restates one reference function in numpy FP64 on reference-layout
arrays (see the package docstring) and cites the file:line it follows.
"""
import numpy as np


# ---------------------------------------------------------------------------
# Boundary conditions
# ---------------------------------------------------------------------------
def apply_bc_all(u, v, w, top_wall_bc_type="dirichlet"):
    """Ghost fill in place; ``solver.py:23-79``."""
    neu = top_wall_bc_type == "neumann"
    u[0, :, :] = u[-1, :, :]                     # solver.py:45
    u[:, 0, :] = u[:, -2, :]                     # solver.py:47
    u[:, -1, :] = u[:, 1, :]                     # solver.py:48
    u[:, :, 0] = -u[:, :, 1]                     # solver.py:50
    u[:, :, -1] = u[:, :, -2] if neu else -u[:, :, -2]   # solver.py:51-54
    v[0, :, :] = v[-2, :, :]                     # solver.py:58
    v[-1, :, :] = v[1, :, :]                     # solver.py:59
    v[:, 0, :] = v[:, -1, :]                     # solver.py:61
    v[:, :, 0] = -v[:, :, 1]                     # solver.py:63
    v[:, :, -1] = v[:, :, -2] if neu else -v[:, :, -2]   # solver.py:64-67
    w[0, :, :] = w[-2, :, :]                     # solver.py:71
    w[-1, :, :] = w[1, :, :]                     # solver.py:72
    w[:, 0, :] = w[:, -2, :]                     # solver.py:74
    w[:, -1, :] = w[:, 1, :]                     # solver.py:75
    w[:, :, 0] = 0.0                             # solver.py:78
    w[:, :, -1] = 0.0                            # solver.py:79


# ---------------------------------------------------------------------------
# Advection (conservative central form)
# ---------------------------------------------------------------------------
def advection_u(u, v, w, nx, ny, nz, dx, dy, dz_f):
    """``operators.py:126-163``; writes ``[1:nx, 1:ny+1, 1:nz+1]``."""
    adv = np.zeros_like(u)
    ui = 0.5 * (u[1:nx, 1:ny+1, 1:nz+1] + u[2:nx+1, 1:ny+1, 1:nz+1])
    uu_r = ui * ui
    ui = 0.5 * (u[0:nx-1, 1:ny+1, 1:nz+1] + u[1:nx, 1:ny+1, 1:nz+1])
    uu_l = ui * ui
    duudx = (uu_r - uu_l) / dx
    vi = 0.5 * (v[1:nx, 1:ny+1, 1:nz+1] + v[2:nx+1, 1:ny+1, 1:nz+1])
    uy = 0.5 * (u[1:nx, 1:ny+1, 1:nz+1] + u[1:nx, 2:ny+2, 1:nz+1])
    vu_t = vi * uy
    vi = 0.5 * (v[1:nx, 0:ny, 1:nz+1] + v[2:nx+1, 0:ny, 1:nz+1])
    uy = 0.5 * (u[1:nx, 0:ny, 1:nz+1] + u[1:nx, 1:ny+1, 1:nz+1])
    vu_b = vi * uy
    dvudy = (vu_t - vu_b) / dy
    wi = 0.5 * (w[1:nx, 1:ny+1, 1:nz+1] + w[2:nx+1, 1:ny+1, 1:nz+1])
    uz = 0.5 * (u[1:nx, 1:ny+1, 1:nz+1] + u[1:nx, 1:ny+1, 2:nz+2])
    wu_t = wi * uz
    wi = 0.5 * (w[1:nx, 1:ny+1, 0:nz] + w[2:nx+1, 1:ny+1, 0:nz])
    uz = 0.5 * (u[1:nx, 1:ny+1, 0:nz] + u[1:nx, 1:ny+1, 1:nz+1])
    wu_b = wi * uz
    dwudz = (wu_t - wu_b) / dz_f[0:nz][None, None, :]
    adv[1:nx, 1:ny+1, 1:nz+1] = duudx + dvudy + dwudz
    return adv


def advection_v(u, v, w, nx, ny, nz, dx, dy, dz_f):
    """``operators.py:166-204``; writes ``[1:nx+1, 1:ny, 1:nz+1]``."""
    adv = np.zeros_like(v)
    ui = 0.5 * (u[1:nx+1, 1:ny, 1:nz+1] + u[1:nx+1, 2:ny+1, 1:nz+1])
    vx = 0.5 * (v[1:nx+1, 1:ny, 1:nz+1] + v[2:nx+2, 1:ny, 1:nz+1])
    uv_r = ui * vx
    ui = 0.5 * (u[0:nx, 1:ny, 1:nz+1] + u[0:nx, 2:ny+1, 1:nz+1])
    vx = 0.5 * (v[0:nx, 1:ny, 1:nz+1] + v[1:nx+1, 1:ny, 1:nz+1])
    uv_l = ui * vx
    duvdx = (uv_r - uv_l) / dx
    vi = 0.5 * (v[1:nx+1, 1:ny, 1:nz+1] + v[1:nx+1, 2:ny+1, 1:nz+1])
    vv_t = vi * vi
    vi = 0.5 * (v[1:nx+1, 0:ny-1, 1:nz+1] + v[1:nx+1, 1:ny, 1:nz+1])
    vv_b = vi * vi
    dvvdy = (vv_t - vv_b) / dy
    wi = 0.5 * (w[1:nx+1, 1:ny, 1:nz+1] + w[1:nx+1, 2:ny+1, 1:nz+1])
    vz = 0.5 * (v[1:nx+1, 1:ny, 1:nz+1] + v[1:nx+1, 1:ny, 2:nz+2])
    wv_t = wi * vz
    wi = 0.5 * (w[1:nx+1, 1:ny, 0:nz] + w[1:nx+1, 2:ny+1, 0:nz])
    vz = 0.5 * (v[1:nx+1, 1:ny, 0:nz] + v[1:nx+1, 1:ny, 1:nz+1])
    wv_b = wi * vz
    dwvdz = (wv_t - wv_b) / dz_f[0:nz][None, None, :]
    adv[1:nx+1, 1:ny, 1:nz+1] = duvdx + dvvdy + dwvdz
    return adv


def advection_w(u, v, w, nx, ny, nz, dx, dy, dz_c):
    """``operators.py:207-247``; writes ``[1:nx+1, 1:ny+1, 1:nz]``."""
    adv = np.zeros_like(w)
    ui = 0.5 * (u[1:nx+1, 1:ny+1, 1:nz] + u[1:nx+1, 1:ny+1, 2:nz+1])
    wx = 0.5 * (w[1:nx+1, 1:ny+1, 1:nz] + w[2:nx+2, 1:ny+1, 1:nz])
    uw_r = ui * wx
    ui = 0.5 * (u[0:nx, 1:ny+1, 1:nz] + u[0:nx, 1:ny+1, 2:nz+1])
    wx = 0.5 * (w[0:nx, 1:ny+1, 1:nz] + w[1:nx+1, 1:ny+1, 1:nz])
    uw_l = ui * wx
    duwdx = (uw_r - uw_l) / dx
    vi = 0.5 * (v[1:nx+1, 1:ny+1, 1:nz] + v[1:nx+1, 1:ny+1, 2:nz+1])
    wy = 0.5 * (w[1:nx+1, 1:ny+1, 1:nz] + w[1:nx+1, 2:ny+2, 1:nz])
    vw_t = vi * wy
    vi = 0.5 * (v[1:nx+1, 0:ny, 1:nz] + v[1:nx+1, 0:ny, 2:nz+1])
    wy = 0.5 * (w[1:nx+1, 0:ny, 1:nz] + w[1:nx+1, 1:ny+1, 1:nz])
    vw_b = vi * wy
    dvwdy = (vw_t - vw_b) / dy
    wi = 0.5 * (w[1:nx+1, 1:ny+1, 1:nz] + w[1:nx+1, 1:ny+1, 2:nz+1])
    ww_t = wi * wi
    wi = 0.5 * (w[1:nx+1, 1:ny+1, 0:nz-1] + w[1:nx+1, 1:ny+1, 1:nz])
    ww_b = wi * wi
    dwwdz = (ww_t - ww_b) / dz_c[1:nz][None, None, :]
    adv[1:nx+1, 1:ny+1, 1:nz] = duwdx + dvwdy + dwwdz
    return adv


# ---------------------------------------------------------------------------
# Diffusion
# ---------------------------------------------------------------------------
def _d2x_u(u, nx, ny, nz, dx):
    ue = np.concatenate([u, u[1:2]], axis=0)     # periodic extension, operators.py:27
    return (ue[2:nx+2, 1:ny+1, 1:nz+1] - 2 * ue[1:nx+1, 1:ny+1, 1:nz+1]
            + ue[0:nx, 1:ny+1, 1:nz+1]) / dx**2


def _d2y_v(v, nx, ny, nz, dy):
    ve = np.concatenate([v, v[:, 1:2]], axis=1)  # operators.py:71
    return (ve[1:nx+1, 2:ny+2, 1:nz+1] - 2 * ve[1:nx+1, 1:ny+1, 1:nz+1]
            + ve[1:nx+1, 0:ny, 1:nz+1]) / dy**2


def diffusion_xy_u(u, nx, ny, nz, dx, dy, nu):
    """``operators.py:474-497``; writes ``[1:nx+1, 1:ny+1, 1:nz+1]``."""
    d = np.zeros_like(u)
    d2y = (u[1:nx+1, 2:ny+2, 1:nz+1] - 2 * u[1:nx+1, 1:ny+1, 1:nz+1]
           + u[1:nx+1, 0:ny, 1:nz+1]) / dy**2
    d[1:nx+1, 1:ny+1, 1:nz+1] = nu * (_d2x_u(u, nx, ny, nz, dx) + d2y)
    return d


def diffusion_xy_v(v, nx, ny, nz, dx, dy, nu):
    """``operators.py:500-523``; writes ``[1:nx+1, 1:ny+1, 1:nz+1]``."""
    d = np.zeros_like(v)
    d2x = (v[2:nx+2, 1:ny+1, 1:nz+1] - 2 * v[1:nx+1, 1:ny+1, 1:nz+1]
           + v[0:nx, 1:ny+1, 1:nz+1]) / dx**2
    d[1:nx+1, 1:ny+1, 1:nz+1] = nu * (d2x + _d2y_v(v, nx, ny, nz, dy))
    return d


def diffusion_xy_w(w, nx, ny, nz, dx, dy, nu):
    """``operators.py:526-548``; writes ``[1:nx+1, 1:ny+1, 1:nz]``."""
    d = np.zeros_like(w)
    d2x = (w[2:nx+2, 1:ny+1, 1:nz] - 2 * w[1:nx+1, 1:ny+1, 1:nz]
           + w[0:nx, 1:ny+1, 1:nz]) / dx**2
    d2y = (w[1:nx+1, 2:ny+2, 1:nz] - 2 * w[1:nx+1, 1:ny+1, 1:nz]
           + w[1:nx+1, 0:ny, 1:nz]) / dy**2
    d[1:nx+1, 1:ny+1, 1:nz] = nu * (d2x + d2y)
    return d


def _d2z_cc(q, nx, ny, nz, dz_c, dz_f):
    """Cell-centred z second difference; ``operators.py:41-50``."""
    dl = dz_c[0:nz][None, None, :]
    dr = dz_c[1:nz+1][None, None, :]
    return ((q[1:nx+1, 1:ny+1, 2:nz+2] - q[1:nx+1, 1:ny+1, 1:nz+1]) / dr
            - (q[1:nx+1, 1:ny+1, 1:nz+1] - q[1:nx+1, 1:ny+1, 0:nz]) / dl) / dz_f[None, None, :]


def diffusion_u(u, nx, ny, nz, dx, dy, dz_c, dz_f, nu):
    """Full Laplacian of u; ``operators.py:18-52``."""
    d = np.zeros_like(u)
    d2y = (u[1:nx+1, 2:ny+2, 1:nz+1] - 2 * u[1:nx+1, 1:ny+1, 1:nz+1]
           + u[1:nx+1, 0:ny, 1:nz+1]) / dy**2
    d[1:nx+1, 1:ny+1, 1:nz+1] = nu * (_d2x_u(u, nx, ny, nz, dx) + d2y
                                      + _d2z_cc(u, nx, ny, nz, dz_c, dz_f))
    return d


def diffusion_v(v, nx, ny, nz, dx, dy, dz_c, dz_f, nu):
    """Full Laplacian of v; ``operators.py:54-88``."""
    d = np.zeros_like(v)
    d2x = (v[2:nx+2, 1:ny+1, 1:nz+1] - 2 * v[1:nx+1, 1:ny+1, 1:nz+1]
           + v[0:nx, 1:ny+1, 1:nz+1]) / dx**2
    d[1:nx+1, 1:ny+1, 1:nz+1] = nu * (d2x + _d2y_v(v, nx, ny, nz, dy)
                                      + _d2z_cc(v, nx, ny, nz, dz_c, dz_f))
    return d


def diffusion_w(w, nx, ny, nz, dx, dy, dz_c, dz_f, nu):
    """Full Laplacian of w; ``operators.py:90-124``.  The z term divides by
    ``dz_c[0:nz-1]`` (``operators.py:120``), kept as the reference has it."""
    d = np.zeros_like(w)
    d2x = (w[2:nx+2, 1:ny+1, 1:nz] - 2 * w[1:nx+1, 1:ny+1, 1:nz]
           + w[0:nx, 1:ny+1, 1:nz]) / dx**2
    d2y = (w[1:nx+1, 2:ny+2, 1:nz] - 2 * w[1:nx+1, 1:ny+1, 1:nz]
           + w[1:nx+1, 0:ny, 1:nz]) / dy**2
    d2z = ((w[1:nx+1, 1:ny+1, 2:nz+1] - w[1:nx+1, 1:ny+1, 1:nz]) / dz_f[1:nz][None, None, :]
           - (w[1:nx+1, 1:ny+1, 1:nz] - w[1:nx+1, 1:ny+1, 0:nz-1]) / dz_f[0:nz-1][None, None, :]
           ) / dz_c[0:nz-1][None, None, :]
    d[1:nx+1, 1:ny+1, 1:nz] = nu * (d2x + d2y + d2z)
    return d


# ---------------------------------------------------------------------------
# Explicit RHS as the two reference code paths compute it
# ---------------------------------------------------------------------------
def rhs_imex_separate(u, v, w, nx, ny, nz, dx, dy, dz_c, dz_f, nu):
    """CPU path of ``solver.py:601-622``: advection + xy diffusion as separate
    ops.  x/y diffusion also lands on the duplicate planes u[nx], v[:, ny]."""
    ru = diffusion_xy_u(u, nx, ny, nz, dx, dy, nu) - advection_u(u, v, w, nx, ny, nz, dx, dy, dz_f)
    rv = diffusion_xy_v(v, nx, ny, nz, dx, dy, nu) - advection_v(u, v, w, nx, ny, nz, dx, dy, dz_f)
    rw = diffusion_xy_w(w, nx, ny, nz, dx, dy, nu) - advection_w(u, v, w, nx, ny, nz, dx, dy, dz_c)
    return ru, rv, rw


def rhs_imex_fused(u, v, w, nx, ny, nz, dx, dy, dz_c, dz_f, nu):
    """CUDA path ``compute_momentum_rhs_fused_imex`` (``operators.py:1037-1225``):
    the same terms, but rhs_u only on ``[1:nx]`` (``:1122``) and rhs_v only on
    ``[:, 1:ny]`` (``:1173``)."""
    ru, rv, rw = rhs_imex_separate(u, v, w, nx, ny, nz, dx, dy, dz_c, dz_f, nu)
    ru[nx] = 0.0
    rv[:, ny] = 0.0
    return ru, rv, rw


def rhs_full_separate(u, v, w, nx, ny, nz, dx, dy, dz_c, dz_f, nu):
    """CPU path of ``compute_momentum_rhs_explicit`` (``solver.py:518-532``)."""
    ru = diffusion_u(u, nx, ny, nz, dx, dy, dz_c, dz_f, nu) - advection_u(u, v, w, nx, ny, nz, dx, dy, dz_f)
    rv = diffusion_v(v, nx, ny, nz, dx, dy, dz_c, dz_f, nu) - advection_v(u, v, w, nx, ny, nz, dx, dy, dz_f)
    rw = diffusion_w(w, nx, ny, nz, dx, dy, dz_c, dz_f, nu) - advection_w(u, v, w, nx, ny, nz, dx, dy, dz_c)
    return ru, rv, rw


def rhs_full_fused(u, v, w, nx, ny, nz, dx, dy, dz_c, dz_f, nu):
    """CUDA path ``compute_momentum_rhs_fused_v2`` (``operators.py:818-1034``):
    rhs_u on ``[1:nx]`` (``:915``), rhs_v on ``[:, 1:ny]`` (``:966``)."""
    ru, rv, rw = rhs_full_separate(u, v, w, nx, ny, nz, dx, dy, dz_c, dz_f, nu)
    ru[nx] = 0.0
    rv[:, ny] = 0.0
    return ru, rv, rw


# ---------------------------------------------------------------------------
# Implicit (Crank-Nicolson) z diffusion
# ---------------------------------------------------------------------------
def pcr_solve(a, b, c, d):
    """Parallel cyclic reduction; ``tridiag.py:33-58`` (shifts ``:20-30``).
    a, b, c are 1-D (n,); d is (batch, n)."""
    n = d.shape[-1]
    a = a.copy(); b = b.copy(); c = c.copy(); d = d.copy()

    def shift(x, s, down, fill):
        y = np.full_like(x, fill)
        if s < n:
            if down:
                y[..., s:] = x[..., :n - s]
            else:
                y[..., :n - s] = x[..., s:]
        return y

    s = 1
    while s < n:
        a_dn = shift(a, s, True, 0.0); b_dn = shift(b, s, True, 1.0)
        c_dn = shift(c, s, True, 0.0)
        a_up = shift(a, s, False, 0.0); b_up = shift(b, s, False, 1.0)
        c_up = shift(c, s, False, 0.0)
        d_dn = shift(d, s, True, 0.0); d_up = shift(d, s, False, 0.0)
        alpha = -a / b_dn
        gamma = -c / b_up
        b = b + alpha * c_dn + gamma * a_up
        d = d + alpha * d_dn + gamma * d_up
        a = alpha * a_dn
        c = gamma * c_up
        s *= 2
    return d / b


def cn_coefficients_uv(dt, nz, dz_c, dz_f, nu, top_wall_bc_type="dirichlet", theta=0.5):
    """Tridiagonal rows for u/v; ``operators.py:581-620``."""
    alpha = theta * dt * nu
    dl, dr, dc = dz_c[0:nz], dz_c[1:nz+1], dz_f[0:nz]
    lo = -alpha / (dl * dc)
    ce = 1.0 + alpha * (1.0 / dl + 1.0 / dr) / dc
    up = -alpha / (dr * dc)
    a, b, c = lo.copy(), ce.copy(), up.copy()
    a[0] = 0.0
    b[0] = ce[0] - lo[0]
    if top_wall_bc_type == "neumann":
        b[nz-1] = ce[nz-1] + up[nz-1]
    else:
        b[nz-1] = ce[nz-1] - up[nz-1]
    c[nz-1] = 0.0
    return a, b, c


def solve_implicit_diffusion_uv(q, dt, nx, ny, nz, dz_c, dz_f, nu, theta=0.5,
                                top_wall_bc_type="dirichlet"):
    """``solve_implicit_diffusion_u`` (``operators.py:563-654``); ``_v``
    (``:657-731``) is the same arithmetic on v's interior ``[1:nx+1, 1:ny+1]``."""
    out = q.copy()
    a, b, c = cn_coefficients_uv(dt, nz, dz_c, dz_f, nu, top_wall_bc_type, theta)
    d = q[1:nx+1, 1:ny+1, 1:nz+1].copy()
    if theta < 1.0:                                         # operators.py:627-644
        beta = (1.0 - theta) * dt * nu
        dl, dr, dc = dz_c[0:nz], dz_c[1:nz+1], dz_f[0:nz]
        U = q[1:nx+1, 1:ny+1, :]
        d2 = ((U[:, :, 2:nz+2] - U[:, :, 1:nz+1]) / dr
              - (U[:, :, 1:nz+1] - U[:, :, 0:nz]) / dl) / dc
        d2[:, :, 0] = ((U[:, :, 2] - U[:, :, 1]) / dr[0] - 2.0 * U[:, :, 1] / dl[0]) / dc[0]
        if top_wall_bc_type == "neumann":
            d2[:, :, nz-1] = (-(U[:, :, nz] - U[:, :, nz-1]) / dl[nz-1]) / dc[nz-1]
        else:
            d2[:, :, nz-1] = (-2.0 * U[:, :, nz] / dr[nz-1]
                              - (U[:, :, nz] - U[:, :, nz-1]) / dl[nz-1]) / dc[nz-1]
        d = d + beta * d2
    x = pcr_solve(a, b, c, d.reshape(nx * ny, nz))          # operators.py:648-652
    out[1:nx+1, 1:ny+1, 1:nz+1] = x.reshape(nx, ny, nz)
    return out


def cn_coefficients_w(dt, nz, dz_c, dz_f, nu, theta=0.5):
    """Tridiagonal rows for w's nz-1 interior faces; ``operators.py:753-777``."""
    alpha = theta * dt * nu
    ni = nz - 1
    dl, dr, dcv = dz_f[0:ni], dz_f[1:nz], dz_c[1:nz]
    lo = -alpha / (dl * dcv)
    ce = 1.0 + alpha * (1.0 / dl + 1.0 / dr) / dcv
    up = -alpha / (dr * dcv)
    a, b, c = lo.copy(), ce.copy(), up.copy()
    a[0] = 0.0
    c[ni-1] = 0.0
    return a, b, c


def solve_implicit_diffusion_w(w, dt, nx, ny, nz, dz_c, dz_f, nu, theta=0.5):
    """``operators.py:734-811``.  The explicit CN half keeps the reference's
    index convention (``:785-803``): row m of the system (face m+1) takes its
    second difference centred on stored face m."""
    out = w.copy()
    a, b, c = cn_coefficients_w(dt, nz, dz_c, dz_f, nu, theta)
    ni = nz - 1
    d = w[1:nx+1, 1:ny+1, 1:nz].copy()
    if theta < 1.0:
        beta = (1.0 - theta) * dt * nu
        dl, dr, dcv = dz_f[0:ni], dz_f[1:nz], dz_c[1:nz]
        W = w[1:nx+1, 1:ny+1, :]
        d2 = np.empty((nx, ny, ni))
        d2[:, :, 1:ni-1] = ((W[:, :, 2:ni] - W[:, :, 1:ni-1]) / dr[1:ni-1]
                            - (W[:, :, 1:ni-1] - W[:, :, 0:ni-2]) / dl[1:ni-1]) / dcv[1:ni-1]
        d2[:, :, 0] = ((W[:, :, 1] - W[:, :, 0]) / dr[0] - W[:, :, 0] / dl[0]) / dcv[0]
        d2[:, :, ni-1] = (-W[:, :, ni-1] / dr[ni-1]
                          - (W[:, :, ni-1] - W[:, :, ni-2]) / dl[ni-1]) / dcv[ni-1]
        d = d + beta * d2
    x = pcr_solve(a, b, c, d.reshape(nx * ny, ni))
    out[1:nx+1, 1:ny+1, 1:nz] = x.reshape(nx, ny, ni)
    return out


# ---------------------------------------------------------------------------
# Divergence, projection, bulk velocity, friction velocity, CFL
# ---------------------------------------------------------------------------
def compute_divergence(u, v, w, nx, ny, nz, dx, dy, dz_f):
    """``utils.py:226-240``; returns (nx, ny, nz)."""
    return ((u[1:nx+1, 1:ny+1, 1:nz+1] - u[0:nx, 1:ny+1, 1:nz+1]) / dx
            + (v[1:nx+1, 1:ny+1, 1:nz+1] - v[1:nx+1, 0:ny, 1:nz+1]) / dy
            + (w[1:nx+1, 1:ny+1, 1:nz+1] - w[1:nx+1, 1:ny+1, 0:nz]) / dz_f[None, None, 0:nz])


def project_velocity(u, v, w, p, nx, ny, nz, dx, dy, dz_c, dz_f, dt):
    """In-place velocity correction u -= dt grad p; ``projection.py:143-165``."""
    u[1:nx+1, 1:ny+1, 1:nz+1] -= dt * ((p[2:nx+2, 1:ny+1, 1:nz+1] - p[1:nx+1, 1:ny+1, 1:nz+1]) / dx)
    v[1:nx+1, 1:ny+1, 1:nz+1] -= dt * ((p[1:nx+1, 2:ny+2, 1:nz+1] - p[1:nx+1, 1:ny+1, 1:nz+1]) / dy)
    w[1:nx+1, 1:ny+1, 1:nz] -= dt * ((p[1:nx+1, 1:ny+1, 2:nz+1] - p[1:nx+1, 1:ny+1, 1:nz])
                                     / dz_c[None, None, 1:nz])
    return u, v, w


def compute_bulk_velocity(u, nx, ny, nz, dx, dy, dz_f, total_volume):
    """``utils.py:207-223`` with ``cell_vol = dx*dy*dz_f`` (``solver.py:231``)."""
    vol = dx * dy * dz_f[None, None, :]
    return float(np.sum(u[1:nx+1, 1:ny+1, 1:nz+1] * vol) / total_volume)


def compute_u_tau(u, z_c, nu, top_wall_bc_type="dirichlet"):
    """``utils.py:176-204``: one-sided wall gradient from the ghost-inclusive
    plane means ``u[:, :, 1]`` and ``u[:, :, -2]``."""
    dist = z_c[1]
    u_tau_bot = np.sqrt(abs(nu * np.mean(u[:, :, 1]) / dist))
    if top_wall_bc_type == "neumann":
        return float(u_tau_bot)
    u_tau_top = np.sqrt(abs(nu * np.mean(u[:, :, -2]) / dist))
    return float(0.5 * (u_tau_bot + u_tau_top))


def compute_cfl_inverse(u, v, w, nx, ny, nz, dx, dy, dz_f, dz_c):
    """Max inverse CFL time scale; ``operators.py:1232-1333``."""
    dxi, dyi = 1.0 / dx, 1.0 / dy
    dzfi = (1.0 / dz_f)[None, None, 0:nz]
    dzci = (1.0 / dz_c)[None, None, 1:nz]
    ux = np.abs(u[1:nx+1, 1:ny+1, 1:nz+1])
    vx = 0.25 * np.abs(v[1:nx+1, 1:ny+1, 1:nz+1] + v[1:nx+1, 0:ny, 1:nz+1]
                       + v[2:nx+2, 1:ny+1, 1:nz+1] + v[2:nx+2, 0:ny, 1:nz+1])
    wx = 0.25 * np.abs(w[1:nx+1, 1:ny+1, 1:nz+1] + w[1:nx+1, 1:ny+1, 0:nz]
                       + w[2:nx+2, 1:ny+1, 1:nz+1] + w[2:nx+2, 1:ny+1, 0:nz])
    dtix = ux * dxi + vx * dyi + wx * dzfi
    uy = 0.25 * np.abs(u[1:nx+1, 1:ny+1, 1:nz+1] + u[1:nx+1, 2:ny+2, 1:nz+1]
                       + u[0:nx, 2:ny+2, 1:nz+1] + u[0:nx, 1:ny+1, 1:nz+1])
    vy = np.abs(v[1:nx+1, 1:ny+1, 1:nz+1])
    wy = 0.25 * np.abs(w[1:nx+1, 1:ny+1, 1:nz+1] + w[1:nx+1, 2:ny+2, 1:nz+1]
                       + w[1:nx+1, 2:ny+2, 0:nz] + w[1:nx+1, 1:ny+1, 0:nz])
    dtiy = uy * dxi + vy * dyi + wy * dzfi
    uz = 0.25 * np.abs(u[1:nx+1, 1:ny+1, 1:nz] + u[0:nx, 1:ny+1, 1:nz]
                       + u[0:nx, 1:ny+1, 2:nz+1] + u[1:nx+1, 1:ny+1, 2:nz+1])
    vz = 0.25 * np.abs(v[1:nx+1, 1:ny+1, 1:nz] + v[1:nx+1, 0:ny, 1:nz]
                       + v[1:nx+1, 0:ny, 2:nz+1] + v[1:nx+1, 1:ny+1, 2:nz+1])
    wz = np.abs(w[1:nx+1, 1:ny+1, 1:nz])
    dtiz = uz * dxi + vz * dyi + wz * dzci
    return float(max(dtix.max(), dtiy.max(), dtiz.max()))


def cfl_dt(dti, cfl_target, dt_min, dt_max):
    """``solver.py:465-496``: dt = clamp(CFL / dti, dt_min, dt_max)."""
    if dti < 1e-10:
        dti = 1.0
    return min(max(cfl_target * (1.0 / dti), dt_min), dt_max)
