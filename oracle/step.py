"""Whole time steps (oracle restatement, test infrastructure only).

``OracleChannel`` restates the state handling of ``ChannelFlow``
(``solver.py:81-710``): IMEX follows ``step_imex`` (``solver.py:580-710``)
verbatim; FE follows the body of ``step_forward_euler``
(``solver.py:537-576``) without its broken return (the reference raises
NameError at ``:578``); AB2 is ``step_imex`` with the full-diffusion RHS of
``compute_momentum_rhs_explicit`` (``solver.py:498-534``) and no implicit
solve, as ``docs/NUMERICAL_METHODS.md:260-284`` describes it (the reference
documents AB2 but ``run_simulation`` cannot select it, ``solver.py:742-752``).

``rhs_path`` names which reference code path the explicit RHS follows:
``"separate"`` = the reference's CPU path (``solver.py:601-622``, the default
parity target), ``"fused"`` = its CUDA path (``operators.py:1037-1225``), which
leaves the duplicate planes u[nx] and v[:, ny] without x/y diffusion.
"""
import numpy as np

from . import ops, poisson
from .grid import generate_grid


def initial_fields(nx, ny, nz, z_c, Lz, U_bulk=1.0, perturbation=0.1, seed=0,
                   init_type="parabolic", top_wall_bc_type="dirichlet"):
    """Laminar profile + uniform noise, ``initflow.py:4-104`` (parabolic /
    uniform / random branches).  The reference draws its noise from the
    unseeded global torch RNG (``initflow.py:90-92``); here it comes from
    ``numpy.random.default_rng(seed)`` so that runs are reproducible."""
    u = np.zeros((nx + 1, ny + 2, nz + 2))
    v = np.zeros((nx + 2, ny + 1, nz + 2))
    w = np.zeros((nx + 2, ny + 2, nz + 1))
    p = np.zeros((nx + 2, ny + 2, nz + 2))
    if init_type in ("parabolic", "vortices"):
        if top_wall_bc_type == "neumann":
            zn = z_c / Lz
            prof = 1.5 * U_bulk * zn * (2 - zn)
        else:
            zn = 2 * z_c / Lz - 1
            prof = 1.5 * U_bulk * (1 - zn ** 2)
        u[:, :, :] = prof[None, None, :]
    if init_type == "uniform":
        u[:, :, :] = U_bulk
    if perturbation > 0.0 and init_type != "vortices":
        rng = np.random.default_rng(seed)
        s = perturbation * U_bulk
        u[1:-1, 1:-1, 2:-2] += (rng.random(u[1:-1, 1:-1, 2:-2].shape) - 0.5) * 2 * s
        v[1:-1, 1:-1, 2:-2] += (rng.random(v[1:-1, 1:-1, 2:-2].shape) - 0.5) * 2 * s
        w[1:-1, 1:-1, 2:-2] += (rng.random(w[1:-1, 1:-1, 2:-2].shape) - 0.5) * 2 * s
    u[:, :, 0] = -u[:, :, 1]; u[:, :, -1] = -u[:, :, -2]       # initflow.py:95-102
    v[:, :, 0] = -v[:, :, 1]; v[:, :, -1] = -v[:, :, -2]
    w[:, :, 0] = 0.0; w[:, :, -1] = 0.0
    return u, v, w, p


class OracleChannel:
    def __init__(self, nx, ny, nz, Lx, Ly, Lz, Re, U_bulk=1.0, gamma=2.6,
                 top_wall_bc_type="dirichlet", rhs_path="separate",
                 stretching_type="symmetric", grid=None):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.Lx, self.Ly, self.Lz = Lx, Ly, Lz
        self.nu = 1.0 / Re
        self.U_bulk = U_bulk
        self.top = top_wall_bc_type
        self.rhs_path = rhs_path
        if grid is None:
            grid = generate_grid(gamma, nz, Lz, stretching_type)
        self.z_f, self.z_c, self.dz_f, self.dz_c = [np.asarray(g, dtype=np.float64) for g in grid]
        self.dx, self.dy = Lx / nx, Ly / ny
        self.total_volume = Lx * Ly * Lz
        self.fd = poisson.initialize_fft_solver(nx, ny, nz, self.dx, self.dy, self.dz_c, self.dz_f)
        self.forcing = 0.0
        self.rhs_prev = None
        self.u = self.v = self.w = self.p = None

    # -- set-up -----------------------------------------------------------
    def set_state(self, u, v, w, p=None, forcing=0.0, rhs_prev=None):
        self.u, self.v, self.w = u.copy(), v.copy(), w.copy()
        self.p = np.zeros((self.nx + 2, self.ny + 2, self.nz + 2)) if p is None else p.copy()
        self.forcing = float(forcing)
        self.rhs_prev = None if rhs_prev is None else tuple(r.copy() for r in rhs_prev)

    def bulk(self, u=None):
        return ops.compute_bulk_velocity(self.u if u is None else u, self.nx, self.ny, self.nz,
                                         self.dx, self.dy, self.dz_f, self.total_volume)

    def init_fresh(self, seed=0, perturbation=0.1, init_type="parabolic"):
        """Fresh start: initial field, rescale to U_bulk and project with dt=1;
        ``solver.py:253-276`` and ``:345-370``."""
        u, v, w, p = initial_fields(self.nx, self.ny, self.nz, self.z_c, self.Lz,
                                    self.U_bulk, perturbation, seed, init_type, self.top)
        self.set_state(u, v, w, p)
        ub = self.bulk()
        if abs(ub) > 1e-9:
            self.u *= self.U_bulk / ub
        self.initial_projection()

    def initial_projection(self):
        """``solver.py:345-370``: div -> Poisson -> project(dt=1) -> BC."""
        div = self.divergence()
        self.p = poisson.solve_poisson_fft(div, self.fd)
        ops.project_velocity(self.u, self.v, self.w, self.p, self.nx, self.ny, self.nz,
                             self.dx, self.dy, self.dz_c, self.dz_f, 1.0)
        ops.apply_bc_all(self.u, self.v, self.w, self.top)

    def divergence(self):
        return ops.compute_divergence(self.u, self.v, self.w, self.nx, self.ny, self.nz,
                                      self.dx, self.dy, self.dz_f)

    def _args(self):
        return (self.nx, self.ny, self.nz, self.dx, self.dy, self.dz_c, self.dz_f, self.nu)

    def explicit_rhs_imex(self):
        f = ops.rhs_imex_fused if self.rhs_path == "fused" else ops.rhs_imex_separate
        return f(self.u, self.v, self.w, *self._args())

    def explicit_rhs_full(self):
        f = ops.rhs_full_fused if self.rhs_path == "fused" else ops.rhs_full_separate
        return f(self.u, self.v, self.w, *self._args())

    # -- projection tail shared by every scheme ---------------------------
    def _project(self, dt):
        div = self.divergence()                                           # solver.py:672
        self.p = poisson.solve_poisson_fft(div / dt, self.fd)             # solver.py:682
        ops.project_velocity(self.u, self.v, self.w, self.p, self.nx, self.ny, self.nz,
                             self.dx, self.dy, self.dz_c, self.dz_f, dt)  # solver.py:692
        ops.apply_bc_all(self.u, self.v, self.w, self.top)                # solver.py:697

    def _ab2_update(self, r, dt):
        """``solver.py:626-651``: forcing on every rhs_u entry, AB2 (Euler on
        the first step), keep r as the next step's history."""
        ru, rv, rw = r
        ru = ru + self.forcing
        if self.rhs_prev is None:
            self.u += dt * ru; self.v += dt * rv; self.w += dt * rw
        else:
            pu, pv, pw = self.rhs_prev
            self.u += dt * (1.5 * ru - 0.5 * pu)
            self.v += dt * (1.5 * rv - 0.5 * pv)
            self.w += dt * (1.5 * rw - 0.5 * pw)
        self.rhs_prev = (ru, rv, rw)

    def _forcing_update(self, dt):
        ub = self.bulk()                                                  # solver.py:701
        self.forcing += (self.U_bulk - ub) / dt * 0.1                     # solver.py:707-708
        return ub, self.forcing

    # -- schemes ----------------------------------------------------------
    def step_imex(self, dt):
        """``solver.py:580-710``."""
        ops.apply_bc_all(self.u, self.v, self.w, self.top)                # :588
        self._ab2_update(self.explicit_rhs_imex(), dt)                    # :593-651
        ops.apply_bc_all(self.u, self.v, self.w, self.top)                # :654
        nx, ny, nz, dz_c, dz_f, nu = self.nx, self.ny, self.nz, self.dz_c, self.dz_f, self.nu
        self.u = ops.solve_implicit_diffusion_uv(self.u, dt, nx, ny, nz, dz_c, dz_f, nu,
                                                 top_wall_bc_type=self.top)   # :660
        self.v = ops.solve_implicit_diffusion_uv(self.v, dt, nx, ny, nz, dz_c, dz_f, nu,
                                                 top_wall_bc_type=self.top)   # :662
        self.w = ops.solve_implicit_diffusion_w(self.w, dt, nx, ny, nz, dz_c, dz_f, nu)  # :664
        ops.apply_bc_all(self.u, self.v, self.w, self.top)                # :668
        self._project(dt)
        return self._forcing_update(dt)

    def step_ab2(self, dt):
        """Fully explicit AB2 with PI forcing (documented scheme)."""
        ops.apply_bc_all(self.u, self.v, self.w, self.top)
        self._ab2_update(self.explicit_rhs_full(), dt)
        ops.apply_bc_all(self.u, self.v, self.w, self.top)
        self._project(dt)
        return self._forcing_update(dt)

    def step_fe(self, dt):
        """``solver.py:537-576``: explicit Euler, forcing fixed at 1.0 on the
        u interior (``:552-554``)."""
        ops.apply_bc_all(self.u, self.v, self.w, self.top)
        ru, rv, rw = self.explicit_rhs_full()
        self.u += dt * ru; self.v += dt * rv; self.w += dt * rw
        nx, ny, nz = self.nx, self.ny, self.nz
        self.u[1:nx+1, 1:ny+1, 1:nz+1] += dt * 1.0
        ops.apply_bc_all(self.u, self.v, self.w, self.top)
        self._project(dt)
        return self.bulk(), 1.0

    def cfl_dt(self, cfl_target, dt_min, dt_max):
        dti = ops.compute_cfl_inverse(self.u, self.v, self.w, self.nx, self.ny, self.nz,
                                      self.dx, self.dy, self.dz_f, self.dz_c)
        return ops.cfl_dt(dti, cfl_target, dt_min, dt_max)
