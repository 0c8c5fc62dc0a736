"""Initial flow fields (set-up, host side).

Same fields as the reference's ``initialize_flow`` (``initflow.py:4-104``):
laminar profile (full parabola for a no-slip top wall, half parabola for a
free-slip one), uniform, or vortex initialisation, plus uniform noise of
amplitude ``perturbation_intensity * U_bulk`` on ``[1:-1, 1:-1, 2:-2]``.
The reference draws the noise from the unseeded global torch RNG on the run
device (``initflow.py:90-92``); here it comes from
``numpy.random.default_rng(seed)`` on the host so runs are reproducible.
"""
import numpy as np


def initialize_flow(nx, ny, nz, z_c, Ly, Lz, U_bulk=1.0, init_type="parabolic", perturbation_intensity=0.0,
                    n_vortices=4, seed=0, top_wall_bc_type="dirichlet"):
    z_c = np.asarray(z_c, dtype=np.float64)
    u = np.zeros((nx + 1, ny + 2, nz + 2))
    v = np.zeros((nx + 2, ny + 1, nz + 2))
    w = np.zeros((nx + 2, ny + 2, nz + 1))
    p = np.zeros((nx + 2, ny + 2, nz + 2))
    if init_type in ("parabolic", "vortices"):
        U_max = 1.5 * U_bulk
        if top_wall_bc_type == "neumann":
            zn = z_c / Lz
            prof = U_max * zn * (2 - zn)
        else:
            zn = 2 * z_c / Lz - 1
            prof = U_max * (1 - zn ** 2)
        u[:, :, :] = prof[None, None, :]
    if init_type == "uniform":
        u[:, :, :] = U_bulk
    elif init_type == "vortices":
        A = perturbation_intensity * U_bulk
        ky = n_vortices * np.pi / Ly
        y_v = np.linspace(0, Ly, ny + 1)
        y_c = 0.5 * (y_v[:-1] + y_v[1:])
        zci = z_c[1:nz + 1]
        yy, zz = np.meshgrid(y_v, zci, indexing="ij")
        v_pert = -A * np.sin(ky * yy) * 2 * np.sin(np.pi * zz / Lz) * np.cos(np.pi * zz / Lz) * (np.pi / Lz)
        v[1:nx + 1, :, 1:nz + 1] += v_pert[None, :, :]
        z_f_local = np.concatenate([[0.0], 0.5 * (zci[:-1] + zci[1:]), [Lz]])
        yy, zz = np.meshgrid(y_c, z_f_local, indexing="ij")
        w_pert = A * np.cos(ky * yy) * ky * np.sin(np.pi * zz / Lz) ** 2
        w[1:nx + 1, 1:ny + 1, :] += w_pert[None, :, :]
    if perturbation_intensity > 0.0 and init_type != "vortices":
        rng = np.random.default_rng(seed)
        s = perturbation_intensity * U_bulk
        u[1:-1, 1:-1, 2:-2] += (rng.random(u[1:-1, 1:-1, 2:-2].shape) - 0.5) * 2 * s
        v[1:-1, 1:-1, 2:-2] += (rng.random(v[1:-1, 1:-1, 2:-2].shape) - 0.5) * 2 * s
        w[1:-1, 1:-1, 2:-2] += (rng.random(w[1:-1, 1:-1, 2:-2].shape) - 0.5) * 2 * s
    u[:, :, 0] = -u[:, :, 1]; u[:, :, -1] = -u[:, :, -2]
    v[:, :, 0] = -v[:, :, 1]; v[:, :, -1] = -v[:, :, -2]
    w[:, :, 0] = 0.0; w[:, :, -1] = 0.0
    return u, v, w, p
