"""Generate vector-Jacobian-product golden vectors by running torch autograd
through the reference TorChannel operators themselves.

Run once in a container that has the reference checked out:

    python tests/golden/make_adjoint_golden.py [--ref /root/reference]

(same matplotlib stub and ``PYTORCH_JIT=0`` set-up as ``make_golden.py``;
CPU, FP64).  Every map takes the degrees of freedom of u, v, w (reference
interiors ``u[1:nx+1, 1:ny+1, 1:nz+1]``, ``v[1:nx+1, 1:ny+1, 1:nz+1]``,
``w[1:nx+1, 1:ny+1, 1:nz]``), fills the ghosts with the reference's own
``apply_bc_all`` (``solver.py:24-79``), applies the reference operator and
returns the interiors it writes.  For a seeded cotangent ``lam`` the file holds
``grad = J^T lam`` from ``torch.autograd.grad``.

Output ``adjoint_16x12x10.npz``:
  rhs_*     explicit IMEX right-hand side of the CPU path (``solver.py:601-622``):
            diffusion_xy - advection (``operators.py:126-247, 474-548``)
  cn_*      ``solve_implicit_diffusion_u/v/w`` (``operators.py:564-811``),
            dt = 0.002, no-slip and free-slip top wall
  bulk_*    ``compute_bulk_velocity`` (``utils.py:208-223``)

The Poisson solve is not differentiated here: its (0,0) mode is singular and
the reference divides by a roundoff-level pivot (``projection_fft.py:197-213``),
so autograd through it amplifies rounding; the projection adjoint is checked by
exact dot-product identities instead.
"""
import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from make_golden import _setup  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    a = ap.parse_args()
    _setup(a.ref)
    import torch
    import operators as O
    import solver as S
    import utils as U

    torch.set_default_dtype(torch.float64)
    nx, ny, nz = 16, 12, 10
    Lx, Ly, Lz = 4 * np.pi, 4 * np.pi / 3, 2.0
    dx, dy = Lx / nx, Ly / ny
    nu = 1.0 / 2870.0
    z_f, z_c, dz_f, dz_c = U.generate_grid(2.6, nz, Lz)
    dz_f = dz_f.double(); dz_c = dz_c.double()
    rng = np.random.default_rng(7)

    def rnd(*shape):
        return torch.tensor(rng.standard_normal(shape))

    def ghosted(ud, vd, wd, top):
        u = torch.zeros(nx + 1, ny + 2, nz + 2); v = torch.zeros(nx + 2, ny + 1, nz + 2)
        w = torch.zeros(nx + 2, ny + 2, nz + 1)
        u = u.index_put((torch.arange(1, nx + 1)[:, None, None], torch.arange(1, ny + 1)[None, :, None],
                         torch.arange(1, nz + 1)[None, None, :]), ud)
        v = v.index_put((torch.arange(1, nx + 1)[:, None, None], torch.arange(1, ny + 1)[None, :, None],
                         torch.arange(1, nz + 1)[None, None, :]), vd)
        w = w.index_put((torch.arange(1, nx + 1)[:, None, None], torch.arange(1, ny + 1)[None, :, None],
                         torch.arange(1, nz)[None, None, :]), wd)
        u = u.clone(); v = v.clone(); w = w.clone()
        S.apply_bc_all(u, v, w, top)
        return u, v, w

    out = {"nx": nx, "ny": ny, "nz": nz, "dz_f": dz_f.numpy(), "dz_c": dz_c.numpy(), "nu": nu,
           "Lx": Lx, "Ly": Ly, "Lz": Lz}
    # state (a laminar profile plus noise) and cotangents
    zc = z_c[1:nz + 1].double()
    ud0 = (1.5 * (1 - (zc - 1) ** 2))[None, None, :] + 0.1 * rnd(nx, ny, nz)
    vd0 = 0.1 * rnd(nx, ny, nz)
    wd0 = 0.1 * rnd(nx, ny, nz - 1)
    out.update(u=ud0.numpy(), v=vd0.numpy(), w=wd0.numpy())

    # ---- explicit IMEX right-hand side (CPU path) ----
    ud, vd, wd = (t.clone().requires_grad_(True) for t in (ud0, vd0, wd0))
    u, v, w = ghosted(ud, vd, wd, "dirichlet")
    ru = O.diffusion_xy_u(u, nx, ny, nz, dx, dy, nu) - O.advection_u(u, v, w, nx, ny, nz, dx, dy, dz_f)
    rv = O.diffusion_xy_v(v, nx, ny, nz, dx, dy, nu) - O.advection_v(u, v, w, nx, ny, nz, dx, dy, dz_f)
    rw = O.diffusion_xy_w(w, nx, ny, nz, dx, dy, nu) - O.advection_w(u, v, w, nx, ny, nz, dx, dy, dz_c)
    ru_i = ru[1:nx + 1, 1:ny + 1, 1:nz + 1]; rv_i = rv[1:nx + 1, 1:ny + 1, 1:nz + 1]; rw_i = rw[1:nx + 1, 1:ny + 1, 1:nz]
    lu, lv, lw = rnd(nx, ny, nz), rnd(nx, ny, nz), rnd(nx, ny, nz - 1)
    g = torch.autograd.grad((ru_i * lu).sum() + (rv_i * lv).sum() + (rw_i * lw).sum(), (ud, vd, wd))
    out.update(rhs_lu=lu.numpy(), rhs_lv=lv.numpy(), rhs_lw=lw.numpy(),
               rhs_ru=ru_i.detach().numpy(), rhs_rv=rv_i.detach().numpy(), rhs_rw=rw_i.detach().numpy(),
               rhs_gu=g[0].numpy(), rhs_gv=g[1].numpy(), rhs_gw=g[2].numpy())

    # ---- Crank-Nicolson z solves ----
    dt = 0.002
    out["cn_dt"] = dt
    for top in ("dirichlet", "neumann"):
        ud, vd, wd = (t.clone().requires_grad_(True) for t in (ud0, vd0, wd0))
        u, v, w = ghosted(ud, vd, wd, top)
        dtt = torch.as_tensor(dt)
        un = O.solve_implicit_diffusion_u(u, dtt, nx, ny, nz, dz_c, dz_f, nu, top_wall_bc_type=top)
        vn = O.solve_implicit_diffusion_v(v, dtt, nx, ny, nz, dz_c, dz_f, nu, top_wall_bc_type=top)
        wn = O.solve_implicit_diffusion_w(w, dtt, nx, ny, nz, dz_c, dz_f, nu)
        oi = (un[1:nx + 1, 1:ny + 1, 1:nz + 1], vn[1:nx + 1, 1:ny + 1, 1:nz + 1], wn[1:nx + 1, 1:ny + 1, 1:nz])
        lu, lv, lw = rnd(nx, ny, nz), rnd(nx, ny, nz), rnd(nx, ny, nz - 1)
        g = torch.autograd.grad((oi[0] * lu).sum() + (oi[1] * lv).sum() + (oi[2] * lw).sum(), (ud, vd, wd))
        tag = "cn_" + top + "_"
        out.update({tag + "lu": lu.numpy(), tag + "lv": lv.numpy(), tag + "lw": lw.numpy(),
                    tag + "ou": oi[0].detach().numpy(), tag + "ov": oi[1].detach().numpy(),
                    tag + "ow": oi[2].detach().numpy(),
                    tag + "gu": g[0].numpy(), tag + "gv": g[1].numpy(), tag + "gw": g[2].numpy()})

    # ---- bulk velocity ----
    ud = ud0.clone().requires_grad_(True)
    u, v, w = ghosted(ud, vd0, wd0, "dirichlet")
    cell_vol = (dx * dy * dz_f)[None, None, :].expand(nx, ny, nz)
    ub = U.compute_bulk_velocity(u, cell_vol, Lx * Ly * Lz)
    (g,) = torch.autograd.grad(ub, (ud,))
    out.update(bulk_ub=float(ub.detach()), bulk_gu=g.numpy())

    path = os.path.join(HERE, "adjoint_16x12x10.npz")
    np.savez(path, **out)
    print("wrote", path)


if __name__ == "__main__":
    main()
