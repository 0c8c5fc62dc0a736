"""Shared helpers for the tests (oracle set-up and comparisons)."""
import numpy as np

from oracle.step import OracleChannel


def rel(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    d = np.max(np.abs(a - b))
    s = np.max(np.abs(b))
    return float(d / (s if s > 0 else 1.0))


def dof(name, a, nx, ny, nz):
    """DOF window of a reference-layout array."""
    if name in ("u", "v"):
        return a[1:nx + 1, 1:ny + 1, 1:nz + 1]
    if name == "w":
        return a[1:nx + 1, 1:ny + 1, 1:nz]
    if name == "p":
        x = a[1:nx + 1, 1:ny + 1, 1:nz + 1]
        return x - x.mean()
    raise KeyError(name)


def make_oracle(nx, ny, nz, seed=0, top="dirichlet", rhs_path="separate", Re=2870.0, gamma=2.6,
                Lx=4 * np.pi, Ly=4 * np.pi / 3, Lz=2.0, stretching="symmetric"):
    oc = OracleChannel(nx, ny, nz, Lx, Ly, Lz, Re, gamma=gamma, top_wall_bc_type=top,
                       rhs_path=rhs_path, stretching_type=stretching)
    oc.init_fresh(seed=seed)
    return oc


def make_gpu(oc, precision="fp64"):
    from torchannel_b200.core import Channel
    ch = Channel(oc.nx, oc.ny, oc.nz, oc.Lx, oc.Ly, oc.Lz, oc.nu, oc.dz_f, oc.dz_c, U_bulk=oc.U_bulk,
                 top_wall_bc_type=oc.top, precision=precision, rhs_path=oc.rhs_path)
    return ch


def np_(t):
    return t.detach().cpu().numpy()
