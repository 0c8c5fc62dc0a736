"""CPU study of single-precision pressure solves on the oracle step (test
infrastructure: it documents why the single-precision Poisson step solves
for an increment; nothing in the package imports it).

The oracle runs the reference IMEX step (``solver.py:580-710``) in FP64 on
the seeded laminar + 0.1 noise field; at selected steps the pressure solve of
``projection_fft.py:101-215`` is repeated on the same predictor u** with
numpy emulations of reduced precision, and the post-projection max|div| of
each variant is printed:

* ``fp64``: the FP64 solve (the reference);
* ``fp64+u32``: the FP64 solve with u, v, w stored in FP32 afterwards (u as
  its deviation from the plane means), the mixed form's storage;
* ``p32``: the FP64 solve, p rounded to FP32;
* ``fp32``: FP32 spectrum (rfft2 / Thomas / irfft2 in float32);
* ``fp32+low64``: the same with the modes kx < 3, |ky| < 3 solved in FP64;
* ``inc1``: the FP32 solve (low modes FP64) of the increment over the
  previous step's p rounded to FP32 (right-hand side div/dt - L p_prev);
* ``inc2``: the same over the linear extrapolation 2 p_prev - p_prev2.

Usage: python -m oracle.precision_study [nx ny nz steps] (default 192 192 128
30; about 3 minutes at that size on one core).
"""
import sys

import numpy as np

from . import ops, poisson
from .step import OracleChannel


def _ghost(pin, nx, ny, nz):
    p = np.zeros((nx + 2, ny + 2, nz + 2))
    p[1:nx + 1, 1:ny + 1, 1:nz + 1] = pin
    p[0] = p[nx]; p[nx + 1] = p[1]
    p[:, 0] = p[:, ny]; p[:, ny + 1] = p[:, 1]
    p[:, :, 0] = p[:, :, 1]; p[:, :, nz + 1] = p[:, :, nz]
    return p


def main(nx=192, ny=192, nz=128, nsteps=30):
    oc = OracleChannel(nx, ny, nz, 4 * np.pi, 4 * np.pi / 3, 2.0, 2870.0)
    oc.init_fresh(seed=0)
    dt = oc.cfl_dt(0.25, 3e-4, 0.011)
    fd = oc.fd
    A, B, C = (fd[k].reshape(-1, nz) for k in ("tri_a", "tri_b", "tri_c"))
    A32, B32, C32 = A.astype(np.float32), B.astype(np.float32), C.astype(np.float32)
    ix = np.arange(fd["tri_a"].shape[0])
    iy = np.arange(fd["tri_a"].shape[1])
    low = ((np.minimum(ix, nx - ix)[:, None] < 3) & (iy[None, :] < 3)).reshape(-1)

    def solve64(rhs):
        return poisson.solve_poisson_fft(rhs, fd)[1:nx + 1, 1:ny + 1, 1:nz + 1]

    def solve32(rhs, low64):
        dh = np.fft.rfft2(rhs.astype(np.float32), axes=(0, 1))
        d = dh.reshape(-1, nz)
        x = poisson.thomas(A32, B32, C32, d, pin_first_row=True)
        if low64:
            x[low] = poisson.thomas(A[low], B[low], C[low], d[low].astype(np.complex128),
                                    pin_first_row=True).astype(np.complex64)
        return np.fft.irfft2(x.reshape(dh.shape), s=(nx, ny), axes=(0, 1)).astype(np.float64)

    def lap(pin):
        return poisson.poisson_residual(_ghost(pin, nx, ny, nz), 0.0, nx, ny, nz, oc.dx, oc.dy, oc.dz_c, oc.dz_f)

    def post_div(pin, round32=False):
        u, v, w = oc.u.copy(), oc.v.copy(), oc.w.copy()
        ops.project_velocity(u, v, w, _ghost(pin, nx, ny, nz), nx, ny, nz, oc.dx, oc.dy, oc.dz_c, oc.dz_f, dt)
        ops.apply_bc_all(u, v, w, oc.top)
        if round32:
            U0 = u.mean(axis=(0, 1), keepdims=True)
            u = (u - U0).astype(np.float32).astype(np.float64) + U0
            v, w = v.astype(np.float32).astype(np.float64), w.astype(np.float32).astype(np.float64)
            ops.apply_bc_all(u, v, w, oc.top)
        return np.abs(ops.compute_divergence(u, v, w, nx, ny, nz, oc.dx, oc.dy, oc.dz_f)).max()

    print(f"{nx}x{ny}x{nz}, dt {dt:.5f}: post-projection max|div|")
    print("step   fp64      fp64+u32  p32       fp32      fp32+low64 inc1      inc2      |p|       |dp1|")
    hist = []
    for n in range(1, nsteps + 1):
        ops.apply_bc_all(oc.u, oc.v, oc.w, oc.top)
        oc._ab2_update(oc.explicit_rhs_imex(), dt)
        ops.apply_bc_all(oc.u, oc.v, oc.w, oc.top)
        oc.u = ops.solve_implicit_diffusion_uv(oc.u, dt, nx, ny, nz, oc.dz_c, oc.dz_f, oc.nu, top_wall_bc_type=oc.top)
        oc.v = ops.solve_implicit_diffusion_uv(oc.v, dt, nx, ny, nz, oc.dz_c, oc.dz_f, oc.nu, top_wall_bc_type=oc.top)
        oc.w = ops.solve_implicit_diffusion_w(oc.w, dt, nx, ny, nz, oc.dz_c, oc.dz_f, oc.nu)
        ops.apply_bc_all(oc.u, oc.v, oc.w, oc.top)
        rhs = oc.divergence() / dt
        p64 = solve64(rhs)
        if n in (1, 2, 5, 10, 15, 20) or n == nsteps:
            cols = [post_div(p64), post_div(p64, True), post_div(p64.astype(np.float32).astype(np.float64)),
                    post_div(solve32(rhs, False)), post_div(solve32(rhs, True))]
            for k in (1, 2):
                if len(hist) >= k:
                    pb = hist[-1] if k == 1 else 2 * hist[-1] - hist[-2]
                    pb = pb.astype(np.float32).astype(np.float64)
                    cols.append(post_div(pb + solve32(rhs - lap(pb), True)))
                else:
                    cols.append(float("nan"))
            cols += [np.abs(p64 - p64.mean()).max(), np.abs(p64 - hist[-1]).max() if hist else float("nan")]
            print(f"{n:4d}  " + "  ".join(f"{x:.2e}" for x in cols), flush=True)
        hist = (hist + [p64])[-2:]
        ops.project_velocity(oc.u, oc.v, oc.w, _ghost(p64, nx, ny, nz), nx, ny, nz, oc.dx, oc.dy, oc.dz_c,
                             oc.dz_f, dt)
        ops.apply_bc_all(oc.u, oc.v, oc.w, oc.top)
        oc._forcing_update(dt)


if __name__ == "__main__":
    a = [int(x) for x in sys.argv[1:5]]
    main(*a)
