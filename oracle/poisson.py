"""FFT/tridiagonal pressure Poisson solve (oracle restatement, test
infrastructure only).  Follows ``projection_fft.py`` of the reference."""
import numpy as np


def initialize_fft_solver(nx, ny, nz, dx, dy, dz_c, dz_f):
    """Modified wavenumbers and per-mode tridiagonal rows;
    ``projection_fft.py:3-99`` (materialised exactly like the reference)."""
    kx = np.fft.fftfreq(nx, d=dx / (2 * np.pi))            # :26
    ky = np.fft.rfftfreq(ny, d=dy / (2 * np.pi))           # :27
    kxm = (2.0 / dx) * np.sin(kx * dx / 2.0)               # :30
    kym = (2.0 / dy) * np.sin(ky * dy / 2.0)               # :31
    k2 = kxm[:, None] ** 2 + kym[None, :] ** 2             # :38-39
    cl = 1.0 / (dz_c[:-1] * dz_f)                          # :48
    cr = 1.0 / (dz_c[1:] * dz_f)                           # :49
    nkx, nky = len(kx), len(ky)
    tri_a = np.zeros((nkx, nky, nz)); tri_a[:, :, 1:] = cl[1:]       # :56-57
    tri_c = np.zeros((nkx, nky, nz)); tri_c[:, :, :-1] = cr[:-1]     # :60-61
    tri_b = -((cl + cr)[None, None, :] + k2[:, :, None])             # :64-65
    tri_b[:, :, 0] += cl[0]                                          # :70
    tri_b[:, :, -1] += cr[-1]                                        # :82
    return dict(kx=kx, ky=ky, k2=k2, tri_a=tri_a, tri_b=tri_b, tri_c=tri_c,
                nx=nx, ny=ny, nz=nz)


def thomas(a, b, c, d, pin_first_row=False):
    """Batched Thomas sweep; ``projection_fft.py:167-215`` (a, b, c, d all
    (batch, n); d may be complex).

    ``pin_first_row=True`` gauges system 0 (the (kx,ky)=(0,0) mode, whose
    matrix is singular): its last unknown is set to 0 instead of being divided
    by the roundoff-level last pivot.  The reference divides; its pivot is
    exactly 0.0 at some sizes (e.g. 24x16x12, and 192x192x128 with numpy's
    grid arithmetic), which turns p into inf/NaN.  Where the reference's pivot
    is non-zero its solution equals the gauged one plus a constant, so the
    velocities after projection are the same."""
    bs, n = d.shape
    cp = np.zeros((bs, n), dtype=d.dtype)
    dp = np.zeros((bs, n), dtype=d.dtype)
    x = np.zeros((bs, n), dtype=d.dtype)
    with np.errstate(divide="ignore", invalid="ignore"):
        cp[:, 0] = c[:, 0] / b[:, 0]
        dp[:, 0] = d[:, 0] / b[:, 0]
        for i in range(1, n):
            den = b[:, i] - a[:, i] * cp[:, i - 1]
            if i < n - 1:
                cp[:, i] = c[:, i] / den
            dp[:, i] = (d[:, i] - a[:, i] * dp[:, i - 1]) / den
    x[:, n - 1] = dp[:, n - 1]
    if pin_first_row:
        x[0, n - 1] = 0.0
    for i in range(n - 2, -1, -1):
        x[:, i] = dp[:, i] - cp[:, i] * x[:, i + 1]
    return x


def solve_poisson_fft(div, fd, gauge=True):
    """rfft2 -> per-mode Thomas -> irfft2 -> ghost fill;
    ``projection_fft.py:101-165``.  Returns p (nx+2, ny+2, nz+2).

    The (0,0) mode is singular (both Neumann closures, nothing pins the mean),
    so p carries an arbitrary constant: compare p modulo its mean.  With
    ``gauge=True`` (default) the (0,0) mode is pinned, see ``thomas``."""
    nx, ny, nz = fd["nx"], fd["ny"], fd["nz"]
    dh = np.fft.rfft2(div, axes=(0, 1))                               # :118
    nkx, nky = dh.shape[0], dh.shape[1]
    ph = thomas(fd["tri_a"].reshape(-1, nz), fd["tri_b"].reshape(-1, nz),
                fd["tri_c"].reshape(-1, nz), dh.reshape(-1, nz),
                pin_first_row=gauge)                                  # :125-132
    pin = np.fft.irfft2(ph.reshape(nkx, nky, nz), s=(nx, ny), axes=(0, 1))  # :139
    p = np.zeros((nx + 2, ny + 2, nz + 2))
    p[1:nx+1, 1:ny+1, 1:nz+1] = pin                                   # :146
    p[0] = p[nx]; p[nx+1] = p[1]                                      # :150-151
    p[:, 0] = p[:, ny]; p[:, ny+1] = p[:, 1]                          # :154-155
    p[:, :, 0] = p[:, :, 1]                                           # :159
    p[:, :, nz+1] = p[:, :, nz]                                       # :163
    return p


def poisson_residual(p, rhs, nx, ny, nz, dx, dy, dz_c, dz_f):
    """Discrete residual L p - rhs of the operator the solve inverts
    (x/y: 3-point periodic; z: ``projection_fft.py:44-82`` rows with Neumann
    closures), on the interior."""
    pi = p[1:nx+1, 1:ny+1, 1:nz+1]
    lap = (np.roll(pi, -1, 0) - 2 * pi + np.roll(pi, 1, 0)) / dx**2
    lap += (np.roll(pi, -1, 1) - 2 * pi + np.roll(pi, 1, 1)) / dy**2
    cl = 1.0 / (dz_c[:-1] * dz_f)
    cr = 1.0 / (dz_c[1:] * dz_f)
    up = np.concatenate([pi[:, :, 1:], pi[:, :, -1:]], axis=2)
    dn = np.concatenate([pi[:, :, :1], pi[:, :, :-1]], axis=2)
    lap += cr * (up - pi) - cl * (pi - dn)
    return lap - rhs
