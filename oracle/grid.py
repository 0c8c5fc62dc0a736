"""Wall-normal grid generation (oracle restatement, test infrastructure only).

Follows ``utils.py:5-45`` (``generate_grid``) and ``utils.py:47-113``
(``generate_hybrid_grid``) of the reference.
"""
import numpy as np


def generate_grid(gamma, nz, Lz, stretching_type="symmetric"):
    """tanh-stretched z grid; ``utils.py:5-45``.

    Returns (z_f[nz+1], z_c[nz+2] with mirrored ghosts, dz_f[nz], dz_c[nz+1]).
    """
    k = np.linspace(0.0, nz, nz + 1)                      # utils.py:22
    if stretching_type == "bottom":                        # utils.py:24-30
        xi = k / nz
        z_f = Lz * (1.0 - np.tanh(gamma * (1.0 - xi)) / np.tanh(gamma))
    else:                                                  # utils.py:31-35
        xi = (2 * k / nz) - 1
        z_f = 0.5 * Lz * (1 + np.tanh(gamma * xi) / np.tanh(gamma))
    return _finish(z_f)


def generate_hybrid_grid(nz_uniform, nz_stretched, z_transition, Lz, gamma):
    """Uniform [0, z_t] + one-sided tanh [z_t, Lz]; ``utils.py:47-113``."""
    z_f_uniform = np.linspace(0.0, z_transition, nz_uniform + 1)   # utils.py:68-69
    H = Lz - z_transition                                            # utils.py:73
    k = np.linspace(0.0, nz_stretched, nz_stretched + 1)
    xi = k / nz_stretched
    z_loc = H * (1.0 - np.tanh(gamma * (1.0 - xi)) / np.tanh(gamma))  # utils.py:80
    z_f = np.concatenate([z_f_uniform, z_transition + z_loc[1:]])    # utils.py:83
    z_f, z_c, dz_f, dz_c = _finish(z_f)
    if np.any(dz_f <= 0) or np.any(z_f[1:] <= z_f[:-1]):             # utils.py:106-109
        raise ValueError("Non-monotonic hybrid grid")
    return z_f, z_c, dz_f, dz_c


def _finish(z_f):
    """Cell centres with mirrored ghosts and spacings; ``utils.py:37-43``."""
    z_c_inn = 0.5 * (z_f[:-1] + z_f[1:])
    z_c = np.concatenate([[-z_c_inn[0]], z_c_inn, [2 * z_f[-1] - z_c_inn[-1]]])
    dz_f = z_f[1:] - z_f[:-1]
    dz_c = z_c[1:] - z_c[:-1]
    return z_f, z_c, dz_f, dz_c
