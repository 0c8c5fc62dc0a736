"""Wall-normal grid generation (set-up, host side).

Same arithmetic as the reference's ``generate_grid`` (``utils.py:5-45``) and
``generate_hybrid_grid`` (``utils.py:47-113``), in numpy FP64.
"""
import numpy as np


def _centres(z_f):
    z_c_inn = 0.5 * (z_f[:-1] + z_f[1:])
    z_c = np.concatenate([[-z_c_inn[0]], z_c_inn, [2 * z_f[-1] - z_c_inn[-1]]])
    return z_f, z_c, z_f[1:] - z_f[:-1], z_c[1:] - z_c[:-1]


def generate_grid(gamma, nz, Lz, stretching_type="symmetric"):
    """tanh stretching clustered at both walls ('symmetric') or at the bottom
    wall only ('bottom').  Returns z_f (nz+1), z_c (nz+2, mirrored ghosts),
    dz_f (nz), dz_c (nz+1)."""
    k = np.linspace(0.0, nz, nz + 1)
    if stretching_type == "bottom":
        z_f = Lz * (1.0 - np.tanh(gamma * (1.0 - k / nz)) / np.tanh(gamma))
    elif stretching_type == "symmetric":
        z_f = 0.5 * Lz * (1 + np.tanh(gamma * ((2 * k / nz) - 1)) / np.tanh(gamma))
    else:
        raise ValueError(f"Invalid stretching type: {stretching_type}")
    return _centres(z_f)


def generate_hybrid_grid(nz_uniform, nz_stretched, z_transition, Lz, gamma):
    """Uniform cells on [0, z_transition], one-sided tanh above."""
    z_u = np.linspace(0.0, z_transition, nz_uniform + 1)
    xi = np.linspace(0.0, nz_stretched, nz_stretched + 1) / nz_stretched
    z_s = (Lz - z_transition) * (1.0 - np.tanh(gamma * (1.0 - xi)) / np.tanh(gamma))
    z_f = np.concatenate([z_u, z_transition + z_s[1:]])
    out = _centres(z_f)
    if np.any(out[2] <= 0):
        raise ValueError("Non-positive cell spacing detected in hybrid grid!")
    return out
