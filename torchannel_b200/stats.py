"""Turbulence statistics bound to a device channel, with the interface and
file formats of the reference's ``TurbulenceStats`` (``turbstats.py:5-402``).

The running sums live on the device in FP64 (kernel (e), ``tc_stats_*``);
``accumulate_statistics`` adds one sample of the channel's current state.
"""
import os

import numpy as np

_SUMS = ("U_sum", "uu_sum", "vv_sum", "ww_sum", "uw_sum",
         "E_uu_2d_sum", "E_vv_2d_sum", "E_ww_2d_sum", "E_uw_2d_sum")


class TurbulenceStatsB200:
    def __init__(self, channel, z_c, Re_tau_target, z_plus_target=15.0):
        self.ch = channel
        self.nx, self.ny, self.nz = channel.nx, channel.ny, channel.nz
        self.Lx, self.Ly, self.Lz = channel.Lx, channel.Ly, channel.Lz
        self.nu = channel.nu
        self.z_c = np.asarray(z_c, dtype=np.float64)
        self.u_tau_target = Re_tau_target * self.nu / (self.Lz / 2.0)          # turbstats.py:52-53
        self.k_bot, self.k_top = channel.stats_init(self.z_c, Re_tau_target, z_plus_target)
        dx, dy = self.Lx / self.nx, self.Ly / self.ny
        self.kx = 2 * np.pi * np.fft.rfftfreq(self.nx, d=dx)[1:]               # turbstats.py:98-99
        self.ky = 2 * np.pi * np.fft.rfftfreq(self.ny, d=dy)[1:]

    @property
    def n_samples(self):
        return self.ch.stats_read()["n_samples"]

    def accumulate_statistics(self, u=None, v=None, w=None, u_tau_current=None):
        """Add one sample of the channel's current state (the field arguments
        of the reference signature are accepted and not needed: the device
        state is the sample)."""
        self.ch.stats_accumulate()

    def sums(self):
        return self.ch.stats_read()

    def finalize_statistics(self):
        """``turbstats.py:230-303``."""
        s = self.sums()
        n = s["n_samples"]
        if n == 0:
            raise RuntimeError("No samples accumulated - cannot finalize statistics")
        U = s["U_sum"] / n
        dz_utau = float(self.z_c[1])
        dUdz_wall = float(0.5 * (U[0] + U[-1]) / dz_utau)
        u_tau = float(np.sqrt(self.nu * dUdz_wall))
        return {
            "n_samples": n, "z_c": self.z_c[1:self.nz + 1].copy(),
            "U_mean": U, "uu_mean": s["uu_sum"] / n, "vv_mean": s["vv_sum"] / n,
            "ww_mean": s["ww_sum"] / n, "uw_mean": s["uw_sum"] / n,
            "kx": self.kx[:self.nx // 2], "ky": self.ky[:self.ny // 2],
            "E_uu_2d": s["E_uu_2d_sum"] / n, "E_vv_2d": s["E_vv_2d_sum"] / n,
            "E_ww_2d": s["E_ww_2d_sum"] / n, "E_uw_2d": s["E_uw_2d_sum"] / n,
            "z_plus_target": self.k_bot,                 # the reference stores k_bot here (turbstats.py:296)
            "Re_tau_target": self.u_tau_target * (self.Lz / 2) / self.nu,
            "nu": self.nu, "Re": 1.0 / self.nu, "u_tau": u_tau,
        }

    def save_statistics(self, filepath):
        np.savez_compressed(filepath, **self.finalize_statistics())

    @staticmethod
    def load_statistics(filepath):
        if not os.path.exists(filepath):
            raise FileNotFoundError(f"Statistics file not found: {filepath}")
        data = np.load(filepath)
        return {k: data[k] for k in data.files}

    def save_state(self, filepath):
        """``turbstats.py:334-362``: running sums, n_samples and the grid."""
        s = self.sums()
        state = {"n_samples": s["n_samples"]}
        state.update({k: np.asarray(s[k]) for k in _SUMS})
        state.update(nx=self.nx, ny=self.ny, nz=self.nz)
        np.savez_compressed(filepath, **state)

    def load_state(self, filepath):
        """``turbstats.py:364-402``; a grid mismatch raises ValueError."""
        if not os.path.exists(filepath):
            raise FileNotFoundError(f"Statistics state file not found: {filepath}")
        data = np.load(filepath)
        if data["nx"] != self.nx or data["ny"] != self.ny or data["nz"] != self.nz:
            raise ValueError(
                f"Grid dimension mismatch! State file has (nx={data['nx']}, ny={data['ny']}, nz={data['nz']}) "
                f"but current simulation has (nx={self.nx}, ny={self.ny}, nz={self.nz})")
        self.ch.stats_write({k: data[k] for k in _SUMS}, int(data["n_samples"]))
