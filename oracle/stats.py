"""Turbulence statistics accumulator (oracle restatement, test infrastructure
only).  Follows ``turbstats.py:5-402`` of the reference."""
import numpy as np


def stats_plane_indices(nz, Lz, z_c, nu, Re_tau_target, z_plus_target=15.0):
    """k_bot / k_top (ghost-offset z_c indices nearest to z+ from each wall);
    ``turbstats.py:52-69``."""
    u_tau_target = Re_tau_target * nu / (Lz / 2.0)
    zt = z_plus_target * nu / u_tau_target
    zci = z_c[1:nz+1]
    k_bot = int(np.argmin(np.abs(zci - zt))) + 1
    k_top = int(np.argmin(np.abs(zci - (Lz - zt)))) + 1
    return k_bot, k_top, u_tau_target


class TurbulenceStats:
    """Running sums of U(z), u'u', v'v', w'w', u'w' and 2-D spectra at z+."""

    def __init__(self, nx, ny, nz, Lx, Ly, Lz, z_c, dx, dy, nu, Re_tau_target,
                 z_plus_target=15.0):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.Lz, self.z_c, self.nu = Lz, z_c, nu
        self.k_bot, self.k_top, self.u_tau_target = stats_plane_indices(
            nz, Lz, z_c, nu, Re_tau_target, z_plus_target)
        self.n_samples = 0
        self.U_sum = np.zeros(nz); self.uu_sum = np.zeros(nz)
        self.vv_sum = np.zeros(nz); self.ww_sum = np.zeros(nz)
        self.uw_sum = np.zeros(nz)
        shp = (nx // 2, ny // 2)
        self.E_uu_2d_sum = np.zeros(shp); self.E_vv_2d_sum = np.zeros(shp)
        self.E_ww_2d_sum = np.zeros(shp); self.E_uw_2d_sum = np.zeros(shp)
        self.kx = 2 * np.pi * np.fft.rfftfreq(nx, d=dx)[1:]     # turbstats.py:98
        self.ky = 2 * np.pi * np.fft.rfftfreq(ny, d=dy)[1:]

    def accumulate_statistics(self, u, v, w):
        """``turbstats.py:101-228``."""
        nx, ny, nz = self.nx, self.ny, self.nz
        ui = u[0:nx+1, 1:ny+1, 1:nz+1]
        vi = v[1:nx+1, 0:ny+1, 1:nz+1]
        wi = w[1:nx+1, 1:ny+1, 0:nz+1]
        uc = 0.5 * (ui[:-1] + ui[1:])                    # :120
        U = uc.mean(axis=(0, 1)); self.U_sum += U
        uf = uc - U
        vc = 0.5 * (vi[:, :-1] + vi[:, 1:])              # :130
        vf = vc - vc.mean(axis=(0, 1))
        wc = 0.5 * (wi[:, :, :-1] + wi[:, :, 1:])        # :135
        wf = wc - wc.mean(axis=(0, 1))
        self.uu_sum += (uf * uf).mean(axis=(0, 1))      # :140-148
        self.vv_sum += (vf * vf).mean(axis=(0, 1))
        self.ww_sum += (wf * wf).mean(axis=(0, 1))
        self.uw_sum += (uf * wf).mean(axis=(0, 1))
        kb, kt = self.k_bot - 1, self.k_top - 1
        norm = float(nx * ny) ** 2
        ub, vb, wb = (np.fft.rfft2(f[:, :, kb]) for f in (uf, vf, wf))      # :165-167
        ut, vt, wt = (np.fft.rfft2(f) for f in (uf[:, :, kt], vf[:, :, kt], -wf[:, :, kt]))  # :171-173
        Euu = 0.5 * (np.abs(ub) ** 2 + np.abs(ut) ** 2) / norm             # :176-191
        Evv = 0.5 * (np.abs(vb) ** 2 + np.abs(vt) ** 2) / norm
        Eww = 0.5 * (np.abs(wb) ** 2 + np.abs(wt) ** 2) / norm
        Euw = 0.5 * ((ub * np.conj(wb)).real + (ut * np.conj(wt)).real) / norm
        nkx, nky = nx // 2, ny // 2

        def fold(E):                                     # :201-214
            return E[1:nkx+1, 1:nky+1] + E[nx-nkx:nx, 1:nky+1][::-1]

        self.E_uu_2d_sum += fold(Euu)[:nkx, :nky]        # :222-225
        self.E_vv_2d_sum += fold(Evv)[:nkx, :nky]
        self.E_ww_2d_sum += fold(Eww)[:nkx, :nky]
        self.E_uw_2d_sum += fold(Euw)[:nkx, :nky]
        self.n_samples += 1

    def finalize(self):
        """``turbstats.py:230-303`` (means only)."""
        n = self.n_samples
        return dict(U_mean=self.U_sum / n, uu_mean=self.uu_sum / n,
                    vv_mean=self.vv_sum / n, ww_mean=self.ww_sum / n,
                    uw_mean=self.uw_sum / n, E_uu_2d=self.E_uu_2d_sum / n,
                    E_vv_2d=self.E_vv_2d_sum / n, E_ww_2d=self.E_ww_2d_sum / n,
                    E_uw_2d=self.E_uw_2d_sum / n)
