"""Host-side failure handling (CPU): corrupt restart files and mismatched
statistics states are refused with a clear error before any device work
(utils.py:402-444, turbstats.py:364-402)."""
import os

import numpy as np
import pytest

from torchannel_b200 import io as tio
from torchannel_b200.grid import generate_grid
from torchannel_b200.stats import TurbulenceStatsB200


def _fields(tmp_path, nx=8, ny=6, nz=5, name="fields.npz", **over):
    rng = np.random.default_rng(0)
    arr = dict(u=rng.standard_normal((nx + 1, ny + 2, nz + 2)), v=rng.standard_normal((nx + 2, ny + 1, nz + 2)),
               w=rng.standard_normal((nx + 2, ny + 2, nz + 1)), p=rng.standard_normal((nx + 2, ny + 2, nz + 2)))
    arr.update(over)
    z_f, z_c, _, _ = generate_grid(2.6, nz, 2.0)
    return tio.save_flow_fields(arr["u"], arr["v"], arr["w"], arr["p"], z_c, z_f, 1.0, 2.0, 3, 0.25, 0.03, 1e-3,
                                str(tmp_path), name)


def test_truncated_field_file_raises(tmp_path):
    path = _fields(tmp_path)
    size = os.path.getsize(path)
    for keep in (size // 2, size - 30, 100):
        bad = str(tmp_path / f"trunc_{keep}.npz")
        with open(path, "rb") as f, open(bad, "wb") as g:
            g.write(f.read(keep))
        with pytest.raises(ValueError, match="Cannot read field file"):
            tio.load_flow_fields(bad)


def test_garbage_field_file_raises(tmp_path):
    bad = str(tmp_path / "garbage.npz")
    with open(bad, "wb") as f:
        f.write(np.random.default_rng(1).bytes(4096))
    with pytest.raises(ValueError):
        tio.load_flow_fields(bad)


def test_missing_field_file_raises(tmp_path):
    with pytest.raises(FileNotFoundError):
        tio.load_flow_fields(str(tmp_path / "absent.npz"))


def test_field_file_missing_key_raises(tmp_path):
    path = str(tmp_path / "nokey.npz")
    np.savez(path, u=np.zeros((9, 8, 7)), v=np.zeros((10, 7, 7)))
    with pytest.raises(ValueError, match="missing keys"):
        tio.load_flow_fields(path)


def test_field_file_inconsistent_shapes_raise(tmp_path):
    path = _fields(tmp_path, name="shape.npz", w=np.zeros((10, 8, 7)))   # w of nz = 6 beside u of nz = 5
    with pytest.raises(ValueError, match="w has shape"):
        tio.load_flow_fields(path)


class _FakeChannel:
    """The slice of ``core.Channel`` the statistics binding uses, without a
    device: stats_init picks fixed planes, stats_read / stats_write keep the
    sums in host memory."""

    def __init__(self, nx, ny, nz):
        self.nx, self.ny, self.nz = nx, ny, nz
        self.Lx, self.Ly, self.Lz, self.nu = 4 * np.pi, 4 * np.pi / 3, 2.0, 1 / 2870.0
        self.sums = {k: np.zeros(nz) for k in ("U_sum", "uu_sum", "vv_sum", "ww_sum", "uw_sum")}
        self.sums.update({k: np.zeros((nx // 2, ny // 2))
                          for k in ("E_uu_2d_sum", "E_vv_2d_sum", "E_ww_2d_sum", "E_uw_2d_sum")})
        self.n = 0
        self.writes = 0

    def stats_init(self, z_c, Re_tau, zp):
        return 2, self.nz - 1

    def stats_read(self):
        return dict(self.sums, n_samples=self.n)

    def stats_write(self, sums, n):
        self.sums = {k: np.asarray(v) for k, v in sums.items()}
        self.n = n
        self.writes += 1


def test_stats_state_grid_mismatch_raises(tmp_path):
    z_f, z_c, _, _ = generate_grid(2.6, 10, 2.0)
    a = TurbulenceStatsB200(_FakeChannel(16, 12, 10), z_c, 180.0)
    a.ch.n = 4
    a.ch.sums["U_sum"][:] = 1.5
    path = str(tmp_path / "state.npz")
    a.save_state(path)
    # same grid: loads the sums
    b = TurbulenceStatsB200(_FakeChannel(16, 12, 10), z_c, 180.0)
    b.load_state(path)
    assert b.ch.n == 4 and np.all(b.ch.sums["U_sum"] == 1.5)
    # other grid: ValueError (turbstats.py:379-383), nothing written
    for shape in ((16, 12, 12), (32, 12, 10), (16, 24, 10)):
        z_f2, z_c2, _, _ = generate_grid(2.6, shape[2], 2.0)
        c = TurbulenceStatsB200(_FakeChannel(*shape), z_c2, 180.0)
        with pytest.raises(ValueError, match="Grid dimension mismatch"):
            c.load_state(path)
        assert c.ch.writes == 0


def test_stats_state_missing_file_raises(tmp_path):
    z_f, z_c, _, _ = generate_grid(2.6, 10, 2.0)
    a = TurbulenceStatsB200(_FakeChannel(16, 12, 10), z_c, 180.0)
    with pytest.raises(FileNotFoundError):
        a.load_state(str(tmp_path / "none.npz"))
