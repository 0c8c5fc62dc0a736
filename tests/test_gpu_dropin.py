"""``ChannelFlowB200`` against the reference's own ``run_simulation`` (golden
vectors from tests/golden/make_golden.py): same YAML, same initial field, same
adaptive-dt loop, statistics and saves; the files written are compared."""
import os

import numpy as np
import pytest
import yaml

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _cfg(path, res, nx, ny, nz, field_file=None, **over):
    cfg = {
        "grid": {"nx": nx, "ny": ny, "nz": nz},
        "domain": {"Lx": float(4 * np.pi), "Ly": float(4 * np.pi / 3), "Lz": 2.0, "stretching_type": "symmetric"},
        "flow": {"Re": 2870.0, "Re_tau": 180.0, "U_bulk": 1.0, "gamma": 2.6},
        "boundary_conditions": {"top_wall": {"type": "dirichlet"}},
        "initialization": {"type": "parabolic", "perturbation_intensity": 0.1},
        "solver": {"type": "fft"},
        "time": {"dt": 0.002, "n_steps": 20, "CFL_target": 0.25, "dt_update_interval": 5, "dt_max": 0.011,
                 "dt_min": 0.0003, "scheme": "IMEX"},
        "compute": {"device": "cuda"},
        "output": {"results_folder": res, "n_out": 5, "n_save": 10},
        "statistics": {"n_stats": 5, "t_stats": 0.0, "z_plus_target": 15.0},
    }
    if field_file:
        cfg["initialization"]["field_file"] = field_file
    for k, v in over.items():
        sec, key = k.split("__")
        cfg[sec][key] = v
    with open(path, "w") as f:
        yaml.safe_dump(cfg, f)
    return path


def _start_file(tmp_path, S):
    from torchannel_b200 import io as tio
    from torchannel_b200.grid import generate_grid
    z_f, z_c, _, _ = generate_grid(2.6, int(S["nz"]), 2.0)
    return tio.save_flow_fields(S["u0"], S["v0"], S["w0"], np.zeros((int(S["nx"]) + 2, int(S["ny"]) + 2,
                                                                    int(S["nz"]) + 2)),
                                z_c, z_f, float(4 * np.pi), float(4 * np.pi / 3), 0, 0.0, 0.0, 0.0,
                                str(tmp_path), "start.npz")


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(np.asarray(b))), 1e-300))


def test_run_simulation_matches_reference(torch_cuda, golden, tmp_path):
    from torchannel_b200.solver import ChannelFlowB200
    S = golden("run_16x12x10.npz")
    nx, ny, nz = int(S["nx"]), int(S["ny"]), int(S["nz"])
    start = _start_file(tmp_path, S)
    res = str(tmp_path / "res")
    cf = ChannelFlowB200(_cfg(str(tmp_path / "c.yaml"), res, nx, ny, nz, field_file=start), verbose=False)
    cf.run_simulation()
    assert abs(cf.dt - float(S["final_dt"])) < 1e-15
    fin = np.load(os.path.join(res, "fields_final.npz"))
    for c in "uvw":
        assert rel(fin[c], S["final_" + c]) < 1e-10, c
    assert int(fin["step"]) == int(S["final_step"]) and abs(float(fin["time"]) - float(S["final_time"])) < 1e-12
    assert abs(float(fin["u_tau"]) - float(S["final_u_tau"])) < 1e-10
    ts = np.load(os.path.join(res, "timeseries.npz"))
    assert np.array_equal(ts["step"], S["ts_step"])
    assert np.allclose(ts["time"], S["ts_time"], rtol=0, atol=1e-12)
    assert np.allclose(ts["u_bulk"], S["ts_u_bulk"], rtol=0, atol=1e-12)
    assert np.allclose(ts["u_tau"], S["ts_u_tau"], rtol=0, atol=1e-10)
    assert np.allclose(ts["forcing"], S["ts_forcing"], rtol=1e-8, atol=1e-12)
    st = np.load(os.path.join(res, "turbulence_stats.npz"))
    for k in ("U_mean", "uu_mean", "vv_mean", "ww_mean", "uw_mean", "E_uu_2d", "E_vv_2d", "E_ww_2d", "E_uw_2d"):
        assert rel(st[k], S["stats_" + k]) < 1e-9, k
    for k in ("n_samples", "z_plus_target"):
        assert int(st[k]) == int(S["stats_" + k]), k
    for k in ("kx", "ky", "z_c"):
        assert rel(st[k], S["stats_" + k]) < 1e-14, k
    assert abs(float(st["u_tau"]) - float(S["stats_u_tau"])) < 1e-9
    sv = np.load(os.path.join(res, "turbulence_stats_state.npz"))
    assert set(sv.files) == {k[len("state_"):] for k in S if k.startswith("state_")}
    assert rel(sv["U_sum"], S["state_U_sum"]) < 1e-9
    sv_f = np.load(os.path.join(res, "fields.npz"))
    assert set(sv_f.files) >= {"u", "v", "w", "p", "z_c", "z_f", "Lx", "Ly", "step", "time", "u_tau", "forcing"}


def test_restart_with_history_is_bit_continuous(torch_cuda, tmp_path):
    from torchannel_b200.solver import ChannelFlowB200
    nx, ny, nz = 24, 16, 12
    ref = ChannelFlowB200(_cfg(str(tmp_path / "a.yaml"), str(tmp_path / "a"), nx, ny, nz,
                               time__n_steps=12, time__dt_update_interval=0, output__n_save=6,
                               statistics__n_stats=0), verbose=False)
    ref.run_simulation()
    # first half, saving the AB2 history with the fields
    r1 = ChannelFlowB200(_cfg(str(tmp_path / "b.yaml"), str(tmp_path / "b"), nx, ny, nz,
                              time__n_steps=6, time__dt_update_interval=0, output__n_save=6,
                              output__save_history=True, statistics__n_stats=0), verbose=False)
    r1.run_simulation()
    r2 = ChannelFlowB200(_cfg(str(tmp_path / "c.yaml"), str(tmp_path / "c"), nx, ny, nz,
                              field_file=str(tmp_path / "b" / "fields.npz"), time__n_steps=12,
                              time__dt_update_interval=0, output__n_save=6, statistics__n_stats=0), verbose=False)
    r2.run_simulation()
    a = np.load(str(tmp_path / "a" / "fields_final.npz"))
    c = np.load(str(tmp_path / "c" / "fields_final.npz"))
    for k in "uvw":
        # the restart re-projects the loaded field (solver.py:342-375): roundoff only
        assert np.max(np.abs(a[k] - c[k])) < 1e-13, k
    assert int(c["step"]) == 12


def test_field_accessors_and_schemes(torch_cuda, tmp_path):
    from torchannel_b200.solver import ChannelFlowB200
    cf = ChannelFlowB200(_cfg(str(tmp_path / "d.yaml"), str(tmp_path / "d"), 24, 16, 12, statistics__n_stats=0),
                         verbose=False)
    u = cf.u
    assert tuple(u.shape) == (25, 18, 14) and tuple(cf.v.shape) == (26, 17, 14) and tuple(cf.w.shape) == (26, 18, 13)
    ub, f = cf.step_imex(0.002)
    assert abs(float(ub) - 1.0) < 1e-3
    ub, f = cf.step_forward_euler(0.0005)
    assert f == 1.0
    with pytest.raises(NotImplementedError):
        cf.step_rk3(0.001)
    dt = cf.compute_cfl_dt()
    assert cf.dt_min <= dt <= cf.dt_max


def test_nonfinite_state_writes_error_file_and_stops(torch_cuda, tmp_path):
    """A NaN in the field is caught at the next save point: fields_error.npz
    is written with the reference's keys and the loop stops there
    (solver.py:862-881); no fields.npz is written for that step."""
    from torchannel_b200.solver import ChannelFlowB200
    res = str(tmp_path / "e")
    cf = ChannelFlowB200(_cfg(str(tmp_path / "e.yaml"), res, 24, 16, 12, time__n_steps=20,
                              time__dt_update_interval=0, output__n_save=4, output__n_out=2,
                              statistics__n_stats=0), verbose=False)
    u = cf.u.cpu().numpy()
    u[5, 6, 7] = np.nan
    cf.set_fields(u, cf.v, cf.w)
    last = cf.run_simulation()
    assert last == 4 and cf.current_step == 4
    err = np.load(os.path.join(res, "fields_error.npz"))
    assert set(err.files) == {"u", "v", "w", "p", "z_c", "z_f", "Lx", "Ly", "step", "time", "u_tau", "forcing"}
    assert int(err["step"]) == 4
    assert not np.all(np.isfinite(err["u"]))
    assert not os.path.exists(os.path.join(res, "fields.npz"))
