"""File formats shared with the reference (CPU): our writers produce the keys
and dtypes the reference writes, and our reader loads the reference's files."""
import os

import numpy as np

from torchannel_b200 import io as tio
from torchannel_b200.grid import generate_grid, generate_hybrid_grid


def test_reference_files_load(golden):
    S = golden("run_16x12x10.npz")
    # the golden run stored the reference's own fields_final.npz under final_*
    keys = {k[len("final_"):] for k in S if k.startswith("final_") and k != "final_dt"}
    assert keys == {"u", "v", "w", "p", "z_c", "z_f", "Lx", "Ly", "step", "time", "u_tau", "forcing"}


def test_fields_roundtrip(tmp_path):
    nx, ny, nz = 8, 6, 5
    rng = np.random.default_rng(0)
    u, v, w, p = (rng.standard_normal(s) for s in ((nx + 1, ny + 2, nz + 2), (nx + 2, ny + 1, nz + 2),
                                                     (nx + 2, ny + 2, nz + 1), (nx + 2, ny + 2, nz + 2)))
    z_f, z_c, _, _ = generate_grid(2.6, nz, 2.0)
    path = tio.save_flow_fields(u, v, w, p, z_c, z_f, 1.0, 2.0, 7, 0.5, 0.03, 1e-3, str(tmp_path), "f.npz",
                                extra={"rhs_u_prev": u})
    d = np.load(path)
    assert d["u"].dtype == np.float64 and d["u"].shape == u.shape
    assert int(d["step"]) == 7 and float(d["time"]) == 0.5
    back = tio.load_flow_fields(path)
    assert np.array_equal(back["w"], w) and back["Ly"] == 2.0 and "rhs_u_prev" in back


def test_timeseries_append(tmp_path):
    p = str(tmp_path / "ts.npz")
    c = {"step": np.array([5, 10], dtype=np.int32), "time": np.array([0.1, 0.2]), "u_bulk": np.ones(2),
         "u_tau": np.ones(2) * 0.03, "forcing": np.zeros(2)}
    tio.append_timeseries(p, c)
    tio.append_timeseries(p, c)
    d = np.load(p)
    assert list(d["step"]) == [5, 10, 5, 10] and d["step"].dtype == np.int32


def test_grid_csv(tmp_path):
    z_f, z_c, dz_f, dz_c = generate_grid(2.6, 10, 2.0)
    path = tio.save_grid_csv(z_f, z_c, dz_f, dz_c, str(tmp_path))
    lines = open(path).read().splitlines()
    assert lines[0] == "z_f,z_c,dz_f,dz_c" and len(lines) == 1 + 12


def test_product_grid_matches_reference(golden):
    G = golden("ops_16x12x10.npz")
    for st in ("symmetric", "bottom"):
        z_f, z_c, dz_f, dz_c = generate_grid(2.6, 48, 2.0, st)
        assert np.max(np.abs(z_f - G[f"grid_{st}_z_f"])) < 1e-14
        assert np.max(np.abs(dz_c - G[f"grid_{st}_dz_c"])) < 1e-14
    z_f, z_c, dz_f, dz_c = generate_hybrid_grid(20, 30, 0.25, 2.0, 1.8)
    assert np.max(np.abs(z_f - G["grid_hybrid_z_f"])) < 1e-14


def test_initialize_flow_matches_oracle():
    from oracle.step import initial_fields
    from torchannel_b200.init import initialize_flow
    nx, ny, nz = 16, 12, 10
    z_f, z_c, _, _ = generate_grid(2.6, nz, 2.0)
    for top in ("dirichlet", "neumann"):
        a = initialize_flow(nx, ny, nz, z_c, 4 * np.pi / 3, 2.0, 1.0, "parabolic", 0.1, seed=4, top_wall_bc_type=top)
        b = initial_fields(nx, ny, nz, z_c, 2.0, 1.0, 0.1, seed=4, top_wall_bc_type=top)
        for x, y in zip(a, b):
            assert np.array_equal(x, y)
