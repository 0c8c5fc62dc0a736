"""Field, time-series, statistics and grid files in the reference's formats.

* ``save_flow_fields`` / ``load_flow_fields``: ``np.savez`` with keys
  u, v, w, p, z_c, z_f, Lx, Ly, step, time, u_tau, forcing (reference layout,
  float64) as ``utils.py:369-444`` writes and reads them.  Extra keys written
  by ``save_flow_fields(..., extra=...)`` (the AB2 history) are ignored by the
  reference's reader, which only indexes the keys above.
* ``append_timeseries``: ``np.savez_compressed`` of step, time, u_bulk,
  u_tau, forcing, appended to an existing file (``solver.py:889-929``).
* ``save_grid_csv``: the ``grid.csv`` of ``utils.py:115-139``.
"""
import csv
import os
import zipfile

import numpy as np


def _np(x):
    if hasattr(x, "detach"):
        return x.detach().cpu().numpy()
    return np.asarray(x)


def _scalar(x):
    if hasattr(x, "item"):
        return x.item()
    return x


def save_flow_fields(u, v, w, p, z_c, z_f, Lx, Ly, step, time, u_tau, forcing, results_folder,
                     filename="fields.npz", extra=None):
    path = os.path.join(results_folder, filename)
    d = dict(u=_np(u), v=_np(v), w=_np(w), p=_np(p), z_c=_np(z_c), z_f=_np(z_f), Lx=Lx, Ly=Ly,
             step=step, time=time, u_tau=_scalar(u_tau), forcing=_scalar(forcing))
    if extra:
        d.update({k: _np(a) for k, a in extra.items()})
    np.savez(path, **d)
    return path


FIELD_KEYS = ("u", "v", "w", "p", "z_c", "z_f", "Lx", "Ly", "step", "time", "u_tau", "forcing")


def load_flow_fields(filepath):
    """Read a ``fields*.npz`` (``utils.py:402-444``).  A missing file raises
    FileNotFoundError as in the reference; a truncated or corrupt archive, a
    missing key, or a field with an inconsistent shape raises ValueError
    naming the file, instead of the reference's unchecked ``np.load``
    indexing (which fails late or not at all)."""
    if not os.path.exists(filepath):
        raise FileNotFoundError(f"Field file not found: {filepath}")
    try:
        with np.load(filepath) as data:
            missing = [k for k in FIELD_KEYS if k not in data.files]
            if missing:
                raise ValueError(f"missing keys {missing}")
            out = {k: np.array(data[k]) for k in ("u", "v", "w", "p", "z_c", "z_f")}
            out.update(Lx=float(data["Lx"]), Ly=float(data["Ly"]), step=int(data["step"]),
                       time=float(data["time"]), u_tau=float(data["u_tau"]), forcing=float(data["forcing"]))
            for k in data.files:
                if k not in out:
                    out[k] = np.array(data[k])
    except (zipfile.BadZipFile, EOFError, OSError, ValueError, KeyError) as e:
        raise ValueError(f"Cannot read field file {filepath}: {e}") from e
    u, v, w, p = out["u"], out["v"], out["w"], out["p"]
    if u.ndim != 3 or v.ndim != 3 or w.ndim != 3 or p.ndim != 3:
        raise ValueError(f"Field file {filepath}: u, v, w, p must be 3-D")
    nx, ny, nz = u.shape[0] - 1, u.shape[1] - 2, u.shape[2] - 2
    want = {"v": (nx + 2, ny + 1, nz + 2), "w": (nx + 2, ny + 2, nz + 1), "p": (nx + 2, ny + 2, nz + 2)}
    for k, s in want.items():
        if out[k].shape != s:
            raise ValueError(f"Field file {filepath}: {k} has shape {out[k].shape}, expected {s} for "
                             f"u of shape {u.shape}")
    return out


def append_timeseries(path, chunk):
    keys = ("step", "time", "u_bulk", "u_tau", "forcing")
    if os.path.exists(path):
        old = np.load(path)
        merged = {k: np.concatenate([old[k], chunk[k]]) for k in keys}
    else:
        merged = {k: chunk[k] for k in keys}
    np.savez_compressed(path, **merged)


def save_grid_csv(z_f, z_c, dz_f, dz_c, results_folder):
    arrs = [np.asarray(a, dtype=np.float64) for a in (z_f, z_c, dz_f, dz_c)]
    n = max(len(a) for a in arrs)
    pad = [np.concatenate([a, np.full(n - len(a), np.nan)]) for a in arrs]
    path = os.path.join(results_folder, "grid.csv")
    with open(path, "w", newline="") as f:
        wr = csv.writer(f)
        wr.writerow(["z_f", "z_c", "dz_f", "dz_c"])
        for i in range(n):
            wr.writerow([pad[0][i], pad[1][i], pad[2][i], pad[3][i]])
    return path
