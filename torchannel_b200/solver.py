"""``ChannelFlowB200``: a drop-in for the reference's ``ChannelFlow``
(``solver.py:81-970``) whose time step runs in the B200 kernels.

Same YAML keys (``solver.py:83-331``), same step methods and return values,
same ``run_simulation`` loop (scheme selection, adaptive dt every
``dt_update_interval`` steps with the 5% rule, diagnostics every ``n_out``,
statistics every ``n_stats`` once ``time >= t_stats``, checkpoints every
``n_save`` with the NaN/Inf check), and the same output files
(``fields_init.npz``, ``fields.npz``, ``fields_final.npz``,
``fields_error.npz``, ``timeseries.npz``, ``turbulence_stats*.npz``,
``grid.csv``).  Matplotlib figures are not produced.

Additional keys (absent from the reference, ignored by it):
``compute.precision`` ("fp64" default, or "mixed"), ``compute.rhs_path``
("separate" default = the reference's CPU-path semantics, or "fused" = its
CUDA-path semantics), and ``output.save_history`` (store the AB2 history in
``fields*.npz`` so a restart continues bit-for-bit; the reference restarts with
an Euler step, ``solver.py:377-383``).  ``time.scheme: AB2`` selects the
fully explicit AB2 the reference documents but cannot select.

The fields ``u, v, w, p`` are properties: reading one materialises the
reference-layout float64 CUDA tensor (ghosts filled) from the device state;
assigning one loads it back.
"""
import os
import time as _time

import numpy as np
import torch
import yaml

from . import io as tio
from .core import Channel
from .grid import generate_grid, generate_hybrid_grid
from .init import initialize_flow
from .stats import TurbulenceStatsB200


class ChannelFlowB200:
    def __init__(self, config_file="config.yaml", seed=None, verbose=True):
        with open(config_file, "r") as f:
            config = yaml.safe_load(f)
        self.config = config
        self.verbose = verbose
        dev = config.get("compute", {}).get("device", "auto")
        if dev == "cpu" or not torch.cuda.is_available():
            raise RuntimeError("ChannelFlowB200 runs on a CUDA device (B200); no CPU path")
        self.device = torch.device("cuda")
        g = config["grid"]
        self.nx, self.ny, self.nz = int(g["nx"]), int(g["ny"]), int(g["nz"])
        d = config["domain"]
        self.Lx, self.Ly, self.Lz = float(d["Lx"]), float(d["Ly"]), float(d["Lz"])
        self.stretching_type = d.get("stretching_type", "symmetric")
        if self.stretching_type not in ("symmetric", "bottom", "hybrid"):
            raise ValueError(f"Invalid stretching type: {self.stretching_type}. "
                             "Must be 'symmetric', 'bottom', or 'hybrid'")
        fl = config["flow"]
        self.nu = 1.0 / fl["Re"]
        self.Re_tau = fl["Re_tau"]
        self.U_bulk = fl["U_bulk"]
        self.gamma = fl["gamma"]
        self.top_wall_bc_type = config.get("boundary_conditions", {}).get("top_wall", {}).get("type", "dirichlet")
        if self.top_wall_bc_type not in ("dirichlet", "neumann"):
            raise ValueError(f"Invalid top wall BC type: {self.top_wall_bc_type}. Must be 'dirichlet' or 'neumann'")
        t = config["time"]
        self.dt = t["dt"]
        self.n_steps = t["n_steps"]
        self.t_max = t.get("t_max", 1000.0)
        self.cfl_target = t["CFL_target"]
        self.dt_update_interval = t.get("dt_update_interval", 0)
        self.dt_max = t.get("dt_max", 0.01)
        self.dt_min = t.get("dt_min", 0.0001)
        self.time_scheme = t.get("scheme", "IMEX")
        out = config.get("output", {})
        self.results_folder = out.get("results_folder", "results")
        self.n_out = out.get("n_out", out.get("print_interval", 10))
        self.n_save = out.get("n_save", out.get("slice_interval", 100))
        self.save_history = bool(out.get("save_history", False))
        os.makedirs(self.results_folder, exist_ok=True)
        init = config.get("initialization", {})
        field_file = init.get("field_file", None)
        is_restart = field_file is not None
        if not is_restart and out.get("clean_results_on_fresh_start", False):
            for fn in os.listdir(self.results_folder):
                fp = os.path.join(self.results_folder, fn)
                if os.path.isfile(fp) or os.path.islink(fp):
                    os.unlink(fp)
        comp = config.get("compute", {})
        self.precision = comp.get("precision", "fp64")
        self.rhs_path = comp.get("rhs_path", "separate")
        solver_type = config.get("solver", {}).get("type", "fft")
        if solver_type != "fft":
            raise ValueError(f"Unknown or unsupported solver type: {solver_type} (the B200 step uses the FFT solver)")
        self.solver_type = solver_type

        # grid (solver.py:192-219)
        if self.stretching_type == "hybrid":
            self.z_f, self.z_c, self.dz_f, self.dz_c = generate_hybrid_grid(
                g.get("nz_uniform", 75), g.get("nz_stretched", 75), d.get("z_transition", 0.25), self.Lz,
                d.get("gamma_stretched", 1.8))
            self.nz = len(self.dz_f)
        else:
            self.z_f, self.z_c, self.dz_f, self.dz_c = generate_grid(self.gamma, self.nz, self.Lz,
                                                                     self.stretching_type)
        self.dx, self.dy = self.Lx / self.nx, self.Ly / self.ny
        self.total_volume = self.Lx * self.Ly * self.Lz
        tio.save_grid_csv(self.z_f, self.z_c, self.dz_f, self.dz_c, self.results_folder)

        self.ch = Channel(self.nx, self.ny, self.nz, self.Lx, self.Ly, self.Lz, self.nu, self.dz_f, self.dz_c,
                          U_bulk=self.U_bulk, top_wall_bc_type=self.top_wall_bc_type, precision=self.precision,
                          rhs_path=self.rhs_path)
        hist = None
        if is_restart:
            fields = tio.load_flow_fields(field_file)
            u, v, w = fields["u"], fields["v"], fields["w"]
            if init.get("reset_time", False):
                self.initial_step, self.time = 0, 0.0
            else:
                self.initial_step, self.time = int(fields["step"]), float(fields["time"])
            forcing0 = 0.0                                                 # solver.py:249
            if all(k in fields for k in ("rhs_u_prev", "rhs_v_prev", "rhs_w_prev")):
                hist = (fields["rhs_u_prev"], fields["rhs_v_prev"], fields["rhs_w_prev"])
                forcing0 = float(fields["forcing"])
        else:
            u, v, w, _ = initialize_flow(self.nx, self.ny, self.nz, self.z_c, self.Ly, self.Lz, U_bulk=self.U_bulk,
                                         init_type=init["type"],
                                         perturbation_intensity=init.get("perturbation_intensity", 0.0),
                                         n_vortices=init.get("n_vortices", 4),
                                         seed=0 if seed is None else seed,
                                         top_wall_bc_type=self.top_wall_bc_type)
            self.initial_step, self.time = 0, 0.0
            forcing0 = 0.0
        self.initial_time = self.time
        self.ch.set_state(u, v, w, forcing=forcing0)
        if not is_restart:                                                  # solver.py:271-276
            ub = self.ch.bulk_velocity()
            if abs(ub) > 1e-9:
                self.ch.set_state(np.asarray(u) * (self.U_bulk / ub), v, w, forcing=forcing0)

        # statistics (solver.py:297-333)
        st = config.get("statistics", {})
        self.n_stats = st.get("n_stats", 0)
        self.t_stats = st.get("t_stats", 10.0)
        self.turbulence_stats = None
        if self.n_stats > 0:
            self.stats_output_path = os.path.join(self.results_folder, st.get("output_file", "turbulence_stats.npz"))
            self.stats_state_path = os.path.join(self.results_folder,
                                                 st.get("state_file", "turbulence_stats_state.npz"))
            self.turbulence_stats = TurbulenceStatsB200(self.ch, self.z_c, self.Re_tau,
                                                        st.get("z_plus_target", 15.0))
            if st.get("restart_state_file", None) is not None:
                self.turbulence_stats.load_state(st["restart_state_file"])

        d0 = self.ch.diagnostics()
        tio.save_flow_fields(self.u, self.v, self.w, self.p, self.z_c, self.z_f, self.Lx, self.Ly, 0, 0.0,
                             d0["u_tau"], 0.0, self.results_folder, "fields_init.npz")
        # initial projection with dt = 1 (solver.py:342-375), done on restarts too
        self.ch.project_initial()
        self._log(f"Initial divergence after projection: max(|div|) = {self.ch.diagnostics()['max_div']:.6e}")
        if hist is not None:
            self.ch.set_history(*hist)
        self.current_step = self.initial_step

    # -- state views --------------------------------------------------------
    @property
    def u(self):
        return self.ch.get_field("u")

    @property
    def v(self):
        return self.ch.get_field("v")

    @property
    def w(self):
        return self.ch.get_field("w")

    @property
    def p(self):
        return self.ch.get_field("p")

    def set_fields(self, u, v, w, keep_forcing=True):
        f = self.forcing if keep_forcing else 0.0
        self.ch.set_state(u, v, w, forcing=f)

    @property
    def forcing(self):
        return float(self.ch.scalars[0].item())

    @forcing.setter
    def forcing(self, value):
        self.ch.set_forcing(value)

    def _log(self, msg):
        if self.verbose:
            print(msg, flush=True)

    # -- reference API --------------------------------------------------------
    def apply_bc_uvw(self):
        """Ghosts are implied by the DOF layout and filled whenever a field is
        read (apply_bc_all, solver.py:23-79): nothing to do."""

    def compute_cfl_dt(self):
        """``solver.py:465-496``."""
        dti = self.ch.cfl_inverse()
        if dti < 1e-10:
            dti = 1.0
        return min(max(self.cfl_target * (1.0 / dti), self.dt_min), self.dt_max)

    def _scalars_out(self):
        sc = self.ch.scalars
        return sc[1].clone(), sc[0].clone()

    def step_imex(self, dt):
        """``solver.py:580-710``; returns (u_bulk, forcing) as 0-d CUDA tensors."""
        self.ch.step("IMEX", dt)
        return self._scalars_out()

    def step_ab2(self, dt):
        """Fully explicit AB2 (docs/NUMERICAL_METHODS.md:260-284)."""
        self.ch.step("AB2", dt)
        return self._scalars_out()

    def step_forward_euler(self, dt):
        """``solver.py:537-576``; the reference's return raises NameError
        (``:578``); this returns (u_bulk, 1.0), the hard-coded forcing."""
        self.ch.step("FE", dt)
        return self.ch.scalars[1].clone(), 1.0

    def step_rk3(self, dt):
        raise NotImplementedError("RK3 scheme not yet implemented. Use 'AB2', 'IMEX', or 'FE' time stepping.")

    def run_simulation(self):
        """``solver.py:738-970``."""
        steps = {"IMEX": self.step_imex, "FE": self.step_forward_euler, "RK3": self.step_rk3,
                 "AB2": self.step_ab2}
        if self.time_scheme not in steps:
            raise ValueError(f"Unknown time stepping scheme: {self.time_scheme}. Use 'IMEX', 'FE', 'AB2' or 'RK3'.")
        step_function = steps[self.time_scheme]
        hdr = f"{'Step':>6} {'Time':>10} {'dt':>10} {'max(div)':>12} {'u_bulk':>10} {'u_tau':>10} {'forcing':>12}"
        self._log("=" * 90)
        self._log(f"Time stepping scheme: {self.time_scheme}  |  Grid: {self.nx}x{self.ny}x{self.nz}")
        self._log("=" * 90)
        self._log(hdr)
        chunk = self.n_save // self.n_out + 1
        ts = {"step": np.zeros(chunk, dtype=np.int32), "time": np.zeros(chunk), "u_bulk": np.zeros(chunk),
              "u_tau": np.zeros(chunk), "forcing": np.zeros(chunk)}
        ts_idx = 0
        start = _time.time()
        step = self.initial_step
        u_bulk_s = u_tau_s = forcing_s = max_div = 0.0
        while step < self.n_steps and self.time < self.t_max:
            step += 1
            self.current_step = step
            if step > 0 and step % (10 * self.n_out) == 0:
                self._log(hdr)
            if self.dt_update_interval > 0 and step % self.dt_update_interval == 0 and step > 0:
                dt_new = self.compute_cfl_dt()
                if abs(dt_new - self.dt) / self.dt > 0.05:
                    self.dt = dt_new
            u_bulk, forcing = step_function(self.dt)
            self.time += self.dt
            diag = None
            if step % self.n_out == 0:
                diag = self.ch.diagnostics()
                max_div, u_tau_s = diag["max_div"], diag["u_tau"]
                u_bulk_s = float(u_bulk.item()) if torch.is_tensor(u_bulk) else float(u_bulk)
                forcing_s = float(forcing.item()) if torch.is_tensor(forcing) else float(forcing)
                ts["step"][ts_idx] = step
                ts["time"][ts_idx] = self.time
                ts["u_bulk"][ts_idx] = u_bulk_s
                ts["u_tau"][ts_idx] = u_tau_s
                ts["forcing"][ts_idx] = forcing_s
                ts_idx += 1
            if self.n_stats > 0 and self.time >= self.t_stats and step % self.n_stats == 0:
                self.turbulence_stats.accumulate_statistics()
            if step % self.n_save == 0:
                d = diag if diag is not None else self.ch.diagnostics()
                if d["nonfinite"]:
                    self._log(f"ERROR: NaN or Inf detected in solution at step {step}, time = {self.time:.6f}")
                    ub_err = d["u_bulk"]
                    tio.save_flow_fields(self.u, self.v, self.w, self.p, self.z_c, self.z_f, self.Lx, self.Ly,
                                         step, self.time, d["u_tau"], (self.U_bulk - ub_err) / self.dt,
                                         self.results_folder, "fields_error.npz")
                    break
                if step % self.n_out != 0:
                    u_tau_s = d["u_tau"]
                    forcing_s = float(forcing.item()) if torch.is_tensor(forcing) else float(forcing)
                if ts_idx > 0:
                    tio.append_timeseries(os.path.join(self.results_folder, "timeseries.npz"),
                                          {k: a[:ts_idx] for k, a in ts.items()})
                    ts_idx = 0
                self._save("fields.npz", step, u_tau_s, forcing_s)
                if self.turbulence_stats is not None and self.turbulence_stats.n_samples > 0:
                    self.turbulence_stats.save_state(self.stats_state_path)
            if step % self.n_out == 0:
                self._log(f"{step:6d} {self.time:10.6f} {self.dt:10.6f} {max_div:12.3e} {u_bulk_s:10.6f} "
                          f"{u_tau_s:10.6f} {forcing_s:12.3e}")
        self.loop_seconds = _time.time() - start  # wall time of the step loop (before the final files)
        self._log("=" * 90)
        self._log(f"Simulation complete: {step} steps, total time = {self.time:.6f}, final dt = {self.dt:.6f}")
        self._log(f"Total wall time: {self.loop_seconds:.2f}s")
        if self.turbulence_stats is not None and self.turbulence_stats.n_samples > 0:
            self.turbulence_stats.save_state(self.stats_state_path)
            self.turbulence_stats.save_statistics(self.stats_output_path)
        d = self.ch.diagnostics()
        ubf = self.ch.bulk_velocity()
        self._save("fields_final.npz", step, d["u_tau"], (self.U_bulk - ubf) / self.dt)
        self.current_step = step
        return step

    def _save(self, name, step, u_tau, forcing):
        extra = None
        if self.save_history and self.time_scheme in ("IMEX", "AB2"):
            try:
                ru, rv, rw = self.ch.get_history()
                extra = {"rhs_u_prev": ru, "rhs_v_prev": rv, "rhs_w_prev": rw}
                forcing = self.forcing
            except RuntimeError:
                extra = None
        tio.save_flow_fields(self.u, self.v, self.w, self.p, self.z_c, self.z_f, self.Lx, self.Ly, step,
                             self.time, u_tau, forcing, self.results_folder, name, extra=extra)
