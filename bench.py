"""Throughput of the TorChannel IMEX time step on B200.

Workload (one "step" = one IMEX time step of the channel):
  192 x 192 x 128 staggered grid, Lx = 4 pi, Ly = 4 pi / 3, Lz = 2, tanh
  stretching gamma = 2.6, Re_bulk = 2870, U_bulk = 1; seeded laminar profile
  + 0.1 uniform noise, rescaled and projected divergence-free, then 10 IMEX
  warm-up steps to give a developed AB2 history; dt from the CFL rule
  (CFL 0.25, clamp [3e-4, 1.1e-2]) held fixed during the timed region.
Metric: grid-point-steps/s = nx*ny*nz*steps / seconds (whole job, all ranks).

Arms:
  default           this repo's CUDA path, mixed precision (FP32 velocity fields,
                    history, stencils and CN sweeps; FP64 Poisson, CN tables,
                    bulk forcing); the plain FP64 form is timed in the same run
                    as "fp64_plain" (--precision fp64 makes it the headline)
  --impl reference  the CPU oracle (numpy FP64 restatement of the reference
                    step, oracle/) on all usable host cores (one replica per
                    core), bounded sample

Multi-GPU: one process per GPU, each advancing its own independent channel
(ensemble replicas, no collective on the hot path); value = sum over ranks of
grid-point-steps / max-over-ranks time.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX, NY, NZ = 192, 192, 128
LX, LY, LZ = 4 * np.pi, 4 * np.pi / 3, 2.0
RE, GAMMA = 2870.0, 2.6
CFL, DT_MIN, DT_MAX = 0.25, 3e-4, 0.011
METRIC = "grid-point-steps/s at 192x192x128 IMEX step"
WORKLOAD = "IMEX channel step 192x192x128 (Re_bulk 2870, gamma 2.6, seeded laminar+0.1 noise)"
# algorithmic traffic of one IMEX step: 24 stored words per grid point
# (pass 1: 13, Poisson: 4, projection: 7)
WORDS_PER_POINT = 24


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--run-steps", type=int, default=2000, help="steps of --workload config1")
    ap.add_argument("--workload", default="step", choices=["step", "ensemble", "poisson", "adjoint", "config1"],
                    help="step: the headline IMEX step; ensemble: 16 uneven channels (config 4); "
                         "poisson: the FFT Poisson solve alone at 192x192x128 and 384x384x256 (config 2); "
                         "adjoint: gradient of a time-averaged kinetic energy, 96x96x64, 200 steps (config 3); "
                         "config1: the 2000-step run of config 1 through the drop-in solver, FP64 and mixed")
    ap.add_argument("--checkpoint-every", type=int, default=20)
    ap.add_argument("--adjoint-mode", default="auto", choices=["auto", "store", "recompute"])
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--no-fp64-compare", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--batch-only", default=None, metavar="ROWS,CTAS",
                    help="--workload ensemble: only the ensemble launches, with this fixed shape (CN rows bound, "
                         "CTAs per SM) and graphs off, every launch visible to a profiler")
    ap.add_argument("--no-tma-rhs", action="store_true",
                    help="stage the explicit-RHS tiles with per-thread loads instead of tensor copies")
    ap.add_argument("--tma-rhs-mode", type=int, default=0,
                    help="tile shape of the tensor-copy RHS (1..6, tc_use_tma_rhs; 0: the default shape)")
    ap.add_argument("--poisson-middle", type=int, default=None, choices=[0, 1, 2],
                    help="form of the Poisson middle (tc_use_fused_poisson: 0 three kernels, 1 cluster kernel, "
                         "2 two streaming passes; default: the library's choice)")
    ap.add_argument("--bulk-ffty", action="store_true",
                    help="y transforms staged by bulk copies (tc_use_bulk_ffty) instead of per-lane loads")
    ap.add_argument("--no-fp32-poisson", action="store_true",
                    help="skip the mixed step with the single-precision Poisson solve")
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the forward+adjoint cost ratio (96x96x64, 200 steps) of the step line")
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    return ap.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    return rank, world, local


def initial_state(seed=0):
    """Seeded laminar + noise field (initflow.py:4-104 semantics) on the host."""
    from torchannel_b200.grid import generate_grid
    from torchannel_b200.init import initialize_flow
    z_f, z_c, dz_f, dz_c = generate_grid(GAMMA, NZ, LZ)
    u, v, w, p = initialize_flow(NX, NY, NZ, z_c, LY, LZ, U_bulk=1.0, init_type="parabolic",
                                 perturbation_intensity=0.1, seed=seed)
    return (z_f, z_c, dz_f, dz_c), (u, v, w)


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out = ""
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1])); mx = float(f[2])
            except ValueError:
                continue
            for n, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def load_profile_traffic(precision):
    """DRAM bytes per step from the committed ncu summary (None if absent)."""
    p = os.path.join(ROOT, "profiles", f"step_traffic_192x192x128_{precision}.json")
    if os.path.exists(p):
        return json.load(open(p))
    return None


# ---------------------------------------------------------------------------
# CUDA arm
# ---------------------------------------------------------------------------
def run_b200(a):
    import torch
    import torch.distributed as dist
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl" if torch.cuda.is_available() else "gloo",
                                timeout=__import__("datetime").timedelta(seconds=120))
    from torchannel_b200.core import Channel
    from torchannel_b200 import _lib as L
    grid, (u0, v0, w0) = initial_state(seed=rank)
    z_f, z_c, dz_f, dz_c = grid
    ch = Channel(NX, NY, NZ, LX, LY, LZ, 1.0 / RE, dz_f, dz_c, precision=a.precision)
    if a.no_tma_rhs:
        ch.use_tma_rhs(False)
    elif a.tma_rhs_mode:
        ch.use_tma_rhs(a.tma_rhs_mode)
    if a.poisson_middle is not None:
        ch.use_fused_poisson(a.poisson_middle)
    if a.bulk_ffty:
        ch.use_bulk_ffty(True)
    ch.set_state(u0, v0, w0)
    ub = ch.bulk_velocity()
    ch.set_state(u0 * (1.0 / ub), v0, w0)
    ch.project_initial()
    dt = min(max(CFL * (1.0 / ch.cfl_inverse()), DT_MIN), DT_MAX)
    ch.step("IMEX", dt, 10)
    for _ in range(a.warmup):
        ch.step("IMEX", dt)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        e0.record(stream)
        ch.step("IMEX", dt, a.steps)
        e1.record(stream)
        torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    diag = ch.diagnostics()  # after 10 + warmup + steps steps, as the FP64 comparison below
    stats = None
    if not a.no_fp64_compare and a.precision == "mixed":
        ch.stats_init(z_c, 180.0, 15.0)
        ch.stats_accumulate()
        stats = ch.stats_read()
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    # the other precision on the same state and dt, for the mixed-vs-FP64 comparison
    other = None
    if not a.no_fp64_compare and a.precision == "mixed":
        ch2 = Channel(NX, NY, NZ, LX, LY, LZ, 1.0 / RE, dz_f, dz_c, precision="fp64")
        ch2.set_state(u0, v0, w0)
        ub2 = ch2.bulk_velocity()
        ch2.set_state(u0 * (1.0 / ub2), v0, w0)
        ch2.project_initial()
        ch2.step("IMEX", dt, 10 + a.warmup)
        torch.cuda.synchronize()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        ch2.step("IMEX", dt, a.steps)
        f1.record(stream)
        torch.cuda.synchronize()
        ms2 = f0.elapsed_time(f1)
        if world > 1:
            t = torch.tensor([ms2], device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms2 = float(t.item())
        d2 = ch2.diagnostics()
        ch2.stats_init(z_c, 180.0, 15.0)
        ch2.stats_accumulate()
        st2 = ch2.stats_read()
        other = {"value": NX * NY * NZ * a.steps * world / (ms2 / 1e3), "ms_per_step": ms2 / a.steps,
                 "max_div_after": d2["max_div"], "u_bulk": d2["u_bulk"], "u_tau": d2["u_tau"]}

        def rerr(k):
            return float(np.max(np.abs(stats[k] - st2[k])) / np.max(np.abs(st2[k])))
        other["profile_rel_err"] = {"U": rerr("U_sum"), "uu": rerr("uu_sum"), "vv": rerr("vv_sum"),
                                    "ww": rerr("ww_sum"), "uw": rerr("uw_sum"), "E_uu_2d": rerr("E_uu_2d_sum")}
        del ch2
    # mixed precision with the single-precision Poisson step (FP32 spectrum,
    # FP64 low modes, increment over the previous pressure; the 10 set-up
    # steps use the FP64 solve), same state and dt
    psp = None
    if a.precision == "mixed" and not a.no_fp32_poisson:
        psp = time_fp32_poisson(a, grid, (u0, v0, w0), dt, world, stats)
    # per-phase timing (separate, instrumented pass of the same steps)
    ch.timing(True)
    ch.step("IMEX", dt, min(a.steps, L_RING))
    phases, nst = ch.timing_read()
    ch.timing(False)
    # end-to-end through the public API with host buffers
    e2e = None if a.no_e2e else run_e2e(a, grid, (u0, v0, w0), dt)
    # the second half of the metric: forward + adjoint cost over a forward run
    del ch
    adj = None if a.no_adjoint else measure_adjoint(a, rank, world)["summary"]
    if world > 1:
        dist.destroy_process_group()
    if rank != 0:
        return
    npts = NX * NY * NZ
    sec = ms / 1e3
    value = npts * a.steps * world / sec
    s = 8 if a.precision == "fp64" else 4
    peak, peak_kind = measured_peaks()
    step_bytes = WORDS_PER_POINT * s * npts
    step_ms = ms / a.steps
    kern = kernel_table(phases, nst, s, npts)
    dom = max(kern, key=lambda k: k["ms"])
    prof = load_profile_traffic(a.precision)
    traffic_dom = None
    if prof and dom["name"] in prof.get("per_kernel_bytes", {}):
        traffic_dom = prof["per_kernel_bytes"][dom["name"]]
    roof = {"bound": "hbm", "achieved": dom["gbs"], "peak": peak, "unit": "GB/s",
            "frac": dom["gbs"] / peak, "traffic": traffic_dom, "kernel": dom["name"],
            "peak_source": peak_kind,
            "algorithmic_bytes_per_launch": dom["bytes"], "avg_launch_ms": dom["ms"]}
    step_roof = {"bound": "hbm", "achieved": step_bytes / (step_ms / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                 "frac": step_bytes / (step_ms / 1e3) / 1e9 / peak, "words_per_point": WORDS_PER_POINT,
                 "bytes_per_step": step_bytes, "traffic": prof.get("bytes_per_step") if prof else None}
    cpu = None if a.no_cpu_baseline else cpu_baseline(a.cpu_seconds)
    line = {
        "metric": METRIC, "value": value, "unit": "grid-point-steps/s", "n_gpus": world, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if a.precision == "fp64" else "f32+f64",
        "data": "synthetic (seeded laminar profile + 0.1 uniform noise, projected)",
        "config": {"workload": WORKLOAD, "nx": NX, "ny": NY, "nz": NZ, "scheme": "IMEX",
                   "precision": a.precision, "dt": dt, "parallelism": f"replicas{world}",
                   "l2": "inputs larger than L2 (a step touches both state buffers, the history, the spectrum and p: > 126 MB)"},
        "roofline": roof, "step_roofline": step_roof, "kernels": kern,
        "cpu_baseline": cpu, "e2e": e2e,
        "clocks": clk.summary(),
        "gpu_launches": LAUNCHES_PER_STEP * a.steps,
        "max_div_after": diag["max_div"],
        "adjoint": adj,
        "mixed_fp32_poisson": psp,
    }
    if other is not None:
        line["fp64_plain"] = other
        line["mixed_speedup_over_fp64"] = value / other["value"]
        line["mixed_vs_fp64_after_steps"] = {"steps": 10 + a.warmup + a.steps,
                                             "max_div_mixed": diag["max_div"], "max_div_fp64": other["max_div_after"],
                                             "u_bulk_abs_err": abs(diag["u_bulk"] - other["u_bulk"]),
                                             "u_tau_rel_err": abs(diag["u_tau"] - other["u_tau"]) / other["u_tau"],
                                             "profile_rel_err": other.pop("profile_rel_err")}
    print(json.dumps(line), flush=True)


def time_fp32_poisson(a, grid, fields, dt, world, stats_mixed):
    """The mixed step with the single-precision Poisson solve: set-up as the
    headline run (initial projection, 10 steps, which are the FP64 warm-up of
    the increment's base), warm-up, then K timed steps; returns its speed,
    divergence, per-kernel table and its statistics' distance from the FP64
    Poisson run's."""
    import torch
    import torch.distributed as dist
    from torchannel_b200.core import Channel
    z_f, z_c, dz_f, dz_c = grid
    u0, v0, w0 = fields
    ch = Channel(NX, NY, NZ, LX, LY, LZ, 1.0 / RE, dz_f, dz_c, precision="mixed")
    ch.set_state(u0, v0, w0)
    ub = ch.bulk_velocity()
    ch.set_state(u0 * (1.0 / ub), v0, w0)
    ch.project_initial()
    ch.use_fp32_poisson(True, warm_steps=10)
    ch.step("IMEX", dt, 10 + a.warmup)
    torch.cuda.synchronize()
    stream = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ch.step("IMEX", dt, a.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    d = ch.diagnostics()
    out = {"value": NX * NY * NZ * a.steps * world / (ms / 1e3), "ms_per_step": ms / a.steps,
           "max_div_after": d["max_div"], "u_bulk": d["u_bulk"], "u_tau": d["u_tau"],
           "error_word": ch.error_word()}
    if stats_mixed is not None:
        ch.stats_init(z_c, 180.0, 15.0)
        ch.stats_accumulate()
        st = ch.stats_read()

        def rerr(k):
            return float(np.max(np.abs(st[k] - stats_mixed[k])) / np.max(np.abs(stats_mixed[k])))
        out["profile_rel_err_vs_fp64_poisson"] = {"U": rerr("U_sum"), "uu": rerr("uu_sum"), "ww": rerr("ww_sum"),
                                                  "uw": rerr("uw_sum")}
    ch.timing(True)
    ch.step("IMEX", dt, min(a.steps, L_RING))
    phases, nst = ch.timing_read()
    ch.timing(False)
    out["kernels_ms"] = {k: v / max(nst, 1) for k, v in phases.items()}
    out["note"] = ("FP32 spectrum (x transform, fused y transform / z solve / inverse y transform per kx slab in "
                   "shared memory, inverse x transform), FP64 for the (0,0) mode and kx < 3, |ky| < 3; solves for "
                   "the increment over the previous step's pressure; the first 10 steps use the FP64 solve")
    return out


L_RING = 64
# kernels per IMEX step: rhs, cn, div+fftx, ffty, tri, iffty, ifftx, project(+bulk+forcing)
LAUNCHES_PER_STEP = 8


def kernel_table(phases, nst, s, npts):
    """Per-kernel average launch time and algorithmic bytes per launch.
    Bytes per grid point (s = storage bytes of the velocity fields and AB2
    history, 8 FP64 / 4 mixed; the Poisson spectrum, p and the LU factor
    tables are FP64; a half spectrum holds (nx/2+1)/nx complex per point):
      rhs  : read u, v, w, r_prev; write u*, v*, w*, r      = 12 s
      cn   : read u*, write u** (3 components)              =  6 s
      fftx : read u**, v**, w** (divergence); write X       =  3 s + 16 h
      ffty, iffty : read + write X                          = 32 h
      tri  : read + write X, read the two factor tables     = 32 h + 16 h
      ifftx: read X, write p                                = 16 h + 8
      proj : read u**, v**, w**, p; write u, v, w           =  6 s + 8
    with h = (nx/2+1)/nx.
    """
    hh = (NX / 2 + 1) / NX
    bpp = {"rhs": 12 * s, "cn": 6 * s, "fftx": 3 * s + 16 * hh, "ffty": 32 * hh, "tri": 48 * hh,
           "iffty": 32 * hh, "ifftx": 16 * hh + 8, "proj": 6 * s + 8, "fin": 0}
    out = []
    for k, w in bpp.items():
        ms = phases.get(k, 0.0) / max(nst, 1)
        b = w * npts
        out.append({"name": k, "ms": ms, "bytes": b, "gbs": (b / (ms / 1e3) / 1e9) if ms > 0 else 0.0})
    return out


def run_e2e(a, grid, fields, dt):
    """Same metric through the public ChannelFlow-compatible API with host
    buffers: the initial state goes host->device from pinned memory, each
    step's (u_bulk, forcing) is copied back to its own pinned host slot, and
    the final u, v, w come back at the end; all inside the timed region.  The
    per-step copies are queued behind their steps with no host sync between
    steps (the reference's run loop likewise reads these scalars only every
    n_out steps, solver.py:815-832); one sync ends the region."""
    import torch
    from torchannel_b200.core import Channel
    z_f, z_c, dz_f, dz_c = grid
    u0, v0, w0 = fields
    ch = Channel(NX, NY, NZ, LX, LY, LZ, 1.0 / RE, dz_f, dz_c, precision=a.precision)
    hu = torch.from_numpy(u0).pin_memory(); hv = torch.from_numpy(v0).pin_memory()
    hw = torch.from_numpy(w0).pin_memory()
    out = torch.empty((max(a.steps, 2), 2), dtype=torch.float64).pin_memory()  # one slot per step
    du = torch.empty_like(hu, device="cuda"); dv = torch.empty_like(hv, device="cuda")
    dw = torch.empty_like(hw, device="cuda")
    ou, ov, ow = (torch.empty_like(t).pin_memory() for t in (hu, hv, hw))  # results land in pinned memory
    # one short warm-up pass of the same path, then three timed passes (median)
    secs = []
    for rep in range(4):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        du.copy_(hu, non_blocking=True); dv.copy_(hv, non_blocking=True); dw.copy_(hw, non_blocking=True)
        ch.set_state(du, dv, dw)
        n = a.steps if rep else 2
        for s_ in range(n):
            ch.step("IMEX", dt)
            out[s_].copy_(ch.scalars[:2], non_blocking=True)   # (forcing, u_bulk) of step s_
        u, v, w, _ = ch.get_state()
        ou.copy_(u, non_blocking=True); ov.copy_(v, non_blocking=True); ow.copy_(w, non_blocking=True)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        if not bool(torch.isfinite(out[:n]).all()):
            raise RuntimeError("non-finite (forcing, u_bulk) in the end-to-end run")
        if rep:
            secs.append(t1 - t0)
    sec = sorted(secs)[len(secs) // 2]
    bi = (hu.numel() + hv.numel() + hw.numel()) * 8
    bo = (hu.numel() + hv.numel() + hw.numel()) * 8
    return {"value": NX * NY * NZ * a.steps / sec, "unit": "grid-point-steps/s",
            "h2d_bytes_per_step": bi / a.steps, "d2h_bytes_per_step": bo / a.steps + 16,
            "note": "pinned H2D of the initial u, v, w + set_state, K x (one IMEX step + D2H of its (forcing, "
                    "u_bulk) into its own pinned slot, no host sync between steps), get_state + pinned D2H of "
                    "u, v, w, one sync; median of 3 timed passes"}


# ---------------------------------------------------------------------------
# CPU baseline / reference arm: the numpy oracle step
# ---------------------------------------------------------------------------
def cpu_step_setup(seed=0):
    from oracle.step import OracleChannel
    oc = OracleChannel(NX, NY, NZ, LX, LY, LZ, RE, gamma=GAMMA)
    oc.init_fresh(seed=seed)
    return oc


def cpu_baseline(budget_s, steps=None):
    oc = cpu_step_setup()
    oc.step_imex(0.002)           # warm-up (Euler first step)
    t_all, n = 0.0, 0
    while (steps is None and (t_all < budget_s or n == 0)) or (steps is not None and n < steps):
        t0 = time.perf_counter()
        oc.step_imex(0.002)
        t_all += time.perf_counter() - t0
        n += 1
    return {"value": NX * NY * NZ * n / t_all, "unit": "grid-point-steps/s", "cores": 1, "kind": "port",
            "sample": f"{n} full IMEX steps at {NX}x{NY}x{NZ} of the numpy FP64 oracle (single thread), "
                      f"{t_all:.1f} s"}


def _ref_worker(idx, steps, barrier, queue):
    """One replica of the reference arm: an oracle channel of its own (seed =
    replica index), one warm-up step, then `steps` timed steps started
    together with the other replicas."""
    oc = cpu_step_setup(seed=idx)
    oc.step_imex(0.002)
    barrier.wait()
    t0 = time.perf_counter()
    for _ in range(steps):
        oc.step_imex(0.002)
    queue.put((idx, steps, time.perf_counter() - t0))


def _host_replicas():
    """Replicas the host can run at once: one per usable core, at most one per
    1.6 GB of available memory (an oracle channel at 192^3 holds about 1.1 GB)."""
    try:
        cores = len(os.sched_getaffinity(0))
    except AttributeError:
        cores = os.cpu_count() or 1
    avail = None
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    avail = int(line.split()[1]) * 1024
    except OSError:
        pass
    by_mem = int(avail // (1.6e9)) if avail else cores
    return max(1, min(cores, by_mem))


def run_reference(a):
    """The reference's CPU path on all usable host cores: the numpy oracle
    step (a single-threaded restatement of ChannelFlow.step_imex) run as one
    independent replica per core, started together; value = all replicas'
    grid-point-steps / the slowest replica's time.  Each replica runs
    min(--steps, 5) full 192^3 steps after one warm-up step."""
    import multiprocessing as mp
    rank, world, local = dist_env()
    if rank != 0:
        return
    os.environ["OMP_NUM_THREADS"] = "1"
    P = _host_replicas()
    steps = max(1, min(a.steps, 5))
    ctx = mp.get_context("spawn")
    barrier, queue = ctx.Barrier(P + 1), ctx.Queue()
    procs = [ctx.Process(target=_ref_worker, args=(i, steps, barrier, queue)) for i in range(P)]
    for pr in procs:
        pr.start()
    barrier.wait()
    res = [queue.get() for _ in range(P)]
    for pr in procs:
        pr.join()
    t_max = max(r[2] for r in res)
    value = NX * NY * NZ * steps * P / t_max
    cpu = {"value": value, "unit": "grid-point-steps/s", "cores": P, "kind": "port",
           "sample": f"{P} concurrent replicas x {steps} IMEX steps at {NX}x{NY}x{NZ} (numpy FP64 oracle, one thread "
                     f"each, after one warm-up step), slowest replica {t_max:.1f} s"}
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "grid-point-steps/s",
            "n_gpus": world, "steps": steps, "warmup": 1, "ms_per_step": 1e3 * t_max / steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded laminar profile + 0.1 uniform noise, projected)",
            "config": {"workload": WORKLOAD, "nx": NX, "ny": NY, "nz": NZ, "scheme": "IMEX",
                       "parallelism": f"{P} host replicas"},
            "cpu_baseline": cpu,
            "e2e": {"value": value, "unit": "grid-point-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ensemble(a):
    """16 independent channels of uneven size (nx, ny in {64, 96, 128}, nz in
    {48, 64, 96}, Re_bulk U[2000, 5600], gamma U[2.2, 2.8], per-member seeds),
    mixed precision, each on its own stream; ranks own disjoint members."""
    import torch
    import torch.distributed as dist
    from torchannel_b200.ensemble import Ensemble, aggregate, make_members, partition
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    members = make_members(16, seed=0)
    mine = [members[m] for m in partition(len(members), world, rank)]
    ens = Ensemble(mine, precision=a.precision)
    if a.batch_only:
        rows, ctas = (int(x) for x in a.batch_only.split(","))
        b = ens.batch()
        b.set_shape(rows, ctas)
        b.use_graphs(False)
        ens.step_batch(a.warmup)
        torch.cuda.synchronize()
        b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        b0.record()
        ens.step_batch(a.steps)
        b1.record()
        torch.cuda.synchronize()
        ms_b = b0.elapsed_time(b1)
        value_b, _, max_ms = aggregate(ens.points() * a.steps, ms_b)
        if world > 1:
            dist.destroy_process_group()
        if rank == 0:
            print(json.dumps({"metric": "grid-point-steps/s, 16-member uneven ensemble, ensemble launches only",
                              "value": value_b, "unit": "grid-point-steps/s", "n_gpus": world, "steps": a.steps,
                              "warmup": a.warmup, "ms_per_step": max_ms / a.steps, "higher_is_better": True,
                              "config": {"workload": "ensemble of 16 channels", "shape": [rows, ctas],
                                         "graphs": False}, "info": b.info()}), flush=True)
        return
    ens.step(a.warmup)
    ens.synchronize()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    ens.step(a.steps, concurrent=True)
    ens.synchronize()
    torch.cuda.synchronize()
    ms = (time.perf_counter() - t0) * 1e3
    value, pts, max_ms = aggregate(ens.points() * a.steps, ms)
    t0 = time.perf_counter()
    ens.step(a.steps, concurrent=False)
    torch.cuda.synchronize()
    ms_seq = (time.perf_counter() - t0) * 1e3
    value_seq, _, _ = aggregate(ens.points() * a.steps, ms_seq)
    # autotuned shapes, then the whole ensemble step pair as one graph launch
    tuning = ens.autotune()
    ens.capture()
    pairs = max(1, a.steps // 2)
    ens.step_graph(1)
    torch.cuda.synchronize()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record()
    ens.step_graph(pairs)
    g1.record()
    torch.cuda.synchronize()
    ms_graph = g0.elapsed_time(g1)
    value_graph, _, _ = aggregate(ens.points() * 2 * pairs, ms_graph)
    # one persistent launch per substep for all members, tuned shape
    ens.batch()
    btun = ens.autotune_batch()
    ens.step_batch(2)
    torch.cuda.synchronize()
    b0, b1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    b0.record()
    ens.step_batch(2 * pairs)
    b1.record()
    torch.cuda.synchronize()
    ms_batch = b0.elapsed_time(b1)
    value_batch, _, _ = aggregate(ens.points() * 2 * pairs, ms_batch)
    binfo = ens.batched.info()
    diag = ens.diagnostics()
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps({"metric": "grid-point-steps/s, 16-member uneven ensemble (IMEX)", "value": value,
                          "unit": "grid-point-steps/s", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
                          "ms_per_step": max_ms / a.steps, "higher_is_better": True, "scaling": "strong",
                          "vs_baseline": None, "dtype": "f32+f64" if a.precision == "mixed" else "f64",
                          "data": "synthetic (seeded laminar + 0.1 noise per member)",
                          "config": {"workload": "ensemble of 16 channels", "members": members,
                                     "parallelism": f"members over {world} rank(s), streams per member"},
                          "one_at_a_time": {"value": value_seq},
                          "tuned_one_graph": {"value": value_graph, "ms_per_step": ms_graph / (2 * pairs),
                                              "note": "autotuned member shapes; 2 steps of all members per graph launch"},
                          "tuning": tuning,
                          "batched": {"value": value_batch, "ms_per_step": ms_batch / (2 * pairs),
                                      "launches_per_step": ens.batched.launches_per_step(), "shape": btun,
                                      "units": binfo["units"], "ctas": binfo["ctas"],
                                      "note": "one launch per substep for all members (CN per chunk count, "
                                              "x transforms per length), two steps per graph launch "
                                              "(tc_batch_step)"},
                          "max_div_after": max(d["max_div"] for d in diag)}), flush=True)


def _poisson_residual(p, rhs, dx, dy, dz_c, dz_f):
    """L p - rhs on the interior: 3-point periodic x/y, the stretched z rows
    with Neumann closures (the operator the solve inverts)."""
    pi = p[1:-1, 1:-1, 1:-1]
    lap = (np.roll(pi, -1, 0) - 2 * pi + np.roll(pi, 1, 0)) / dx ** 2
    lap += (np.roll(pi, -1, 1) - 2 * pi + np.roll(pi, 1, 1)) / dy ** 2
    cl, cr = 1.0 / (dz_c[:-1] * dz_f), 1.0 / (dz_c[1:] * dz_f)
    up = np.concatenate([pi[:, :, 1:], pi[:, :, -1:]], axis=2)
    dn = np.concatenate([pi[:, :, :1], pi[:, :, :-1]], axis=2)
    return lap + cr * (up - pi) - cl * (pi - dn) - rhs


def run_poisson(a):
    """Poisson solve alone on a seeded uniform random right-hand side with
    zero dz_f-weighted mean (FP64 spectrum), through tc_poisson_solve on
    device buffers (reference layout in and out)."""
    import torch
    from torchannel_b200.core import Channel
    from torchannel_b200.grid import generate_grid
    rank, world, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    peak, _ = measured_peaks()
    res = []
    for (nx, ny, nz) in ((192, 192, 128), (384, 384, 256)):
        z_f, z_c, dz_f, dz_c = generate_grid(GAMMA, nz, LZ)
        rng = np.random.default_rng(1)
        rhs = rng.random((nx, ny, nz)) - 0.5
        rhs -= np.sum(rhs * dz_f) / (nx * ny * LZ)
        ch = Channel(nx, ny, nz, LX, LY, LZ, 1.0 / RE, dz_f, dz_c, precision=a.precision)
        rd = torch.as_tensor(rhs, device="cuda")
        for _ in range(a.warmup):
            p = ch.poisson_solve(rd)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.steps):
            p = ch.poisson_solve(rd)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / a.steps
        pn = p.cpu().numpy()
        r = _poisson_residual(pn, rhs, LX / nx, LY / ny, dz_c, dz_f)
        algo = 4 * 8 * nx * ny * nz  # read rhs, write/read the spectrum, write p (FP64 words)
        res.append({"grid": [nx, ny, nz], "ms_per_solve": ms, "points_per_s": nx * ny * nz / (ms / 1e3),
                    "algorithmic_gbs": algo / (ms / 1e3) / 1e9, "frac_of_peak": algo / (ms / 1e3) / 1e9 / peak,
                    "max_residual": float(np.max(np.abs(r))), "max_rhs": float(np.max(np.abs(rhs))),
                    "includes": "reference-layout conversion in and out"})
        del ch
    print(json.dumps({"metric": "Poisson solves/s (FFT + per-mode tridiagonal + inverse FFT)",
                      "value": 1e3 / res[0]["ms_per_solve"], "unit": "solves/s at 192x192x128", "n_gpus": 1,
                      "steps": a.steps, "warmup": a.warmup, "higher_is_better": True, "dtype": "f64",
                      "data": "synthetic (seeded uniform random, zero dz_f-weighted mean)",
                      "config": {"workload": "Poisson microbench"}, "results": res}), flush=True)


def run_adjoint(a):
    """Forward + adjoint of J = mean kinetic energy over steps 101..200 of 200
    FP64 IMEX steps (dt 0.003) at 96x96x64 with a seeded 8-mode Fourier body
    force (amplitude 0.01), gradients with respect to the initial field and the
    body force; checked against central finite differences along 8 seeded
    directions.  Replicas: every rank runs its own channel (seed = rank)."""
    import torch
    import torch.distributed as dist
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    r = measure_adjoint(a, rank, world)
    if world > 1:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(r["line"]), flush=True)


def measure_adjoint(a, rank, world):
    """The adjoint workload (see run_adjoint) on this rank; every rank takes
    the same collective steps.  Returns {"line": the workload's JSON line,
    "summary": the keys the step bench line carries}."""
    import torch
    import torch.distributed as dist
    from torchannel_b200.adjoint import AdjointRunner, fourier_body_force, to_internal
    from torchannel_b200 import _lib as L
    from torchannel_b200.core import Channel
    from torchannel_b200.grid import generate_grid
    from torchannel_b200.init import initialize_flow
    nx, ny, nz, dt, N = 96, 96, 64, 0.003, 200
    window = range(101, 201)
    z_f, z_c, dz_f, dz_c = generate_grid(GAMMA, nz, LZ)
    ch = Channel(nx, ny, nz, LX, LY, LZ, 1.0 / RE, dz_f, dz_c, precision="fp64")
    u, v, w, _ = initialize_flow(nx, ny, nz, z_c, LY, LZ, perturbation_intensity=0.1, seed=rank)
    ch.set_state(u, v, w)
    ub = ch.bulk_velocity()
    ch.set_state(u * (1.0 / ub), v, w)
    ch.project_initial()
    q0 = [t.clone() for t in ch.get_state()[:3]]
    F = fourier_body_force(ch, z_f, z_c, seed=100 + rank)
    Fi = to_internal(ch, *F)
    L.check(ch.lib.tc_set_body_force(ch.ctx, *[ctypes.c_void_p(t.data_ptr()) for t in Fi]))
    ev = lambda: torch.cuda.Event(enable_timing=True)  # noqa: E731
    # plain forward (graph replay, body force, no objective hooks), the cost unit
    for _ in range(max(a.warmup, 1)):
        ch.set_state(*q0)
        ch.step("IMEX", dt, N)
    torch.cuda.synchronize()
    e0, e1 = ev(), ev()
    ch.set_state(*q0)
    e0.record()
    ch.step("IMEX", dt, N)
    e1.record()
    torch.cuda.synchronize()
    fwd_ms = e0.elapsed_time(e1)
    def timed(mode):
        r = AdjointRunner(ch, dt, N, window, checkpoint_every=a.checkpoint_every, mode=mode)
        r.set_body_force(*Fi)
        r.forward(*q0)
        r.backward()  # captures the reverse segments
        torch.cuda.synchronize()
        t0, t1, t2 = ev(), ev(), ev()
        t0.record()
        J = r.forward(*q0)
        t1.record()
        gq, gF, _ = r.backward()
        t2.record()
        torch.cuda.synchronize()
        return r, float(J), gq, gF, t0.elapsed_time(t1), t1.elapsed_time(t2)

    # both reverse modes: recomputation from checkpoints and the stored tape
    rr, Jr, gqr, gFr, fc_r, bw_r = timed("recompute")
    rr.close()
    del rr
    runner, Jv, gq, gF, fc_ms, bw_ms = timed(a.adjoint_mode)
    same = Jv == Jr and all(torch.equal(x, y) for x, y in zip(gq + gF, gqr + gFr))
    # finite differences along seeded directions (initial field / body force)
    g = torch.Generator(device="cpu").manual_seed(1234)
    errs = []
    eps = 1e-6
    for trial in range(8):
        d = [torch.randn(t.shape, generator=g, dtype=torch.float64).cuda() for t in gq]
        for t in d:
            t[nz] = 0
        d[2][0] = 0
        on_force = trial % 2 == 1
        ad = sum(float((x * y).sum()) for x, y in zip(gF if on_force else gq, d))
        vals = []
        for sgn in (1.0, -1.0):
            if on_force:
                runner.set_body_force(*[f + sgn * eps * x for f, x in zip(Fi, d)])
                vals.append(float(runner.forward(*q0)))
            else:
                from torchannel_b200.adjoint import from_internal
                dq = from_internal(ch, *d)
                vals.append(float(runner.forward(*[q + sgn * eps * x for q, x in zip(q0, dq)])))
        runner.set_body_force(*Fi)
        fd = (vals[0] - vals[1]) / (2 * eps)
        errs.append(abs(fd - ad) / abs(fd))
    if world > 1:
        t = torch.tensor([fwd_ms, fc_ms + bw_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        fwd_ms, tot = float(t[0]), float(t[1])
    else:
        tot = fc_ms + bw_ms
    runner.close()
    npts = nx * ny * nz
    summary = {"workload": "96x96x64, 200 FP64 IMEX steps (dt 0.003), J = mean KE over steps 101..200, "
                           "gradients w.r.t. the initial field and an 8-mode body force",
               "adjoint_over_forward": tot / fwd_ms, "mode": runner.mode, "forward_ms": fwd_ms,
               "forward_with_hooks_ms": fc_ms, "reverse_sweep_ms": bw_ms,
               "recompute_ratio": (fc_r + bw_r) / fwd_ms, "fd_directions": len(errs),
               "fd_max_rel_error": max(errs), "fd_eps": eps, "store_vs_recompute_bitwise_equal": same}
    line = {
            "metric": "forward+adjoint / forward cost ratio (96x96x64, 200 IMEX steps)",
            "value": tot / fwd_ms, "unit": "ratio", "n_gpus": world, "steps": N, "warmup": a.warmup,
            "ms_per_step": tot / N, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded laminar + 0.1 noise, projected; seeded 8-mode Fourier body force)",
            "config": {"workload": "adjoint: J = mean KE over steps 101..200, gradients w.r.t. q0 and F",
                       "nx": nx, "ny": ny, "nz": nz, "dt": dt, "checkpoint_every": a.checkpoint_every,
                       "adjoint_mode": a.adjoint_mode,
                       "parallelism": f"replicas{world}"},
            "adjoint_mode": runner.mode, "forward_ms": fwd_ms, "forward_with_hooks_ms": fc_ms,
            "reverse_sweep_ms": bw_ms,
            "recompute": {"checkpoint_every": a.checkpoint_every, "ratio": (fc_r + bw_r) / fwd_ms,
                          "forward_with_checkpoints_ms": fc_r, "reverse_sweep_ms": bw_r},
            "store_vs_recompute_bitwise_equal": same,
            "forward_gpss": npts * N * world / (fwd_ms / 1e3),
            "J": Jv, "grad_norm_q0": float(sum((t * t).sum() for t in gq)) ** 0.5,
            "grad_norm_F": float(sum((t * t).sum() for t in gF)) ** 0.5,
            "fd_rel_errors": errs, "fd_max_rel_error": max(errs), "fd_eps": eps}
    return {"line": line, "summary": summary}


def run_config1(a):
    """Config 1 as a run: 192x192x128, seeded laminar + 0.1 noise, adaptive dt
    (CFL 0.25, every 10 steps, the 5% rule), --run-steps IMEX steps,
    statistics every 200 steps from t = 0, diagnostics every 100 steps,
    through ChannelFlowB200.run_simulation, once in plain FP64 and once in
    mixed precision.  Throughput is grid points x steps / wall time of the
    step loop (host loop, dt updates, diagnostics and statistics included;
    the final field files excluded).  The two runs' statistics are compared
    at the end."""
    import shutil
    import tempfile
    import torch
    import yaml
    from torchannel_b200.solver import ChannelFlowB200
    rank, world, local = dist_env()
    if rank != 0:
        return
    torch.cuda.set_device(local)
    out = {}
    tmp = tempfile.mkdtemp(prefix="tc_config1_")
    try:
        for prec in ("fp64", "mixed"):
            res = os.path.join(tmp, prec)
            cfg = {
                "grid": {"nx": NX, "ny": NY, "nz": NZ},
                "domain": {"Lx": float(LX), "Ly": float(LY), "Lz": float(LZ), "stretching_type": "symmetric"},
                "flow": {"Re": RE, "Re_tau": 180.0, "U_bulk": 1.0, "gamma": GAMMA},
                "boundary_conditions": {"top_wall": {"type": "dirichlet"}},
                "initialization": {"type": "parabolic", "perturbation_intensity": 0.1},
                "solver": {"type": "fft"},
                "time": {"dt": 0.002, "n_steps": a.run_steps, "CFL_target": CFL, "dt_update_interval": 10,
                         "dt_max": DT_MAX, "dt_min": DT_MIN, "scheme": "IMEX"},
                "compute": {"device": "cuda", "precision": prec},
                "output": {"results_folder": res, "n_out": 100, "n_save": a.run_steps + 1},
                "statistics": {"n_stats": 200, "t_stats": 0.0, "z_plus_target": 15.0},
            }
            os.makedirs(res, exist_ok=True)
            path = os.path.join(res, "config.yaml")
            with open(path, "w") as f:
                yaml.safe_dump(cfg, f)
            cf = ChannelFlowB200(path, seed=0, verbose=False)
            torch.cuda.synchronize()
            cf.run_simulation()
            torch.cuda.synchronize()
            st = cf.turbulence_stats.finalize_statistics()
            d = cf.ch.diagnostics()
            out[prec] = {"seconds": cf.loop_seconds, "value": NX * NY * NZ * a.run_steps / cf.loop_seconds,
                         "time": cf.time, "final_dt": cf.dt, "max_div": d["max_div"], "u_bulk": d["u_bulk"],
                         "u_tau_stats": st["u_tau"], "n_samples": int(st["n_samples"]), "stats": st}
            del cf
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    f64, mix = out["fp64"]["stats"], out["mixed"]["stats"]

    def rel(k):
        return float(np.max(np.abs(mix[k] - f64[k])) / max(np.max(np.abs(f64[k])), 1e-300))
    m, d64 = out["mixed"], out["fp64"]
    line = {"metric": f"grid-point-steps/s, config 1 run ({a.run_steps} IMEX steps, adaptive dt, statistics)",
            "value": m["value"], "unit": "grid-point-steps/s", "n_gpus": 1, "steps": a.run_steps, "warmup": 0,
            "ms_per_step": m["seconds"] / a.run_steps * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded laminar profile + 0.1 uniform noise)",
            "config": {"workload": "config 1 run through ChannelFlowB200.run_simulation", "nx": NX, "ny": NY,
                       "nz": NZ, "cfl": CFL, "dt_update_interval": 10, "n_stats": 200},
            "fp64_plain": {k: d64[k] for k in ("value", "seconds", "time", "final_dt", "max_div", "u_bulk",
                                                "u_tau_stats", "n_samples")},
            "mixed": {k: m[k] for k in ("seconds", "time", "final_dt", "max_div", "u_bulk", "u_tau_stats",
                                         "n_samples")},
            "mixed_speedup_over_fp64": m["value"] / d64["value"],
            "stats_rel_diff_mixed_vs_fp64": {k: rel(k) for k in ("U_mean", "uu_mean", "vv_mean", "ww_mean",
                                                                  "uw_mean", "E_uu_2d")},
            "u_tau_rel_diff": abs(m["u_tau_stats"] - d64["u_tau_stats"]) / d64["u_tau_stats"]}
    print(json.dumps(line), flush=True)


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    elif a.workload == "ensemble":
        run_ensemble(a)
    elif a.workload == "poisson":
        run_poisson(a)
    elif a.workload == "config1":
        run_config1(a)
    elif a.workload == "adjoint":
        run_adjoint(a)
    else:
        run_b200(a)


if __name__ == "__main__":
    main()
