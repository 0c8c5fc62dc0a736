"""Device context of one channel: owns the workspace (allocated through
torch's caching allocator) and wraps the C ABI with torch tensors.

All field arguments and results use the reference layout (``u`` (nx+1, ny+2,
nz+2), ``v`` (nx+2, ny+1, nz+2), ``w`` (nx+2, ny+2, nz+1), ``p`` (nx+2, ny+2,
nz+2)) in float64, as ``ChannelFlow`` stores them (``initflow.py:6-9``).
"""
import ctypes

import numpy as np
import torch

from . import _lib as L

SCHEMES = {"IMEX": L.TC_IMEX, "AB2": L.TC_AB2, "FE": L.TC_FE}


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class _DevArray:
    """Expose a raw device pointer to torch via __cuda_array_interface__."""

    def __init__(self, ptr, n):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f8", "data": (ptr, False),
                                         "version": 3, "strides": None}


class Channel:
    """One channel on the current CUDA device.

    precision: "fp64" (plain) or "mixed" (FP32 fields, stencils and CN
    sweeps of the deviation from the base profile; FP64 Poisson solve, CN
    tables, bulk forcing and statistics sums).
    rhs_path: "separate" (reference CPU-path semantics, default) or "fused"
    (reference CUDA-path semantics for the duplicate planes u[nx], v[:, ny]).
    """

    def __init__(self, nx, ny, nz, Lx, Ly, Lz, nu, dz_f, dz_c, U_bulk=1.0,
                 top_wall_bc_type="dirichlet", precision="fp64", rhs_path="separate"):
        if not torch.cuda.is_available():
            raise RuntimeError("torchannel_b200 needs a CUDA device (B200, sm_100a); no CPU fallback")
        self.lib = L.lib()
        self.nx, self.ny, self.nz = int(nx), int(ny), int(nz)
        self.Lx, self.Ly, self.Lz = float(Lx), float(Ly), float(Lz)
        self.nu, self.U_bulk = float(nu), float(U_bulk)
        self.top = top_wall_bc_type
        self.precision = precision
        self.rhs_path = rhs_path
        self._dzf = np.ascontiguousarray(np.asarray(dz_f, dtype=np.float64))
        self._dzc = np.ascontiguousarray(np.asarray(dz_c, dtype=np.float64))
        assert self._dzf.shape == (self.nz,) and self._dzc.shape == (self.nz + 1,)
        d = L.GridDesc()
        d.nx, d.ny, d.nz = self.nx, self.ny, self.nz
        d.Lx, d.Ly, d.Lz, d.nu, d.U_bulk = self.Lx, self.Ly, self.Lz, self.nu, self.U_bulk
        d.top_wall = L.TC_TOP_FREESLIP if top_wall_bc_type == "neumann" else L.TC_TOP_NOSLIP
        d.precision = {"fp64": L.TC_FP64, "mixed": L.TC_MIXED}[precision]
        d.rhs_path = {"separate": L.TC_RHS_SEPARATE, "fused": L.TC_RHS_FUSED}[rhs_path]
        d.dz_f = self._dzf.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        d.dz_c = self._dzc.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        self._desc = d
        nb = ctypes.c_size_t()
        L.check(self.lib.tc_workspace_bytes(ctypes.byref(d), ctypes.byref(nb)))
        self.workspace_bytes = nb.value
        self._ws = torch.empty(nb.value + 256, dtype=torch.uint8, device="cuda")
        base = self._ws.data_ptr()
        aligned = (base + 255) & ~255
        ctx = ctypes.c_void_p()
        L.check(self.lib.tc_create(ctypes.byref(d), ctypes.c_void_p(aligned), nb.value, ctypes.byref(ctx)))
        self.ctx = ctx
        sp = ctypes.c_void_p()
        L.check(self.lib.tc_scalars(self.ctx, ctypes.byref(sp)))
        self.scalars = torch.as_tensor(_DevArray(sp.value, 8), device="cuda")
        self.k_bot = self.k_top = None

    def __del__(self):
        try:
            if getattr(self, "ctx", None) is not None and self.ctx.value:
                torch.cuda.synchronize()
                self.lib.tc_destroy(self.ctx)
                self.ctx = None
        except Exception:
            pass

    # -- shapes ------------------------------------------------------------
    def shapes(self):
        nx, ny, nz = self.nx, self.ny, self.nz
        return dict(u=(nx + 1, ny + 2, nz + 2), v=(nx + 2, ny + 1, nz + 2),
                    w=(nx + 2, ny + 2, nz + 1), p=(nx + 2, ny + 2, nz + 2), cell=(nx, ny, nz))

    def _dev(self, a, shape):
        t = torch.as_tensor(a)
        if tuple(t.shape) != tuple(shape):
            raise ValueError(f"expected shape {shape}, got {tuple(t.shape)}")
        return t.to(device="cuda", dtype=torch.float64).contiguous()

    def _empty(self, key):
        return torch.empty(self.shapes()[key], dtype=torch.float64, device="cuda")

    # -- state -------------------------------------------------------------
    def set_state(self, u, v, w, forcing=0.0):
        s = self.shapes()
        u, v, w = self._dev(u, s["u"]), self._dev(v, s["v"]), self._dev(w, s["w"])
        L.check(self.lib.tc_set_state(self.ctx, _ptr(u), _ptr(v), _ptr(w), float(forcing), _stream()))
        torch.cuda.current_stream().synchronize()

    def get_state(self):
        u, v, w, p = (self._empty(k) for k in "uvwp")
        L.check(self.lib.tc_get_state(self.ctx, _ptr(u), _ptr(v), _ptr(w), _ptr(p), _stream()))
        return u, v, w, p

    def get_field(self, name):
        out = self._empty(name)
        args = [None, None, None, None]
        args["uvwp".index(name)] = _ptr(out)
        L.check(self.lib.tc_get_state(self.ctx, *args, _stream()))
        return out

    def get_history(self):
        ru, rv, rw = (self._empty(k) for k in "uvw")
        L.check(self.lib.tc_get_history(self.ctx, _ptr(ru), _ptr(rv), _ptr(rw), _stream()))
        return ru, rv, rw

    def set_history(self, ru, rv, rw):
        s = self.shapes()
        ru, rv, rw = self._dev(ru, s["u"]), self._dev(rv, s["v"]), self._dev(rw, s["w"])
        L.check(self.lib.tc_set_history(self.ctx, _ptr(ru), _ptr(rv), _ptr(rw), _stream()))
        torch.cuda.current_stream().synchronize()

    def set_forcing(self, f):
        L.check(self.lib.tc_set_forcing(self.ctx, float(f), _stream()))

    # -- stepping ----------------------------------------------------------
    def step(self, scheme, dt, n_steps=1):
        L.check(self.lib.tc_step(self.ctx, SCHEMES[scheme] if isinstance(scheme, str) else int(scheme),
                                 float(dt), int(n_steps), _stream()))

    def use_graphs(self, on=True):
        L.check(self.lib.tc_use_graphs(self.ctx, int(bool(on))))

    def set_cn_chunk(self, rows):
        """Rows per chunk of the CN solve (16, 32, or 0 for the default)."""
        L.check(self.lib.tc_set_cn_chunk(self.ctx, int(rows)))

    def use_fused_poisson(self, on=True):
        """Form of the Poisson middle (y transforms and z solve): False / 0 three
        kernels, True / 1 one cluster kernel, 2 two streaming passes (the
        y transform fused with the forward elimination, the back substitution
        with the inverse y transform; the default where the grid allows it).
        Raises when the grid does not allow the form asked for."""
        L.check(self.lib.tc_use_fused_poisson(self.ctx, int(on)))

    def use_bulk_ffty(self, on=True):
        """y transforms of the Poisson solve staged by bulk copies (on) or by
        per-lane loads (off, the default); same results."""
        L.check(self.lib.tc_use_bulk_ffty(self.ctx, int(bool(on))))

    def use_tma_rhs(self, on=True):
        """Explicit-RHS tiles staged by tensor copies (True or a tile-shape
        mode 1..6; mode 1 is the default where the grid allows it) or by
        per-thread loads (False); bit-identical.  An ensemble's RHS stages
        its tiles by tensor copies while all its members have mode 1 on."""
        L.check(self.lib.tc_use_tma_rhs(self.ctx, int(on)))

    def use_fp32_poisson(self, on=True, warm_steps=10):
        """Single-precision Poisson step (mixed precision): FP32 spectrum,
        FP64 for the (0,0) and lowest modes, solving for the increment of p
        over the previous step's pressure; the first `warm_steps` steps after
        set_state use the FP64 solve.  Raises for FP64 contexts and for grids
        whose kx slab does not fit one CTA's shared memory."""
        L.check(self.lib.tc_use_fp32_poisson(self.ctx, int(bool(on)), int(warm_steps)))

    def project_initial(self):
        L.check(self.lib.tc_project_initial(self.ctx, _stream()))

    @property
    def forcing_device(self):
        return self.scalars[0]

    @property
    def u_bulk_device(self):
        return self.scalars[1]

    # -- reductions (host values; these synchronise) -------------------------
    def bulk_velocity(self):
        out = ctypes.c_double()
        L.check(self.lib.tc_bulk_velocity(self.ctx, ctypes.byref(out), _stream()))
        return out.value

    def cfl_inverse(self):
        out = ctypes.c_double()
        L.check(self.lib.tc_cfl(self.ctx, ctypes.byref(out), _stream()))
        return out.value

    def diagnostics(self):
        out = (ctypes.c_double * 5)()
        L.check(self.lib.tc_diagnostics(self.ctx, out, _stream()))
        return dict(max_div=out[0], u_tau=out[1], u_bulk=out[2], forcing=out[3], nonfinite=bool(out[4]))

    # -- operator hooks ----------------------------------------------------
    def divergence(self):
        out = self._empty("cell")
        L.check(self.lib.tc_divergence(self.ctx, _ptr(out), _stream()))
        return out

    def explicit_rhs(self, full=False):
        ru, rv, rw = (self._empty(k) for k in "uvw")
        L.check(self.lib.tc_explicit_rhs(self.ctx, int(bool(full)), _ptr(ru), _ptr(rv), _ptr(rw), _stream()))
        return ru, rv, rw

    def implicit_diffusion(self, dt):
        L.check(self.lib.tc_implicit_diffusion(self.ctx, float(dt), _stream()))

    def poisson_solve(self, rhs):
        rhs = self._dev(rhs, self.shapes()["cell"])
        p = self._empty("p")
        L.check(self.lib.tc_poisson_solve(self.ctx, _ptr(rhs), _ptr(p), _stream()))
        return p

    def project(self, p, dt):
        p = self._dev(p, self.shapes()["p"])
        L.check(self.lib.tc_project(self.ctx, _ptr(p), float(dt), _stream()))
        torch.cuda.current_stream().synchronize()

    # -- statistics ----------------------------------------------------------
    def stats_init(self, z_c, Re_tau_target, z_plus_target=15.0):
        zc = np.ascontiguousarray(np.asarray(z_c, dtype=np.float64))
        kb, kt = ctypes.c_int(), ctypes.c_int()
        L.check(self.lib.tc_stats_init(self.ctx, zc.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                       float(Re_tau_target), float(z_plus_target),
                                       ctypes.byref(kb), ctypes.byref(kt)))
        self.k_bot, self.k_top = kb.value, kt.value
        return self.k_bot, self.k_top

    def stats_accumulate(self):
        L.check(self.lib.tc_stats_accumulate(self.ctx, _stream()))

    def stats_read(self):
        nz, hx, hy = self.nz, self.nx // 2, self.ny // 2
        prof = np.zeros(5 * nz)
        spec = np.zeros(4 * hx * hy)
        n = ctypes.c_int()
        L.check(self.lib.tc_stats_read(self.ctx, prof.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                       spec.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(n)))
        prof = prof.reshape(5, nz)
        spec = spec.reshape(4, hx, hy)
        return dict(U_sum=prof[0], uu_sum=prof[1], vv_sum=prof[2], ww_sum=prof[3], uw_sum=prof[4],
                    E_uu_2d_sum=spec[0], E_vv_2d_sum=spec[1], E_ww_2d_sum=spec[2], E_uw_2d_sum=spec[3],
                    n_samples=n.value)

    def stats_write(self, sums, n_samples):
        prof = np.ascontiguousarray(np.stack([sums[k] for k in ("U_sum", "uu_sum", "vv_sum", "ww_sum", "uw_sum")]),
                                    dtype=np.float64)
        spec = np.ascontiguousarray(np.stack([sums[k] for k in ("E_uu_2d_sum", "E_vv_2d_sum", "E_ww_2d_sum",
                                                                "E_uw_2d_sum")]), dtype=np.float64)
        L.check(self.lib.tc_stats_write(self.ctx, prof.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                        spec.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), int(n_samples)))

    def timing(self, on=True):
        L.check(self.lib.tc_timing_enable(self.ctx, int(bool(on))))

    def timing_read(self):
        """Summed ms per phase over the recorded steps, and the step count."""
        ms = (ctypes.c_double * len(L.PHASES))()
        n = ctypes.c_int()
        L.check(self.lib.tc_timing_read(self.ctx, ms, ctypes.byref(n)))
        return dict(zip(L.PHASES, list(ms))), n.value

    def error_word(self):
        c = ctypes.c_int()
        L.check(self.lib.tc_error(self.ctx, ctypes.byref(c)))
        return c.value
