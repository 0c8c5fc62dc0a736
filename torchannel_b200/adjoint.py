"""Gradients of a time-averaged kinetic-energy objective of the IMEX channel
with respect to the initial velocity field and a body-force field, from the
hand-written CUDA adjoint of every substep (``tc_adjoint_*`` in
``include/torchannel_b200.h``), with checkpointed recomputation of the step
states.  FP64 contexts only.  The reference has no adjoint; the forward map
differentiated is its IMEX step (``solver.py:580-710``) with an added body
force F in the explicit right-hand side.

Objective: J = sum over steps n in ``window`` of weight * KE(q^n), weight =
1/len(window), KE(q) = (1/(2V)) sum W q^2 over the degrees of freedom (W = the
cell volume dx dy dz_f for u and v, the face volume dx dy dz_c for w).

Layouts: public arguments are reference-layout tensors (``u`` (nx+1, ny+2,
nz+2), ``v`` (nx+2, ny+1, nz+2), ``w`` (nx+2, ny+2, nz+1), float64, on the
device); gradients come back in the same layout on the degrees of freedom
(ghost entries 0: the step overwrites ghosts before using them).  The C ABI
works on the internal layout ([k][j][i]; u, v nz planes, w nz+1 face planes),
converted here by index copies.
"""
import ctypes

import torch

from . import _lib as L
from .core import _ptr, _stream


def to_internal(ch, u, v, w):
    """Degrees of freedom of reference-layout u, v, w as three internal fields
    of (nz+1, ny, nx) (u and v with a zero top plane, w with zero walls)."""
    nx, ny, nz = ch.nx, ch.ny, ch.nz
    out = []
    for a in (u, v):
        t = torch.zeros(nz + 1, ny, nx, dtype=torch.float64, device="cuda")
        t[:nz] = a[1:nx + 1, 1:ny + 1, 1:nz + 1].permute(2, 1, 0)
        out.append(t)
    t = torch.zeros(nz + 1, ny, nx, dtype=torch.float64, device="cuda")
    t[1:nz] = w[1:nx + 1, 1:ny + 1, 1:nz].permute(2, 1, 0)
    out.append(t)
    return out


def from_internal(ch, fu, fv, fw):
    """Internal fields back to reference-layout tensors (ghosts 0)."""
    nx, ny, nz = ch.nx, ch.ny, ch.nz
    u = torch.zeros(nx + 1, ny + 2, nz + 2, dtype=torch.float64, device="cuda")
    v = torch.zeros(nx + 2, ny + 1, nz + 2, dtype=torch.float64, device="cuda")
    w = torch.zeros(nx + 2, ny + 2, nz + 1, dtype=torch.float64, device="cuda")
    u[1:nx + 1, 1:ny + 1, 1:nz + 1] = fu[:nz].permute(2, 1, 0)
    v[1:nx + 1, 1:ny + 1, 1:nz + 1] = fv[:nz].permute(2, 1, 0)
    w[1:nx + 1, 1:ny + 1, 1:nz] = fw[1:nz].permute(2, 1, 0)
    return u, v, w


class AdjointRunner:
    """Forward run of ``n_steps`` IMEX steps of ``dt`` from a fresh state
    (Euler first step, as after ``tc_set_state``), accumulating the objective,
    and the reverse sweep.

    mode "recompute": checkpoints (the full step record: state, AB2 history,
    forcing) are kept every ``checkpoint_every`` steps; the reverse sweep
    recomputes each segment from its checkpoint onto a tape of
    checkpoint_every + 1 states and then runs the segment's adjoint steps
    backwards.  Memory: N / C records + C + 1 states.
    mode "store": the forward run itself writes every state to a tape of
    N + 1 states and the reverse sweep recomputes nothing.
    mode "auto": "store" when that tape takes at most a quarter of the free
    device memory, else "recompute"."""

    def __init__(self, ch, dt, n_steps, window, checkpoint_every=10, mode="recompute"):
        if ch.precision != "fp64":
            raise ValueError("the adjoint needs an FP64 channel")
        self.ch, self.lib = ch, ch.lib
        self.dt, self.N = float(dt), int(n_steps)
        self.window = sorted(set(int(n) for n in window))
        if not self.window or self.window[0] < 0 or self.window[-1] > self.N:
            raise ValueError("window must be a non-empty subset of 0..n_steps")
        self.weight = 1.0 / len(self.window)
        self.C = max(1, int(checkpoint_every))
        self.field = (ch.nz + 1) * ch.ny * ch.nx
        if mode == "auto":
            free, _ = torch.cuda.mem_get_info()
            mode = "store" if (self.N + 1) * 3 * self.field * 8 <= free // 4 else "recompute"
        if mode not in ("store", "recompute"):
            raise ValueError("mode must be 'store', 'recompute' or 'auto'")
        self.mode = mode
        nb = ctypes.c_size_t()
        L.check(self.lib.tc_adjoint_scratch_bytes(ch.ctx, ctypes.byref(nb)))
        self.scratch = torch.empty(nb.value // 8 + 2, dtype=torch.float64, device="cuda")
        nr = ctypes.c_size_t()
        L.check(self.lib.tc_internal_doubles(ch.ctx, ctypes.byref(nr)))
        self.nrec = nr.value
        self.ckpt = {}
        self.body = None
        # step hooks: the objective accumulates inside tc_step (weight on the
        # device, 0 outside the window) and the recomputation writes the
        # states of a segment to a tape -- both keep the step graphs valid
        self.J = torch.zeros(1, dtype=torch.float64, device="cuda")
        self.wdev = torch.zeros(1, dtype=torch.float64, device="cuda")
        # tape slot 0: the segment's first state (from its checkpoint), slots
        # 1..C: the states the recomputation produces
        self.slots = self.N + 1 if self.mode == "store" else self.C + 1
        self.tape = torch.zeros(self.slots * 3 * self.field, dtype=torch.float64, device="cuda")
        self.ctr = torch.full((1,), self.slots, dtype=torch.int32, device="cuda")
        L.check(self.lib.tc_set_ke_accumulator(ch.ctx, _ptr(self.J), _ptr(self.wdev), _ptr(self.scratch)))
        L.check(self.lib.tc_set_state_tape(ch.ctx, _ptr(self.tape), self.slots, _ptr(self.ctr)))
        # reverse sweep buffers and the captured adjoint segments
        z = lambda: torch.zeros(self.field, dtype=torch.float64, device="cuda")  # noqa: E731
        self.lam, self.lr, self.lF = [z(), z(), z()], [z(), z(), z()], [z(), z(), z()]
        self.mu = torch.zeros(1, dtype=torch.float64, device="cuda")
        self.graphs = {}
        self.use_graphs = True
        self._closed = False
        ch._adjoint_hooks = id(self)

    def close(self):
        """Remove the step hooks (they point at this runner's buffers) and the
        body force from the channel."""
        if getattr(self, "_closed", True) or getattr(self.ch, "ctx", None) is None:
            return
        self._closed = True
        if getattr(self.ch, "_adjoint_hooks", None) != id(self):
            return  # a newer runner owns the channel's hooks now
        L.check(self.lib.tc_set_ke_accumulator(self.ch.ctx, None, None, None))
        L.check(self.lib.tc_set_state_tape(self.ch.ctx, None, 0, None))
        if self.body is not None:
            self.set_body_force(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- records ---------------------------------------------------------
    def _save(self):
        rec = torch.empty(self.nrec, dtype=torch.float64, device="cuda")
        hh = ctypes.c_int()
        L.check(self.lib.tc_save_internal(self.ch.ctx, _ptr(rec), ctypes.byref(hh), _stream()))
        return rec, hh.value

    def _load(self, rec, hh):
        L.check(self.lib.tc_load_internal(self.ch.ctx, _ptr(rec), int(hh), _stream()))

    def _q(self, rec):
        f = self.field
        return rec[0:f], rec[f:2 * f], rec[2 * f:3 * f]

    def _tq(self, slot):
        f = self.field
        b = slot * 3 * f
        return self.tape[b:b + f], self.tape[b + f:b + 2 * f], self.tape[b + 2 * f:b + 3 * f]

    def set_body_force(self, fu=None, fv=None, fw=None):
        """Body force in the internal layout (kept alive here), or None."""
        if fu is None:
            self.body = None
            L.check(self.lib.tc_set_body_force(self.ch.ctx, None, None, None))
        else:
            self.body = [t.contiguous() for t in (fu, fv, fw)]
            L.check(self.lib.tc_set_body_force(self.ch.ctx, *[_ptr(t) for t in self.body]))

    def _chunks(self, a, b):
        """Sub-ranges of steps [a, b) over which the objective weight is
        constant (step n contributes KE(q^(n+1)) when n+1 is in the window)."""
        out, s = [], a
        for n in range(a + 1, b + 1):
            if n == b or ((n + 1) in self.window) != ((s + 1) in self.window):
                out.append((s, n, (s + 1) in self.window))
                s = n
        return out

    # -- forward -----------------------------------------------------------
    def forward(self, u0, v0, w0, forcing0=0.0):
        """Set the initial state (reference layout), run N steps; returns J as
        a device tensor."""
        ch = self.ch
        ch.set_state(u0, v0, w0, forcing=forcing0)
        self.J.zero_()
        self.ckpt = {}
        if self.mode == "store":
            rec0, hh0 = self._save()
            self.ckpt[0] = (rec0, hh0)
            for a, b in zip(self._tq(0), self._q(rec0)):
                a.copy_(b)
            self.ctr.fill_(1)  # the tape takes q^1 .. q^N
        else:
            self.ctr.fill_(self.slots)  # tape off
        if 0 in self.window:
            self._ke(self.J)
        for s in range(0, self.N, self.C):
            if self.mode == "recompute":
                self.ckpt[s] = self._save()
            for a, b, on in self._chunks(s, min(s + self.C, self.N)):
                self.wdev.fill_(self.weight if on else 0.0)
                ch.step("IMEX", self.dt, b - a)
        self.wdev.fill_(0.0)
        return self.J.clone()

    def _ke(self, J):
        L.check(self.lib.tc_kinetic_energy(self.ch.ctx, self.weight, _ptr(J), _ptr(self.scratch), _stream()))

    # -- reverse -----------------------------------------------------------
    def _segment(self, s, e, first, base):
        """Adjoint steps n = e-1 .. s of one segment (q^n in tape slot n - base)."""
        ch, lib = self.ch, self.lib
        Fp = [_ptr(t) for t in self.lF] if self.body is not None else [None, None, None]
        for n in range(e - 1, s - 1, -1):
            if n + 1 in self.window:
                L.check(lib.tc_adjoint_ke_seed(ch.ctx, self.weight, *[_ptr(t) for t in self._tq(n + 1 - base)],
                                               *[_ptr(t) for t in self.lam], _stream()))
            L.check(lib.tc_adjoint_step(ch.ctx, self.dt, int(first and n == s), *[_ptr(t) for t in self._tq(n - base)],
                                        *[_ptr(t) for t in self.lam], *[_ptr(t) for t in self.lr], *Fp,
                                        _ptr(self.mu), _ptr(self.scratch), _stream()))

    def backward(self, seed=1.0):
        """Reverse sweep; returns (dJ/dq0, dJ/dF, dJ/dforcing0) with dJ/dq0 and
        dJ/dF as internal fields (scaled by `seed`).  Each segment's adjoint
        steps are captured once per (length, window pattern, first-step flag)
        as a CUDA graph and replayed."""
        ch, lib, f = self.ch, self.lib, self.field
        for t in self.lam + self.lr + self.lF:
            t.zero_()
        self.mu.zero_()
        self.wdev.fill_(0.0)
        for s in reversed(range(0, self.N, self.C)):
            e = min(s + self.C, self.N)
            if self.mode == "recompute":
                rec0, hh0 = self.ckpt[s]
                self._load(rec0, hh0)
                for a, b in zip(self._tq(0), self._q(rec0)):
                    a.copy_(b)
                self.ctr.fill_(1)
                ch.step("IMEX", self.dt, e - s)  # tape slot m = q^(s+m)
                base = s
                first = hh0 == 0
                key = (e - s, tuple((n + 1) in self.window for n in range(s, e)), first, self.body is not None)
            else:
                base = 0
                first = s == 0 and self.ckpt[0][1] == 0
                key = ("store", s, e, self.body is not None)
            g = self.graphs.get(key)
            if g is not None:
                g.replay()
            else:
                self._segment(s, e, first, base)
                if self.use_graphs:  # capture for the next segment of this shape
                    g = torch.cuda.CUDAGraph()
                    with torch.cuda.graph(g):
                        self._segment(s, e, first, base)
                    self.graphs[key] = g
        self.ctr.fill_(self.slots)
        if 0 in self.window:
            q0 = self._q(self.ckpt[0][0])
            L.check(lib.tc_adjoint_ke_seed(ch.ctx, self.weight, *[_ptr(t) for t in q0],
                                           *[_ptr(t) for t in self.lam], _stream()))
        shp = (ch.nz + 1, ch.ny, ch.nx)
        gq = [t.view(shp) * seed for t in self.lam]
        gF = [t.view(shp) * seed for t in self.lF] if self.body is not None else None
        return gq, gF, self.mu * seed


class KineticEnergyObjective(torch.autograd.Function):
    """J(u0, v0, w0, Fu, Fv, Fw): the runner's objective as an autograd
    function of the reference-layout initial field and body force (all
    float64 CUDA tensors).  Its backward is the CUDA adjoint."""

    @staticmethod
    def forward(ctx, u0, v0, w0, Fu, Fv, Fw, runner):
        Fi = to_internal(runner.ch, Fu, Fv, Fw)
        runner.set_body_force(*Fi)
        J = runner.forward(u0, v0, w0)
        ctx.runner = runner
        return J[0].clone()

    @staticmethod
    def backward(ctx, gJ):
        r = ctx.runner
        gq, gF, _ = r.backward(seed=float(gJ))
        gu, gv, gw = from_internal(r.ch, *gq)
        fu, fv, fw = from_internal(r.ch, *gF)
        return gu, gv, gw, fu, fv, fw, None


def kinetic_energy_objective(ch, u0, v0, w0, Fu, Fv, Fw, dt, n_steps, window, checkpoint_every=10,
                             mode="recompute"):
    """Convenience: J as a differentiable tensor (see KineticEnergyObjective)."""
    runner = AdjointRunner(ch, dt, n_steps, window, checkpoint_every, mode=mode)
    return KineticEnergyObjective.apply(u0, v0, w0, Fu, Fv, Fw, runner)


def fourier_body_force(ch, z_f, z_c, n_modes=8, amplitude=0.01, seed=0):
    """A seeded body force of ``n_modes`` Fourier modes per component:
    F_c = amplitude * sum_m cos(2 pi (a_m x / Lx + b_m y / Ly) + phi_m)
    sin(pi c_m z / Lz), a_m, b_m in 0..3, c_m in 1..3, phi_m in [0, 2 pi),
    evaluated at each component's staggered positions (so it vanishes on the
    walls).  Returns reference-layout tensors (ghosts 0)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    nx, ny, nz = ch.nx, ch.ny, ch.nz
    dx, dy = ch.Lx / nx, ch.Ly / ny
    z_f = np.asarray(z_f, dtype=np.float64)
    z_c = np.asarray(z_c, dtype=np.float64)
    xs_face, xs_cell = (np.arange(nx) + 1.0) * dx, (np.arange(nx) + 0.5) * dx
    ys_face, ys_cell = (np.arange(ny) + 1.0) * dy, (np.arange(ny) + 0.5) * dy
    pos = {"u": (xs_face, ys_cell, z_c[1:nz + 1]), "v": (xs_cell, ys_face, z_c[1:nz + 1]),
           "w": (xs_cell, ys_cell, z_f[1:nz])}
    out = {}
    for comp in "uvw":
        x, y, z = pos[comp]
        f = np.zeros((len(x), len(y), len(z)))
        for _ in range(n_modes):
            a, b, c = rng.integers(0, 4), rng.integers(0, 4), rng.integers(1, 4)
            phi = rng.uniform(0.0, 2 * np.pi)
            f += (amplitude * np.cos(2 * np.pi * (a * x[:, None, None] / ch.Lx + b * y[None, :, None] / ch.Ly) + phi)
                  * np.sin(np.pi * c * z[None, None, :] / ch.Lz))
        out[comp] = f
    u = torch.zeros(nx + 1, ny + 2, nz + 2, dtype=torch.float64)
    v = torch.zeros(nx + 2, ny + 1, nz + 2, dtype=torch.float64)
    w = torch.zeros(nx + 2, ny + 2, nz + 1, dtype=torch.float64)
    u[1:nx + 1, 1:ny + 1, 1:nz + 1] = torch.from_numpy(out["u"])
    v[1:nx + 1, 1:ny + 1, 1:nz + 1] = torch.from_numpy(out["v"])
    w[1:nx + 1, 1:ny + 1, 1:nz] = torch.from_numpy(out["w"])
    return u.cuda(), v.cuda(), w.cuda()
