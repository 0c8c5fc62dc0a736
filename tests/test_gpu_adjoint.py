"""The CUDA adjoint of the IMEX step (through the C ABI): each substep against
torch autograd through the reference's own operators (golden vectors of
tests/golden/make_adjoint_golden.py), the projection by its dot-product
identity, a whole step against exact directional derivatives of the CUDA
forward step (the step map is quadratic in the state, so central differences
are exact up to rounding), and multi-step objective gradients against central
finite differences."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL = 1e-12


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _chan(nx, ny, nz, top="dirichlet", rhs_path="separate", seed_grid=2.6):
    from oracle.grid import generate_grid
    from torchannel_b200.core import Channel
    _, _, dz_f, dz_c = generate_grid(seed_grid, nz, 2.0)
    return Channel(nx, ny, nz, 4 * np.pi, 4 * np.pi / 3, 2.0, 1 / 2870.0, dz_f, dz_c, top_wall_bc_type=top,
                   rhs_path=rhs_path)


def _int(torch, a, kind, nz):
    """(nx, ny, nz[-1]) DOF array in x, y, z order -> internal (nz+1, ny, nx)."""
    nx, ny = a.shape[0], a.shape[1]
    t = torch.zeros(nz + 1, ny, nx, dtype=torch.float64, device="cuda")
    src = torch.as_tensor(np.ascontiguousarray(np.transpose(a, (2, 1, 0))), device="cuda")
    if kind == "w":
        t[1:nz] = src
    else:
        t[:nz] = src
    return t


def _dof(t, kind, nz):
    a = t.detach().cpu().numpy()
    a = a[1:nz] if kind == "w" else a[:nz]
    return np.transpose(a, (2, 1, 0))


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def _P(ch):
    from torchannel_b200.core import _ptr, _stream
    return _ptr, _stream


def _scratch(torch, ch):
    n = ctypes.c_size_t()
    assert ch.lib.tc_adjoint_scratch_bytes(ch.ctx, ctypes.byref(n)) == 0
    return torch.zeros(n.value // 8 + 2, dtype=torch.float64, device="cuda")


def test_adjoint_rhs_vs_reference_autograd(torch_cuda, golden):
    torch = torch_cuda
    G = golden("adjoint_16x12x10.npz")
    nz = int(G["nz"])
    ch = _chan(int(G["nx"]), int(G["ny"]), nz)
    _ptr, _stream = _P(ch)
    q = [_int(torch, G[c], c, nz) for c in "uvw"]
    lR = [_int(torch, G["rhs_l" + c], c, nz) for c in "uvw"]
    out = [torch.zeros_like(t) for t in q]
    assert ch.lib.tc_adjoint_rhs(ch.ctx, *[_ptr(t) for t in q], *[_ptr(t) for t in lR],
                                 *[_ptr(t) for t in out], _stream()) == 0
    for t, c in zip(out, "uvw"):
        assert rel(_dof(t, c, nz), G["rhs_g" + c]) < TOL, c


@pytest.mark.parametrize("top", ["dirichlet", "neumann"])
def test_adjoint_cn_vs_reference_autograd(torch_cuda, golden, top):
    torch = torch_cuda
    G = golden("adjoint_16x12x10.npz")
    nz = int(G["nz"])
    ch = _chan(int(G["nx"]), int(G["ny"]), nz, top=top)
    _ptr, _stream = _P(ch)
    t = "cn_" + top + "_"
    lam = [_int(torch, G[t + "l" + c], c, nz) for c in "uvw"]
    sc = _scratch(torch, ch)
    assert ch.lib.tc_adjoint_cn(ch.ctx, float(G["cn_dt"]), *[_ptr(x) for x in lam], _ptr(sc), _stream()) == 0
    for x, c in zip(lam, "uvw"):
        assert rel(_dof(x, c, nz), G[t + "g" + c]) < TOL, c
        if c == "w":
            a = x.cpu().numpy()
            assert np.all(a[0] == 0) and np.all(a[nz] == 0)


def _ref_fields(torch, ch, fu, fv, fw):
    """Internal fields -> reference layout (ghosts filled by tc_set_state's caller convention: zeros)."""
    from torchannel_b200.adjoint import from_internal
    return from_internal(ch, fu, fv, fw)


@pytest.mark.parametrize("nx,ny,nz", [(16, 12, 10), (64, 64, 40)])
def test_adjoint_projection_dot_product(torch_cuda, nx, ny, nz):
    """<b, P a> = <P^T b, a> with P the CUDA forward projection (set_state +
    project_initial) and P^T the adjoint one."""
    torch = torch_cuda
    from torchannel_b200.adjoint import to_internal
    ch = _chan(nx, ny, nz)
    _ptr, _stream = _P(ch)
    g = torch.Generator(device="cpu").manual_seed(1)
    mk = lambda: [x.to("cuda") for x in (torch.randn(nz + 1, ny, nx, generator=g, dtype=torch.float64),  # noqa: E731
                                         torch.randn(nz + 1, ny, nx, generator=g, dtype=torch.float64),
                                         torch.randn(nz + 1, ny, nx, generator=g, dtype=torch.float64))]
    a, b = mk(), mk()
    for x in (a, b):
        x[0][nz] = 0; x[1][nz] = 0; x[2][0] = 0; x[2][nz] = 0
    ch.set_state(*_ref_fields(torch, ch, *a))
    ch.project_initial()
    Pa = to_internal(ch, *ch.get_state()[:3])
    sc = _scratch(torch, ch)
    PTb = [x.clone() for x in b]
    assert ch.lib.tc_adjoint_project(ch.ctx, *[_ptr(x) for x in PTb], _ptr(sc), _stream()) == 0
    lhs = sum(float((x * y).sum()) for x, y in zip(b, Pa))
    rhs = sum(float((x * y).sum()) for x, y in zip(PTb, a))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)
    # P^T is a projection too: applying it twice changes nothing
    PTb2 = [x.clone() for x in PTb]
    assert ch.lib.tc_adjoint_project(ch.ctx, *[_ptr(x) for x in PTb2], _ptr(sc), _stream()) == 0
    for x, y in zip(PTb2, PTb):
        assert float((x - y).abs().max()) <= 1e-11 * float(y.abs().max())


class _StepMap:
    """The forward IMEX step as a map of the flat record (q, r_prev, f)."""

    def __init__(self, torch, ch, dt, have_hist):
        self.t, self.ch, self.dt, self.hh = torch, ch, dt, have_hist
        n = ctypes.c_size_t()
        assert ch.lib.tc_internal_doubles(ch.ctx, ctypes.byref(n)) == 0
        self.n = n.value
        self.f = (ch.nz + 1) * ch.ny * ch.nx

    def __call__(self, rec):
        from torchannel_b200.core import _ptr, _stream
        ch = self.ch
        assert ch.lib.tc_load_internal(ch.ctx, _ptr(rec), self.hh, _stream()) == 0
        ch.step("IMEX", self.dt)
        out = self.t.empty(self.n, dtype=self.t.float64, device="cuda")
        hh = ctypes.c_int()
        assert ch.lib.tc_save_internal(ch.ctx, _ptr(out), ctypes.byref(hh), _stream()) == 0
        return out


def _dof_mask(torch, ch):
    """1 on the degrees of freedom of a record (u, v planes < nz; w faces 1..nz-1; forcing)."""
    nx, ny, nz = ch.nx, ch.ny, ch.nz
    m = torch.zeros(nz + 1, ny, nx, dtype=torch.float64, device="cuda")
    mu, mw = m.clone(), m.clone()
    mu[:nz] = 1
    mw[1:nz] = 1
    one = torch.ones(1, dtype=torch.float64, device="cuda")
    return torch.cat([mu.flatten(), mu.flatten(), mw.flatten(), mu.flatten(), mu.flatten(), mw.flatten(), one])


@pytest.mark.parametrize("nx,ny,nz,top,path", [(16, 12, 10, "dirichlet", "separate"),
                                               (24, 36, 20, "neumann", "fused"),
                                               (64, 64, 40, "dirichlet", "separate")])
@pytest.mark.parametrize("have_hist", [0, 1])
@pytest.mark.parametrize("body", [False, True])
def test_adjoint_step_vs_exact_directional_derivative(torch_cuda, nx, ny, nz, top, path, have_hist, body):
    """<lambda_out, J d> = <J^T lambda_out, d> for the whole step (state,
    history, forcing and body force), J d from central differences of the
    CUDA forward step (exact for this quadratic map up to rounding)."""
    torch = torch_cuda
    from torchannel_b200.core import _ptr, _stream
    ch = _chan(nx, ny, nz, top=top, rhs_path=path)
    dt = 0.002
    F = _StepMap(torch, ch, dt, have_hist)
    f = F.f
    mask = _dof_mask(torch, ch)
    g = torch.Generator(device="cpu").manual_seed(11)
    rnd = lambda: torch.randn(F.n, generator=g, dtype=torch.float64).to("cuda") * mask  # noqa: E731
    # base record: laminar-like u plus noise, small history and forcing
    x0 = 0.1 * rnd()
    x0[:f].view(nz + 1, ny, nx)[:nz] += 1.0
    x0[-1] = 0.3
    Fb = [0.01 * rnd()[k * f:(k + 1) * f].view(nz + 1, ny, nx).contiguous() for k in (0, 1, 2)]
    dF = [rnd()[k * f:(k + 1) * f].view(nz + 1, ny, nx).contiguous() for k in (0, 1, 2)]
    lam_out = rnd()
    d = rnd()
    if not have_hist:
        d[3 * f:6 * f] = 0  # the history is not read on an Euler start
    eps = 1e-3

    def run(xrec, Fl):
        if body:
            assert ch.lib.tc_set_body_force(ch.ctx, *[_ptr(t) for t in Fl]) == 0
        return F(xrec)

    Fp = [a + eps * b for a, b in zip(Fb, dF)] if body else Fb
    Fm = [a - eps * b for a, b in zip(Fb, dF)] if body else Fb
    jd = (run(x0 + eps * d, Fp) - run(x0 - eps * d, Fm)) / (2 * eps)
    lhs = float((lam_out * jd).sum())
    # adjoint: lam_out split into state / history / forcing adjoints
    q0 = [x0[k * f:(k + 1) * f].clone() for k in (0, 1, 2)]
    lam = [lam_out[k * f:(k + 1) * f].clone() for k in (0, 1, 2)]
    lr = [lam_out[(3 + k) * f:(4 + k) * f].clone() for k in (0, 1, 2)]
    mu = lam_out[-1:].clone()
    lF = [torch.zeros(f, dtype=torch.float64, device="cuda") for _ in range(3)]
    sc = _scratch(torch, ch)
    if body:
        assert ch.lib.tc_set_body_force(ch.ctx, *[_ptr(t) for t in Fb]) == 0
    assert ch.lib.tc_adjoint_step(ch.ctx, dt, int(not have_hist), *[_ptr(t) for t in q0], *[_ptr(t) for t in lam],
                                  *[_ptr(t) for t in lr], *[_ptr(t) for t in lF], _ptr(mu), _ptr(sc),
                                  _stream()) == 0
    rhs = sum(float((a * d[k * f:(k + 1) * f]).sum()) for k, a in enumerate(lam))
    rhs += sum(float((a * d[(3 + k) * f:(4 + k) * f]).sum()) for k, a in enumerate(lr))
    rhs += float(mu[0] * d[-1])
    if body:
        rhs += sum(float((a * b.flatten()).sum()) for a, b in zip(lF, dF))
    assert abs(lhs - rhs) <= 1e-9 * abs(lhs), (lhs, rhs)


def _initial(torch, ch, seed):
    from oracle.grid import generate_grid
    from torchannel_b200.init import initialize_flow
    _, z_c, _, _ = generate_grid(2.6, ch.nz, 2.0)
    u, v, w, _ = initialize_flow(ch.nx, ch.ny, ch.nz, z_c, ch.Ly, ch.Lz, perturbation_intensity=0.1, seed=seed)
    ch.set_state(u, v, w)
    ch.project_initial()
    return [t.clone() for t in ch.get_state()[:3]]


def _body(torch, ch, seed, amp=0.01):
    from torchannel_b200.adjoint import from_internal
    g = torch.Generator(device="cpu").manual_seed(seed)
    fs = [amp * torch.randn(ch.nz + 1, ch.ny, ch.nx, generator=g, dtype=torch.float64).to("cuda") for _ in range(3)]
    fs[0][ch.nz] = 0; fs[1][ch.nz] = 0; fs[2][0] = 0; fs[2][ch.nz] = 0
    return list(from_internal(ch, *fs))


def test_objective_gradient_vs_finite_differences(torch_cuda):
    """dJ/d(u0, v0, w0, F) from the autograd function against central finite
    differences of J along seeded directions (J = mean kinetic energy over the
    last 6 of 12 steps; checkpoints every 5 steps)."""
    torch = torch_cuda
    from torchannel_b200.adjoint import kinetic_energy_objective, AdjointRunner, KineticEnergyObjective
    ch = _chan(32, 24, 16)
    q0 = _initial(torch, ch, 3)
    Fb = _body(torch, ch, 4)
    dt, N, window = 0.003, 12, range(7, 13)
    xs = [t.clone().requires_grad_(True) for t in q0 + Fb]
    J = kinetic_energy_objective(ch, *xs, dt=dt, n_steps=N, window=window, checkpoint_every=5)
    grads = torch.autograd.grad(J, xs)
    runner = AdjointRunner(ch, dt, N, window, checkpoint_every=5)

    def Jof(ts):
        return float(KineticEnergyObjective.apply(*ts, runner))

    g = torch.Generator(device="cpu").manual_seed(9)
    for trial in range(4):
        d = [torch.randn(t.shape, generator=g, dtype=torch.float64).to("cuda") for t in xs]
        if trial % 2 == 0:
            d = [x if k < 3 else torch.zeros_like(x) for k, x in enumerate(d)]  # initial field only
        base = [t.detach() for t in xs]
        eps = 1e-6
        Jp = Jof([b + eps * x for b, x in zip(base, d)])
        Jm = Jof([b - eps * x for b, x in zip(base, d)])
        fd = (Jp - Jm) / (2 * eps)
        ad = sum(float((gr * x).sum()) for gr, x in zip(grads, d))
        assert abs(fd - ad) <= 1e-5 * abs(fd), (trial, fd, ad)


def test_checkpoint_interval_does_not_change_the_gradient(torch_cuda):
    """Recomputation from checkpoints every 1, 4 or 20 steps and the stored
    tape give the same objective and gradients bit for bit (second backward
    of a runner replays the captured segments)."""
    torch = torch_cuda
    from torchannel_b200.adjoint import AdjointRunner, to_internal
    ch = _chan(32, 24, 16)
    q0 = _initial(torch, ch, 5)
    Fb = _body(torch, ch, 6)
    out = []
    for C, mode in ((1, "recompute"), (4, "recompute"), (20, "recompute"), (4, "store")):
        r = AdjointRunner(ch, 0.003, 9, range(4, 10), checkpoint_every=C, mode=mode)
        r.set_body_force(*to_internal(ch, *Fb))
        J = r.forward(*q0)
        gq, gF, mu = r.backward()
        res = (float(J), [t.cpu() for t in gq + gF], float(mu))
        gq2, gF2, mu2 = r.backward()  # replayed graphs
        for a, b in zip(res[1], gq2 + gF2):
            assert torch.equal(a, b.cpu())
        out.append(res)
    for o in out[1:]:
        assert o[0] == out[0][0]
        for a, b in zip(o[1], out[0][1]):
            assert torch.equal(a, b)
        assert o[2] == out[0][2]
