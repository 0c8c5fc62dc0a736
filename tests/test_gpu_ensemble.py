"""Ensemble on one GPU: the single-graph ensemble step against member-by-member
steps (bit-identical), and the autotuner leaves every member's state as it
found it."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _members():
    from torchannel_b200.ensemble import make_members
    return make_members(4, seed=3, sizes_xy=(32, 48, 64), sizes_z=(16, 24, 40))


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_graph_ensemble_matches_member_steps(torch_cuda, precision):
    torch = torch_cuda
    from torchannel_b200.ensemble import Ensemble
    a = Ensemble(_members(), precision=precision)
    b = Ensemble(_members(), precision=precision)
    a.capture()          # one eager step, then the graph of two steps per member
    a.step_graph(3)      # + 6 steps
    torch.cuda.synchronize()
    b.step(7, concurrent=True)
    b.synchronize()
    for ca, cb in zip(a.channels, b.channels):
        for x, y in zip(ca.get_state()[:3], cb.get_state()[:3]):
            assert torch.equal(x, y)
        assert torch.equal(ca.scalars[:2], cb.scalars[:2])


def test_autotune_restores_state(torch_cuda):
    torch = torch_cuda
    from torchannel_b200.ensemble import Ensemble
    a = Ensemble(_members(), precision="mixed")
    b = Ensemble(_members(), precision="mixed")
    for e in (a, b):
        e.step(2)
        e.synchronize()
    tun = a.autotune(steps=4, repeats=1)
    assert len(tun) == 4 and all(t["cn_rows"] in (16, 32) for t in tun)
    for x in (a, b):
        x.step(3)
        x.synchronize()
    for ca, cb in zip(a.channels, b.channels):
        for x, y in zip(ca.get_state()[:3], cb.get_state()[:3]):
            # the tuned shapes change the arithmetic only by rounding
            assert float((x - y).abs().max()) <= 1e-5 * float(y.abs().max())


@pytest.mark.parametrize("nx,ny,nz", [(16, 12, 10), (24, 36, 70)])
def test_cn_chunk_32_matches_oracle(torch_cuda, nx, ny, nz):
    from oracle import ops
    from tests._util import dof, make_gpu, make_oracle, np_, rel
    oc = make_oracle(nx, ny, nz)
    rng = np.random.default_rng(4)
    u = 1.0 + 0.1 * rng.standard_normal((nx + 1, ny + 2, nz + 2))
    v = 0.1 * rng.standard_normal((nx + 2, ny + 1, nz + 2))
    w = 0.1 * rng.standard_normal((nx + 2, ny + 2, nz + 1))
    ops.apply_bc_all(u, v, w)
    dt = 0.002
    ru = ops.solve_implicit_diffusion_uv(u, dt, nx, ny, nz, oc.dz_c, oc.dz_f, oc.nu)
    rw = ops.solve_implicit_diffusion_w(w, dt, nx, ny, nz, oc.dz_c, oc.dz_f, oc.nu)
    ch = make_gpu(oc)
    ch.set_cn_chunk(32)
    ch.set_state(u, v, w)
    ch.implicit_diffusion(dt)
    gu, gv, gw, _ = ch.get_state()
    assert rel(dof("u", np_(gu), nx, ny, nz), dof("u", ru, nx, ny, nz)) < 1e-12
    assert rel(dof("w", np_(gw), nx, ny, nz), dof("w", rw, nx, ny, nz)) < 1e-12
