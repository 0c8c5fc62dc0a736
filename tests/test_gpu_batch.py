"""Ensemble launches (tc_batch_*): one persistent launch per substep for all
members must advance every member exactly as its own tc_step does
(bit-identical with the same CN chunk length), through the eager first step,
the two-step graph and the table rebuilds."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def _members(n=5, seed=7):
    from torchannel_b200.ensemble import make_members
    return make_members(n, seed=seed, sizes_xy=(64, 96, 128), sizes_z=(16, 24, 40))


def _pair(precision, members=None):
    from torchannel_b200.ensemble import Ensemble
    ms = members or _members()
    return Ensemble(ms, precision=precision), Ensemble(ms, precision=precision)


def _same(torch, ea, eb):
    for ca, cb in zip(ea.channels, eb.channels):
        for x, y in zip(ca.get_state()[:3], cb.get_state()[:3]):
            assert torch.equal(x, y)
        assert torch.equal(ca.scalars[:2], cb.scalars[:2])


def _rows(e, rows=16):
    """Each member's CN chunk length under the ensemble shape: the shape's
    rows for every member."""
    return [rows for _ in e.channels]


def _step_members(torch, e, n, scheme="IMEX", bound=16):
    for ch, dt, r in zip(e.channels, e.dts, _rows(e, bound)):
        ch.set_cn_chunk(r)
        ch.step(scheme, dt, n)
    torch.cuda.synchronize()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("n_steps", [1, 3, 8])
def test_batch_matches_member_steps(torch_cuda, precision, n_steps):
    torch = torch_cuda
    a, b = _pair(precision)
    a.batch()
    a.step_batch(n_steps)
    torch.cuda.synchronize()
    _step_members(torch, b, n_steps)
    _same(torch, a, b)


@pytest.mark.parametrize("scheme", ["AB2", "FE"])
def test_batch_explicit_schemes(torch_cuda, scheme):
    torch = torch_cuda
    a, b = _pair("fp64")
    dts = [0.2 * dt for dt in a.dts]  # explicit diffusion: smaller steps
    a.dts = b.dts = dts
    a.batch()
    a.step_batch(6, scheme=scheme)
    torch.cuda.synchronize()
    _step_members(torch, b, 6, scheme=scheme)
    _same(torch, a, b)


@pytest.mark.parametrize("rows,ctas", [(32, 0), (16, 1), (32, 3), (16, -1)])
def test_batch_shapes(torch_cuda, rows, ctas):
    torch = torch_cuda
    a, b = _pair("mixed")
    a.batch().set_shape(rows, ctas)
    a.step_batch(7)
    torch.cuda.synchronize()
    _step_members(torch, b, 7, bound=rows)
    _same(torch, a, b)
    info = a.batched.info()
    assert info["cn_rows"] == rows and info["ctas_per_sm"] == ctas and info["built"]
    assert a.batched.member_cn_rows() == _rows(b, rows)
    assert info["cn_chunks"] == -(-max(c.nz for c in a.channels) // rows)
    nsm = torch.cuda.get_device_properties(0).multi_processor_count
    for k, g in info["ctas"].items():
        assert 1 <= g <= info["units"][k]
        if k in ("fftx", "ifftx", "cn", "tri", "proj"):  # one CTA per unit (CN, x transforms: a launch per class)
            assert g == info["units"][k]
        elif ctas > 0:
            assert g <= ctas * nsm
        if ctas < 0 and k != "ffty":
            assert g == info["units"][k]
    # RHS, CN per chunk count, x per length, two y, z solve, inverse x per length, projection
    assert a.batched.launches_per_step() == (1 + len({-(-c.nz // rows) for c in a.channels}) + 3
                                             + 2 * len({c.nx for c in a.channels}) + 1)


def test_batch_interleaved_with_member_steps(torch_cuda):
    """A member stepped on its own between ensemble calls (buffer parity
    changes) and a dt change force the tables to be rebuilt."""
    torch = torch_cuda
    a, b = _pair("mixed")
    a.batch()
    a.step_batch(4)
    torch.cuda.synchronize()
    a.channels[1].step("IMEX", a.dts[1], 1)
    old = list(a.dts)
    a.dts = b.dts = [0.9 * dt for dt in old]
    a.step_batch(5)
    torch.cuda.synchronize()
    for i, (ch, dt0, dt, r) in enumerate(zip(b.channels, old, b.dts, _rows(b))):
        ch.set_cn_chunk(r)
        ch.step("IMEX", dt0, 4)
        if i == 1:
            ch.step("IMEX", dt0, 1)
        ch.step("IMEX", dt, 5)
    torch.cuda.synchronize()
    _same(torch, a, b)


def test_batch_uneven_large_members(torch_cuda):
    """Members up to 256 points in x / y (the N1 <= 16 kernel set) and nz
    above 256 (32-row CN chunks)."""
    torch = torch_cuda
    ms = [dict(nx=256, ny=64, nz=20, Re=3000.0, gamma=2.4, seed=1),
          dict(nx=64, ny=192, nz=300, Re=2500.0, gamma=2.6, seed=2),
          dict(nx=96, ny=96, nz=12, Re=4000.0, gamma=2.2, seed=3)]
    a, b = _pair("mixed", ms)
    a.batch()
    assert a.batched.info()["cn_rows"] == 32
    a.step_batch(6)
    torch.cuda.synchronize()
    _step_members(torch, b, 6, bound=32)
    _same(torch, a, b)


def test_batch_rejects_unsupported(torch_cuda):
    from torchannel_b200 import _lib as L
    from torchannel_b200.ensemble import ChannelBatch, Ensemble
    e = Ensemble(_members(2) + [dict(nx=48, ny=64, nz=16, Re=3000.0, gamma=2.4, seed=9)], precision="fp64")
    with pytest.raises(L.TCError):
        ChannelBatch(e.channels)
    e2 = Ensemble(_members(2), precision="fp64")
    m = Ensemble(_members(1), precision="mixed")
    with pytest.raises(L.TCError):
        ChannelBatch(e2.channels + m.channels)
    with pytest.raises(L.TCError):
        ChannelBatch([e2.channels[0], e2.channels[0]])


def test_batch_autotune_restores_state(torch_cuda):
    torch = torch_cuda
    a, b = _pair("mixed")
    a.batch()
    tun = a.autotune_batch(steps=4, repeats=1, ctas=(-1, 2))
    assert tun["cn_rows"] in (16, 32) and len(tun["ms_per_step"]) == 4
    a.batched.set_shape(16, 0)
    a.step_batch(4)
    torch.cuda.synchronize()
    _step_members(torch, b, 4)
    for ca, cb in zip(a.channels, b.channels):
        for x, y in zip(ca.get_state()[:3], cb.get_state()[:3]):
            # a restored mixed state re-derives its base profile: rounding only
            assert float((x - y).abs().max()) <= 1e-5 * float(y.abs().max())


def test_batch_stays_divergence_free(torch_cuda):
    torch = torch_cuda
    from torchannel_b200.ensemble import Ensemble
    e = Ensemble(_members(6, seed=11), precision="mixed")
    e.batch()
    e.step_batch(20)
    torch.cuda.synchronize()
    for d in e.diagnostics():
        assert np.isfinite(d["max_div"]) and d["max_div"] < 1e-5


def test_autotune_mode_restores_state(torch_cuda):
    torch = torch_cuda
    from torchannel_b200.ensemble import Ensemble
    e = Ensemble(_members(3, seed=5), precision="fp64")
    before = [[t.clone() for t in ch.get_state()[:3]] for ch in e.channels]
    times = e.autotune_mode(steps=2, repeats=1)
    assert set(times) == {"batch", "streams"} and e.mode in times
    for ch, b in zip(e.channels, before):
        for x, y in zip(ch.get_state()[:3], b):
            assert torch.equal(x, y)


def test_batch_rhs_follows_member_rhs_form(torch_cuda):
    """The ensemble's RHS stages its tiles by tensor copies (kb_rhs_tma, one
    unit per k_rhs_tma tile) while every member has its tensor-copy RHS on in
    the default shape, and runs the per-thread staged kernel otherwise; a
    member switched between ensemble calls rebuilds the tables, and the
    members stay bit-identical to their own steps through both forms."""
    torch = torch_cuda
    from torchannel_b200.ensemble import Ensemble
    ms = _members(4, seed=3)
    a, b = Ensemble(ms, precision="mixed"), Ensemble(ms, precision="mixed")
    a.batch()
    a.step_batch(5)
    torch.cuda.synchronize()
    tiles = sum(-(-c.nx // 32) * -(-c.ny // 8) * -(-c.nz // 8) for c in a.channels)
    assert a.batched.info()["units"]["rhs"] == tiles
    a.channels[2].use_tma_rhs(0)
    b.channels[2].use_tma_rhs(0)
    a.step_batch(4)
    torch.cuda.synchronize()
    assert a.batched.info()["units"]["rhs"] != tiles
    a.channels[2].use_tma_rhs(1)
    b.channels[2].use_tma_rhs(1)
    a.batched.set_shape(16, -1)
    a.step_batch(5)
    torch.cuda.synchronize()
    info = a.batched.info()
    assert info["units"]["rhs"] == tiles and info["ctas"]["rhs"] == tiles
    _step_members(torch, b, 14)
    _same(torch, a, b)


def test_batch_rhs_member_groups(torch_cuda):
    """More members than one RHS launch parameter holds (32): the tensor-copy
    RHS runs as one launch per group, bit-identical to the members' steps."""
    torch = torch_cuda
    from torchannel_b200.ensemble import make_members
    a, b = _pair("mixed", make_members(34, seed=4, sizes_xy=(64,), sizes_z=(16, 24)))
    a.batch()
    a.step_batch(5)
    torch.cuda.synchronize()
    _step_members(torch, b, 5)
    _same(torch, a, b)
