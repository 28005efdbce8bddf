"""Operator layer: the 3-D checkpoint-and-recompute gradient, storage modes,
initial-state continuation, CFL sub-stepping and the Maxwell3D operator;
linearizations of MaxwellTM and Maxwell3D (repeated vjps).

The checkpoint gradient recomputes each segment's snapshots bit for bit and
chains the adjoint state across segments.  With one shot (or a batched
model) the coefficient gradient accumulates into one buffer in the same
order as the stored-history pass, so it is bit-identical; with several shots
of one model each adjoint call sums its per-shot accumulators once, so the
segments add partial sums: equal within the stated tolerance (FP32 relative
L2 <= 1e-5, FP64 <= 1e-12).  Everything else is asserted bit-identical.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import tide_b200 as tide
from oracle_harness import rel_l2
from tide_b200 import em3d

pytestmark = pytest.mark.gpu


def _case(seed, nz, ny, nx, shots, nt, dtype=torch.float32, n_rec=5, batched=False):
    g = torch.Generator().manual_seed(seed)
    shape = (shots, nz, ny, nx) if batched else (nz, ny, nx)
    eps = (1.5 + 6.0 * torch.rand(shape, generator=g, dtype=torch.float64)).to(dtype)
    sig = (0.006 * torch.rand(shape, generator=g, dtype=torch.float64)).to(dtype)
    mu = torch.ones(shape, dtype=dtype)
    dx = 0.02
    dt = 0.9 * dx / (299792458.0 / float(eps.min().double().sqrt()) * 3 ** 0.5)
    t = torch.arange(nt, dtype=torch.float64) * dt
    amp = torch.sin(2 * np.pi * 6e8 * t) * torch.exp(-((t - 3e-9) / 1e-9) ** 2)
    amp = (amp.view(1, 1, nt).repeat(shots, 1, 1)
           * (1 + 0.2 * torch.arange(shots)).view(shots, 1, 1)).to(dtype)
    src = torch.stack([torch.randint(2, n - 2, (shots, 1), generator=g) for n in (nz, ny, nx)], -1)
    rec = torch.stack([torch.randint(0, n, (shots, n_rec), generator=g) for n in (nz, ny, nx)], -1)
    return dict(eps=eps, sig=sig, mu=mu, dx=dx, dt=dt, amp=amp, src=src, rec=rec)


def _run(c, dev, *, grads=True, seed=4, **kw):
    eps = c["eps"].to(dev).requires_grad_(grads)
    sig = c["sig"].to(dev).requires_grad_(grads)
    out = em3d.maxwell3d(eps, sig, c["mu"].to(dev), c["dx"], c["dt"], c["amp"].to(dev),
                         c["src"].to(dev), c["rec"].to(dev), pml_width=3, **kw)
    r = out[-1]
    state = [t.detach().clone() for t in out[:-1]]
    if not grads:
        return r.detach(), state, None, None
    w = torch.randn(r.shape, generator=torch.Generator().manual_seed(seed), dtype=r.dtype).to(dev)
    (r * w).sum().backward()
    after = [t.detach() for t in out[:-1]]
    for a, b in zip(state, after):
        assert torch.equal(a, b), "backward changed the returned final state"
    return r.detach(), state, eps.grad.detach(), sig.grad.detach()


@pytest.mark.parametrize("dtype,shots,batched,k,seg", [
    (torch.float64, 1, False, 1, 7), (torch.float32, 1, False, 2, 8),
    (torch.float64, 3, False, 1, 10), (torch.float32, 3, False, 2, 6),
    (torch.float32, 2, True, 1, 9),
])
def test_checkpoint_gradient_equals_stored(cuda_device, dtype, shots, batched, k, seg):
    c = _case(11 + shots, 9, 10, 11, shots, 40, dtype=dtype, batched=batched)
    kw = dict(model_gradient_sampling_interval=k)
    r_d, st_d, ge_d, gs_d = _run(c, cuda_device, storage_mode="device", **kw)
    r_c, st_c, ge_c, gs_c = _run(c, cuda_device, storage_mode="checkpoint",
                                 storage_chunk_steps=seg, **kw)
    assert torch.equal(r_d.cpu(), r_c.cpu())
    for a, b in zip(st_d, st_c):
        assert torch.equal(a.cpu(), b.cpu())
    tol = 1e-12 if dtype == torch.float64 else 1e-5
    if shots == 1 or batched:
        assert torch.equal(ge_d.cpu(), ge_c.cpu()) and torch.equal(gs_d.cpu(), gs_c.cpu())
    assert rel_l2(ge_c, ge_d) <= tol and rel_l2(gs_c, gs_d) <= tol
    assert float(ge_d.abs().sum()) > 0


def test_checkpoint_bf16_equals_stored_bf16(cuda_device):
    c = _case(5, 10, 9, 12, 2, 36)
    kw = dict(storage_compression=True)
    r_d, _, ge_d, gs_d = _run(c, cuda_device, storage_mode="device", **kw)
    r_c, _, ge_c, gs_c = _run(c, cuda_device, storage_mode="checkpoint", storage_chunk_steps=5, **kw)
    assert torch.equal(r_d.cpu(), r_c.cpu())
    assert rel_l2(ge_c, ge_d) <= 1e-5 and rel_l2(gs_c, gs_d) <= 1e-5
    # BF16 snapshots against FP32 snapshots: the stated BF16 gradient error
    _, _, ge_f, gs_f = _run(c, cuda_device, storage_mode="device")
    assert rel_l2(ge_d, ge_f) < 1e-2 and rel_l2(gs_d, gs_f) < 1e-2


def test_cpu_and_auto_modes_equal_device(cuda_device):
    c = _case(7, 8, 9, 10, 2, 30)
    _, _, ge_d, gs_d = _run(c, cuda_device, storage_mode="device")
    _, _, ge_c, gs_c = _run(c, cuda_device, storage_mode="cpu")
    _, _, ge_a, gs_a = _run(c, cuda_device, storage_mode="auto", storage_bytes_limit_device=1)
    for a, b in ((ge_d, ge_c), (gs_d, gs_c), (ge_d, ge_a), (gs_d, gs_a)):
        assert torch.equal(a.cpu(), b.cpu())


def test_initial_state_continuation(cuda_device):
    """Two calls of 20 steps chained through the returned state equal one
    call of 40 steps (receivers and final state, bit for bit)."""
    c = _case(17, 9, 8, 10, 2, 40)
    r_full, st_full, _, _ = _run(c, cuda_device, grads=False)
    c1 = dict(c, amp=c["amp"][..., :20])
    r1, st1, _, _ = _run(c1, cuda_device, grads=False)
    init = dict(zip(("Ex_0", "Ey_0", "Ez_0", "Hx_0", "Hy_0", "Hz_0") + em3d.MEM_NAMES, st1))
    c2 = dict(c, amp=c["amp"][..., 20:])
    r2, st2, _, _ = _run(c2, cuda_device, grads=False, **init)
    assert torch.equal(torch.cat([r1, r2]).cpu(), r_full.cpu())
    for a, b in zip(st2, st_full):
        assert torch.equal(a.cpu(), b.cpu())


def test_cfl_substepping(cuda_device):
    """dt above the CFL bound runs ratio internal steps: equal to a run at
    the internal dt with the upsampled source, receivers downsampled."""
    c = _case(23, 8, 8, 9, 1, 30, dtype=torch.float64)
    dt_user = 2.5 * c["dt"]
    vmax = float((1.0 / torch.sqrt(c["eps"] * c["mu"])).max()) * tide.C0
    with pytest.warns(UserWarning):
        inner, ratio = tide.cfl_condition([c["dx"]] * 3, dt_user, vmax)
    assert ratio == 3
    cu = dict(c, dt=dt_user)
    with pytest.warns(UserWarning):
        r_u, st_u, _, _ = _run(cu, cuda_device, grads=False)
    ci = dict(c, dt=inner, amp=tide.upsample(c["amp"].to(cuda_device), ratio))
    r_i, st_i, _, _ = _run(ci, cuda_device, grads=False)
    assert r_u.shape == (30, 1, 5)
    assert torch.equal(r_u.cpu(), tide.downsample(r_i.movedim(0, -1), ratio).movedim(-1, 0).cpu())
    for a, b in zip(st_u, st_i):
        assert torch.equal(a.cpu(), b.cpu())


def test_maxwell3d_operator(cuda_device):
    c = _case(29, 9, 10, 8, 2, 32)
    dev = cuda_device
    acq = tide.Acquisition(c["src"].to(dev), c["rec"].to(dev))
    exp = tide.Experiment(acq, c["amp"].to(dev))
    disc = tide.Discretization(c["dx"], c["dt"], boundary=tide.CPML(3))
    op = tide.Maxwell3D(disc, exp, storage=tide.StorageOptions(mode=tide.StorageMode.CHECKPOINT))
    model = tide.EMModel(c["eps"].to(dev), c["sig"].to(dev), c["mu"].to(dev))
    res = op(model)
    r_f, st_f, _, _ = _run(c, dev, grads=False)
    assert torch.equal(res.receiver_data.cpu(), r_f.cpu())
    for a, b in zip(res.final_state.tensors(), st_f):
        assert torch.equal(a.cpu(), b.cpu())
    # continuation through EM3DState
    res2 = op(model, state=res.final_state)
    assert res2.receiver_data.shape == res.receiver_data.shape
    # linearize: vjp equals the autograd gradient
    lin = op.linearize(model)
    w = torch.randn(res.receiver_data.shape, generator=torch.Generator().manual_seed(4),
                    dtype=res.receiver_data.dtype).to(dev)
    g = lin.vjp(w)
    _, _, ge, gs = _run(c, dev, storage_mode="checkpoint")
    assert torch.equal(g.epsilon.cpu(), ge.cpu()) and torch.equal(g.sigma.cpu(), gs.cpu())
    assert torch.equal(lin.primal.receiver_data.cpu(), r_f.cpu())
    g2 = lin.vjp(w)  # the checkpoints are kept for further vjps
    assert torch.equal(g2.epsilon.cpu(), g.epsilon.cpu())
    g3 = lin.vjp(2 * w)  # linear in the cotangent
    assert rel_l2(g3.epsilon, 2 * g.epsilon) <= 1e-6


@pytest.mark.parametrize("mode", ["device", "checkpoint", "cpu"])
def test_maxwelltm_linearize_repeated_vjp(cuda_device, mode):
    dev = cuda_device
    g = torch.Generator().manual_seed(3)
    ny, nx, S, nt = 30, 44, 2, 60
    eps = (2.0 + 4.0 * torch.rand((ny, nx), generator=g, dtype=torch.float64)).float().to(dev)
    sig = (0.005 * torch.rand((ny, nx), generator=g, dtype=torch.float64)).float().to(dev)
    mu = torch.ones((ny, nx), device=dev)
    dx = 0.02
    dt = 0.9 * dx / (tide.C0 / float(eps.min().sqrt()) * 2 ** 0.5)
    amp = tide.ricker(500e6, nt, dt, dtype=torch.float32).view(1, 1, nt).repeat(S, 1, 1).to(dev)
    src = torch.tensor([[[10, 12]], [[15, 30]]], device=dev)
    rec = torch.tensor([[[5, 5 + 3 * j] for j in range(10)]] * S, device=dev)
    op = tide.MaxwellTM(tide.Discretization(dx, dt, boundary=tide.CPML(8)),
                        tide.Experiment(tide.Acquisition(src, rec), amp),
                        storage=tide.StorageOptions(mode=tide.StorageMode(mode)))
    model = tide.EMModel(eps, sig, mu)
    lin = op.linearize(model)
    w = torch.randn(lin.primal.receiver_data.shape, generator=torch.Generator().manual_seed(1)).to(dev)
    g1 = lin.vjp(w)
    g2 = lin.vjp(w)
    assert torch.equal(g1.epsilon.cpu(), g2.epsilon.cpu())
    assert torch.equal(g1.sigma.cpu(), g2.sigma.cpu())
    # equals a plain autograd gradient through the functional API
    e = eps.clone().requires_grad_(True)
    s_ = sig.clone().requires_grad_(True)
    out = tide.maxwelltm(e, s_, mu, dx, dt, amp, src, rec, pml_width=8, storage_mode=mode)
    (out[-1] * w).sum().backward()
    assert torch.equal(e.grad.cpu(), g1.epsilon.cpu()) and torch.equal(s_.grad.cpu(), g1.sigma.cpu())


def test_unbuilt_options_raise(cuda_device):
    c = _case(3, 6, 6, 6, 1, 5)
    with pytest.raises(NotImplementedError):
        _run(c, cuda_device, grads=False, forward_callback=lambda s: None)


@pytest.mark.parametrize("mode", ["cpu", "disk"])
@pytest.mark.parametrize("dtype,shots,k,compression", [
    (torch.float64, 2, 1, False), (torch.float32, 3, 2, False), (torch.float32, 1, 1, "bf16"),
])
def test_3d_host_and_disk_storage_equal_device(cuda_device, tmp_path, mode, dtype, shots, k,
                                               compression):
    """cpu (pinned host history, copies on a storage stream) and disk (one
    file per snapshot kind through a pinned staging ring) give the device
    mode's receivers and gradients bit for bit; the files are removed."""
    c = _case(21 + shots, 9, 10, 11, shots, 37, dtype=dtype)
    kw = dict(model_gradient_sampling_interval=k, storage_compression=compression)
    ref = _run(c, cuda_device, storage_mode="device", **kw)
    got = _run(c, cuda_device, storage_mode=mode, storage_path=str(tmp_path), **kw)
    assert torch.equal(ref[0], got[0])
    assert torch.equal(ref[2], got[2]) and torch.equal(ref[3], got[3])
    import gc

    gc.collect()
    assert list(tmp_path.iterdir()) == []
