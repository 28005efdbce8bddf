"""Parity of the CUDA TM2D path against the CPU oracle and the reference.

Inputs are prepared once on the CPU and copied to the GPU so both sides see
bit-identical coefficients and CPML profiles; the CUDA kernels keep the
reference's operation order without FMA contraction, so forward fields,
receivers, snapshots, adjoint fields and source gradients are bit-identical
to the oracle.  The model gradient sums its per-shot image terms step-major
(shots summed at every imaged step) instead of the reference's per-shot
accumulators: it is bit-identical to the oracle run in that order and within
the FP32 tolerance of the reference order.  The asserted tolerance
(relative L2 <= 1e-5, the FP32 bar) is written next to each equality.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from cases import clone_problem, config1_problem, hetero_inputs, hetero_problem, random_problem
from conftest import GOLDEN
from oracle_harness import rel_l2, set_grad_order
from tide_b200 import _native as nat
from tide_b200 import storage as stg
from tide_b200 import tm2d

pytestmark = pytest.mark.gpu
TOL = 1e-5  # FP32 parity bar: relative L2


def _zeros_r(pb, device="cpu"):
    return torch.zeros((pb.nt, pb.n_shots, pb.n_rec), dtype=pb.dtype, device=device)


def _cuda_forward(pb_cpu, dev):
    g = clone_problem(pb_cpu, dev)
    r = _zeros_r(g, dev)
    tm2d.native_forward(g, g.ca, g.cb, g.f, r, 0, g.nt)
    torch.cuda.synchronize()
    return g, r


def _assert_same(a, b, what):
    a, b = a.detach().cpu(), b.detach().cpu()
    err = rel_l2(a, b)
    assert err <= TOL, f"{what}: rel l2 {err}"
    assert torch.equal(a, b), f"{what}: not bit-identical (rel l2 {err})"


@pytest.mark.parametrize("stencil", [2, 4, 6, 8])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("batched", [False, True])
def test_forward_bitwise_vs_oracle(oracle, cuda_device, stencil, dtype, batched):
    pb = random_problem(100 + stencil, 45, 71, 3, 120, stencil=stencil, dtype=dtype, batched=batched)
    g, r_gpu = _cuda_forward(pb, cuda_device)
    r = _zeros_r(pb)
    oracle.forward(pb, pb.ca, pb.cb, pb.f, r)
    _assert_same(r_gpu, r, "receivers")
    for name, a, b in zip(("Ey", "Hx", "Hz", "mEyx", "mEyz", "mHxz", "mHzx"), g.fields, pb.fields):
        _assert_same(a, b, name)
    assert nat.device_status(cuda_device) == 0


def test_config1_vs_reference_cpu_golden(cuda_device):
    """Config 1 through the ABI: bit-identical to the reference CPU backend."""
    z = np.load(GOLDEN / "config1.npz")
    pb = config1_problem(torch.float32)
    _, r = _cuda_forward(pb, cuda_device)
    _assert_same(r, torch.from_numpy(z["r_native_f32"]), "config1 receivers")
    pb64 = config1_problem(torch.float64)
    _, r64 = _cuda_forward(pb64, cuda_device)
    _assert_same(r64, torch.from_numpy(z["r_native_f64"]), "config1 receivers fp64")
    # error of the FP32 result against the FP64 reference run
    assert rel_l2(r, torch.from_numpy(z["r_native_f64"])) < 1e-5


def test_config1_public_api(cuda_device):
    """Public functional API on CUDA (coefficients prepared on the GPU)."""
    import tide_b200 as tide

    z = np.load(GOLDEN / "config1.npz")
    nt, dt = 300, 4e-11
    eps = torch.full((96, 96), 4.0, device=cuda_device)
    amp = tide.ricker(800e6, nt, dt, device=cuda_device).view(1, 1, nt)
    out = tide.maxwelltm(eps, torch.zeros_like(eps), torch.ones_like(eps), 0.02, dt, amp,
                         torch.tensor([[[20, 48]]], device=cuda_device),
                         torch.tensor([[[20, 60]]], device=cuda_device), stencil=2, pml_width=10)
    assert rel_l2(out[-1], torch.from_numpy(z["r_native_f32"])) <= TOL


@pytest.mark.parametrize("fmt", [0, 1])
def test_snapshots_bitwise(oracle, cuda_device, fmt):
    pb = random_problem(7, 33, 41, 2, 50)
    S, ny, nx, nt = pb.n_shots, pb.ny, pb.nx, pb.nt
    sdt = torch.bfloat16 if fmt else torch.float32
    # oracle stores
    st_o = (torch.zeros((nt, S, ny, nx), dtype=sdt), torch.zeros((nt, S, ny, nx), dtype=sdt))
    qb = clone_problem(pb)
    r_o = _zeros_r(qb)
    oracle.forward(qb, qb.ca, qb.cb, qb.f, r_o, store=st_o, k=1, fmt=fmt, need_ca=True, need_cb=True)
    g = clone_problem(pb, cuda_device)
    snaps = stg.allocate(stg.STORAGE_DEVICE, sdt, fmt, nt, S, ny, nx, cuda_device, True, True)
    snaps.ey_dev.zero_(); snaps.curl_dev.zero_()
    r = _zeros_r(g, cuda_device)
    tm2d._run_forward_storage(g, g.ca, g.cb, g.f, r, snaps, True, True, None, 0)
    torch.cuda.synchronize()
    _assert_same(r, r_o, "receivers with storage")
    assert torch.equal(snaps.ey_dev.cpu(), st_o[0])
    assert torch.equal(snaps.curl_dev.cpu(), st_o[1])


def _abi_gradients(pb_cpu, dev, grad_r, mode=stg.STORAGE_DEVICE, fmt=0, k=None, opts=None):
    g = clone_problem(pb_cpu, dev)
    if k is not None:
        g.grad_interval = k
    S, ny, nx, nt = g.n_shots, g.ny, g.nx, g.nt
    sdt = torch.bfloat16 if fmt else g.dtype
    n_store = (nt + g.grad_interval - 1) // g.grad_interval
    snaps = stg.allocate(mode, sdt, fmt, n_store, S, ny, nx, dev, True, True)
    r = _zeros_r(g, dev)
    tm2d._run_forward_storage(g, g.ca, g.cb, g.f, r, snaps, True, True, None, 0)
    gca, gcb, gf = tm2d._run_backward(g, g.ca, g.cb, grad_r.to(dev), snaps, True, True, True,
                                      opts or {})
    torch.cuda.synchronize()
    return r, gca, gcb, gf


@pytest.mark.parametrize("stencil", [2, 4, 8])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_backward_bitwise_vs_oracle(oracle, cuda_device, stencil, dtype):
    pb = random_problem(200 + stencil, 37, 53, 3, 90, stencil=stencil, dtype=dtype)
    gen = torch.Generator().manual_seed(5)
    grad_r = torch.randn((pb.nt, pb.n_shots, pb.n_rec), generator=gen, dtype=torch.float64).to(dtype)
    r, gca, gcb, gf = _abi_gradients(pb, cuda_device, grad_r)
    qb = clone_problem(pb)
    store = (torch.zeros((pb.nt, pb.n_shots, pb.ny, pb.nx), dtype=dtype),
             torch.zeros((pb.nt, pb.n_shots, pb.ny, pb.nx), dtype=dtype))
    r_o = _zeros_r(qb)
    oracle.forward(qb, qb.ca, qb.cb, qb.f, r_o, store=store, need_ca=True, need_cb=True)
    set_grad_order(oracle, 1)
    try:
        oca, ocb, ogf, _ = oracle.backward(qb, qb.ca, qb.cb, grad_r, store)
    finally:
        set_grad_order(oracle, 0)
    _assert_same(r, r_o, "receivers")
    _assert_same(gca[0], oca, "grad_ca")
    _assert_same(gcb[0], ocb, "grad_cb")
    _assert_same(gf.reshape(ogf.shape), ogf, "grad_f")
    # against the reference's summation order: FP32 tolerance
    rca, rcb, _, _ = oracle.backward(qb, qb.ca, qb.cb, grad_r, store)
    assert rel_l2(gca[0], rca) <= TOL and rel_l2(gcb[0], rcb) <= TOL


def test_backward_batched_model(oracle, cuda_device):
    pb = random_problem(31, 29, 37, 3, 70, batched=True)
    grad_r = torch.randn((pb.nt, pb.n_shots, pb.n_rec), generator=torch.Generator().manual_seed(1))
    _, gca, gcb, _ = _abi_gradients(pb, cuda_device, grad_r)
    qb = clone_problem(pb)
    store = (torch.zeros((pb.nt, 3, pb.ny, pb.nx)), torch.zeros((pb.nt, 3, pb.ny, pb.nx)))
    oracle.forward(qb, qb.ca, qb.cb, qb.f, _zeros_r(qb), store=store, need_ca=True, need_cb=True)
    oca, ocb, _, _ = oracle.backward(qb, qb.ca, qb.cb, grad_r, store)
    _assert_same(gca, oca, "batched grad_ca")
    _assert_same(gcb, ocb, "batched grad_cb")
    assert float(gca.abs().sum()) > 0


@pytest.mark.parametrize("k", [1, 3])
def test_bf16_and_interval_vs_oracle(oracle, cuda_device, k):
    pb = random_problem(41, 31, 39, 2, 64)
    grad_r = torch.randn((pb.nt, pb.n_shots, pb.n_rec), generator=torch.Generator().manual_seed(2))
    _, gca, gcb, _ = _abi_gradients(pb, cuda_device, grad_r, fmt=1, k=k)
    qb = clone_problem(pb)
    qb.grad_interval = k
    n_store = (pb.nt + k - 1) // k
    store = (torch.zeros((n_store, 2, pb.ny, pb.nx), dtype=torch.bfloat16),
             torch.zeros((n_store, 2, pb.ny, pb.nx), dtype=torch.bfloat16))
    oracle.forward(qb, qb.ca, qb.cb, qb.f, _zeros_r(qb), store=store, k=k, fmt=1,
                   need_ca=True, need_cb=True)
    set_grad_order(oracle, 1)
    try:
        oca, ocb, _, _ = oracle.backward(qb, qb.ca, qb.cb, grad_r, store, k=k, fmt=1)
    finally:
        set_grad_order(oracle, 0)
    _assert_same(gca[0], oca, "bf16 grad_ca")
    _assert_same(gcb[0], ocb, "bf16 grad_cb")


def test_cpu_offload_mode_equals_device_mode(cuda_device):
    """Pinned-host offload on a side stream gives the same gradients."""
    pb = random_problem(51, 35, 45, 2, 80)
    grad_r = torch.randn((pb.nt, pb.n_shots, pb.n_rec), generator=torch.Generator().manual_seed(3))
    a = _abi_gradients(pb, cuda_device, grad_r, mode=stg.STORAGE_DEVICE)
    b = _abi_gradients(pb, cuda_device, grad_r, mode=stg.STORAGE_CPU)
    for x, y, n in zip(a, b, ("r", "gca", "gcb", "gf")):
        _assert_same(x, y, n)


def test_chunked_backward_equals_single(cuda_device):
    """Backward split into callback chunks (start_t continuation)."""
    pb = random_problem(61, 30, 40, 2, 75)
    grad_r = torch.randn((pb.nt, pb.n_shots, pb.n_rec), generator=torch.Generator().manual_seed(4))
    seen = []
    a = _abi_gradients(pb, cuda_device, grad_r)
    b = _abi_gradients(pb, cuda_device, grad_r,
                       opts={"backward_callback": lambda s: seen.append(s.step), "callback_frequency": 16})
    assert seen == [59, 43, 27, 11, 0]
    for x, y, n in zip(a, b, ("r", "gca", "gcb", "gf")):
        _assert_same(x, y, n)


@pytest.mark.parametrize("stencil", [2, 4])
def test_gradients_vs_reference_autograd(cuda_device, stencil):
    """Public API end to end (FP64) against the reference's exact autograd gradient."""
    import tide_b200 as tide

    z = np.load(GOLDEN / "hetero_grad.npz")
    c = hetero_inputs(torch.float64)
    eps = c["eps"].to(cuda_device).requires_grad_(True)
    sig = c["sig"].to(cuda_device).requires_grad_(True)
    out = tide.maxwelltm(eps, sig, c["mu"].to(cuda_device), c["dx"], c["dt"],
                         c["amp"].to(cuda_device), c["src"].to(cuda_device),
                         c["rec"].to(cuda_device), stencil=stencil, pml_width=c["pml"])
    loss = (out[-1] * c["w"].to(cuda_device)).sum()
    ge, gs = torch.autograd.grad(loss, [eps, sig])
    assert rel_l2(out[-1], torch.from_numpy(z[f"r_f64_s{stencil}"])) < 1e-12
    assert rel_l2(ge, torch.from_numpy(z[f"geps_f64_s{stencil}"])) < 1e-10
    assert rel_l2(gs, torch.from_numpy(z[f"gsig_f64_s{stencil}"])) < 1e-10


def test_points_edge_cases(oracle, cuda_device):
    """Duplicate, negative and out-of-domain source/receiver indices."""
    pb = random_problem(71, 26, 34, 2, 40, n_rec=6)
    N = pb.ny * pb.nx
    si = pb.sources_i.clone()
    si = torch.cat([si, si, torch.tensor([[-1], [pb.nx + 0]])], dim=1)  # duplicate + skip + fd-pad row
    pb.sources_i = si.contiguous()
    pb.n_src = 3
    f = torch.randn((pb.nt, pb.n_shots, 3), generator=torch.Generator().manual_seed(9))
    pb.f = f.reshape(-1).contiguous()
    ri = pb.receivers_i.clone()
    ri[0, 1] = ri[0, 0]
    ri[1, 2] = -1
    ri[1, 3] = N - 1  # last cell, outside the update domain
    pb.receivers_i = ri.contiguous()
    g, r_gpu = _cuda_forward(pb, cuda_device)
    r = _zeros_r(pb)
    oracle.forward(pb, pb.ca, pb.cb, pb.f, r)
    _assert_same(r_gpu, r, "receivers with edge-case points")
    _assert_same(g.fields[0], pb.fields[0], "Ey with edge-case points")


def test_no_sources_no_receivers(cuda_device):
    pb = random_problem(81, 20, 24, 1, 10)
    pb.sources_i = torch.empty(0, dtype=torch.long)
    pb.receivers_i = torch.empty(0, dtype=torch.long)
    pb.n_src = pb.n_rec = 0
    pb.f = torch.empty(0)
    g = clone_problem(pb, cuda_device)
    g.fields[0].fill_(1.0)
    tm2d.native_forward(g, g.ca, g.cb, g.f, torch.empty(0, device=cuda_device), 0, g.nt)
    torch.cuda.synchronize()
    assert torch.isfinite(g.fields[0]).all()


def test_out_of_range_index_sets_device_error(cuda_device):
    """A source index beyond the shot is skipped and reported, never written."""
    pb = random_problem(91, 20, 24, 1, 5)
    pb.sources_i = torch.tensor([[pb.ny * pb.nx + 5]])
    g = clone_problem(pb, cuda_device)
    tm2d.native_forward(g, g.ca, g.cb, g.f, _zeros_r(g, cuda_device), 0, g.nt)
    assert nat.device_status(cuda_device) == 1
    assert nat.device_status(cuda_device) == 0


def test_bad_arguments_raise_not_exit(cuda_device):
    pb = random_problem(92, 20, 24, 1, 5)
    g = clone_problem(pb, cuda_device)
    fn = nat.get_backend_function("maxwell_tm", "forward_with_storage", 2, torch.float32, cuda_device)
    with pytest.raises(nat.NativeError, match="storage_mode"):
        snaps = stg.SnapshotBuffers(7, 0, torch.float32, 5, g.ny * g.nx * 4, *(torch.empty(0),) * 4)
        tm2d._run_forward_storage(g, g.ca, g.cb, g.f, _zeros_r(g, cuda_device), snaps, True, True,
                                  None, 0)
    with pytest.raises(nat.NativeError, match="file names"):
        snaps = stg.allocate(stg.STORAGE_DISK, torch.float32, 0, 5, g.n_shots, g.ny, g.nx,
                             cuda_device, True, True)
        snaps.files = None  # no file names
        tm2d._run_forward_storage(g, g.ca, g.cb, g.f, _zeros_r(g, cuda_device), snaps, True, True,
                                  None, 0)
    del fn


def test_config2_geometry_slice(oracle, cuda_device):
    """Config-2 padded geometry (553 x 1065, CPML 20), 2 shots, 40 steps."""
    pb = random_problem(2, 512, 1024, 2, 40, pml=20, n_rec=256)
    assert (pb.ny, pb.nx) == (553, 1065)
    g, r_gpu = _cuda_forward(pb, cuda_device)
    r = _zeros_r(pb)
    oracle.forward(pb, pb.ca, pb.cb, pb.f, r)
    _assert_same(r_gpu, r, "config-2 receivers")
    _assert_same(g.fields[0], pb.fields[0], "config-2 Ey")


@pytest.mark.parametrize("dtype,compression", [(torch.float32, False), (torch.float32, True),
                                               (torch.float64, False)])
@pytest.mark.parametrize("k,chunk", [(1, 0), (1, 17), (3, 10), (2, 1)])
def test_checkpoint_gradient_equals_stored(cuda_device, dtype, compression, k, chunk):
    """storage_mode='checkpoint' (segments recomputed from saved states) gives
    bit-identical receivers and epsilon/sigma/source gradients to the stored
    history, for segment lengths that do and do not divide nt."""
    import tide_b200 as tide

    c = hetero_inputs(dtype)
    dev = cuda_device

    def run(mode):
        eps = c["eps"].to(dev).requires_grad_(True)
        sig = c["sig"].to(dev).requires_grad_(True)
        amp = c["amp"].to(dev).requires_grad_(True)
        out = tide.maxwelltm(eps, sig, c["mu"].to(dev), c["dx"], c["dt"], amp,
                             c["src"].to(dev), c["rec"].to(dev), pml_width=c["pml"],
                             model_gradient_sampling_interval=k, storage_mode=mode,
                             storage_compression=compression, storage_chunk_steps=chunk)
        loss = (out[-1] * c["w"].to(dev)).sum()
        g = torch.autograd.grad(loss, [eps, sig, amp])
        return (out[-1].detach(), *out[:7], *g)

    a, b = run("device"), run("checkpoint")
    names = ("r", "Ey", "Hx", "Hz", "mEyx", "mEyz", "mHxz", "mHzx", "geps", "gsig", "gamp")
    for x, y, n in zip(a, b, names):
        _assert_same(x, y, n)


def test_checkpoint_callbacks(cuda_device):
    """Forward and backward callbacks see the same steps and states in the
    checkpointed mode as in the stored mode."""
    import tide_b200 as tide

    c = hetero_inputs(torch.float32)
    dev = cuda_device

    def run(mode):
        seen = []
        eps = c["eps"].to(dev).requires_grad_(True)
        fcb = lambda s: seen.append(("f", s.step, float(s.wavefields["Ey"].abs().sum())))  # noqa: E731
        bcb = lambda s: seen.append(("b", s.step, float(s.wavefields["lambda_Ey"].abs().sum()),  # noqa: E731
                                     float(s.gradients["ca"].abs().sum())))
        out = tide.maxwelltm(eps, c["sig"].to(dev), c["mu"].to(dev), c["dx"], c["dt"],
                             c["amp"].to(dev), c["src"].to(dev), c["rec"].to(dev),
                             pml_width=c["pml"], storage_mode=mode, storage_chunk_steps=13,
                             forward_callback=fcb, backward_callback=bcb, callback_frequency=9)
        (out[-1] * c["w"].to(dev)).sum().backward()
        return seen, eps.grad

    sa, ga = run("device")
    sb, gb = run("checkpoint")
    assert sa == sb
    _assert_same(ga, gb, "grad eps")
