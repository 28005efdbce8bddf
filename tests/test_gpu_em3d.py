"""Parity of the CUDA 3-D Maxwell (Yee) path against the 3-D CPU oracle.

Problems are prepared once on the CPU (tide_b200.em3d.prepare_em3d) and
copied to the GPU, so both sides see identical coefficients, CPML profiles
and indices.  The kernels keep the reference's operation order without FMA
contraction and divide by kappa as the reference CPU backend does, so
receivers, fields, CPML memories, snapshots, adjoint fields, source
gradients and coefficient gradients are bit-identical to the oracle (which
is itself bit-identical to the reference CPU forward and equal to the
reference's autograd gradient, see test_em3d_oracle.py).  The FP32 bar
(relative L2 <= 1e-5) is asserted next to every equality.
"""

from __future__ import annotations

import copy

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from oracle_harness import Oracle3D, rel_l2
from tide_b200 import _native as nat
from tide_b200 import em3d
from tide_b200 import storage as stg

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _same(a, b, what):
    a, b = a.detach().cpu(), b.detach().cpu()
    err = rel_l2(a, b)
    assert err <= TOL, f"{what}: rel l2 {err}"
    assert torch.equal(a, b), f"{what}: not bit-identical (rel l2 {err})"


def _to(pb, dev):
    q = copy.copy(pb)
    mv = lambda t: t.detach().to(dev).clone()  # noqa: E731
    q.ca, q.cb, q.cq, q.f = mv(pb.ca), mv(pb.cb), mv(pb.cq), mv(pb.f)
    q.profiles = {k: mv(v) for k, v in pb.profiles.items()}
    q.sources_i, q.receivers_i = mv(pb.sources_i), mv(pb.receivers_i)
    q.fields = [mv(t) for t in pb.fields]
    q.memories = [mv(t) for t in pb.memories]
    q.device = torch.device(dev)
    return q


def _problem(seed, nz, ny, nx, shots, nt, *, pml=3, dtype=torch.float32, batched=False,
             comps=("ey", "ey"), k=1, n_rec=4, stencil=2):
    g = torch.Generator().manual_seed(seed)
    shape = (shots, nz, ny, nx) if batched else (nz, ny, nx)
    eps = 1.5 + 6.0 * torch.rand(shape, generator=g, dtype=torch.float64)
    sig = 0.006 * torch.rand(shape, generator=g, dtype=torch.float64)
    mu = torch.ones(shape, dtype=torch.float64)
    dx = 0.02
    dt = 0.9 * dx / (299792458.0 / float(eps.min().sqrt()) * 3 ** 0.5)
    dt = dt if stencil == 2 else 0.5 * dt  # inside the stability limit of orders 4 to 8
    t = torch.arange(nt, dtype=torch.float64) * dt
    amp = (torch.sin(2 * np.pi * 6e8 * t) * torch.exp(-((t - 3e-9) / 1e-9) ** 2))
    amp = amp.view(1, 1, nt).repeat(shots, 1, 1) * (1 + 0.2 * torch.arange(shots)).view(shots, 1, 1)
    src = torch.stack([torch.randint(0, n, (shots, 1), generator=g) for n in (nz, ny, nx)], -1)
    rec = torch.stack([torch.randint(0, n, (shots, n_rec), generator=g) for n in (nz, ny, nx)], -1)
    return em3d.prepare_em3d(eps.to(dtype), sig.to(dtype), mu.to(dtype), dx, dt, amp.to(dtype),
                             src, rec, pml_width=pml, source_component=comps[0],
                             receiver_component=comps[1], model_gradient_sampling_interval=k,
                             stencil=stencil)


def _unpack(pb, mems, axes):
    return [pb.layout.unpack(m.cpu(), a) for m, a in zip(mems, axes)]


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("batched", [False, True])
@pytest.mark.parametrize("shape", [(9, 11, 13, 2), (5, 4, 40, 3), (20, 16, 12, 1)])
def test_forward_bitwise_vs_oracle(cuda_device, dtype, batched, shape):
    nz, ny, nx, pml = shape
    pb = _problem(7 + nz, nz, ny, nx, 2, 45, pml=pml, dtype=dtype, batched=batched,
                  comps=("ez", "ex") if nz == 5 else ("ey", "ey"))
    g = _to(pb, cuda_device)
    r = torch.zeros((g.nt, g.n_shots, g.n_rec), device=cuda_device, dtype=dtype)
    em3d.native_forward(g, g.ca, g.cb, g.f, r, 0, g.nt)
    torch.cuda.synchronize()
    r_o = torch.zeros((pb.nt, pb.n_shots, pb.n_rec), dtype=dtype)
    f_o, m_o = Oracle3D.full_state(pb)
    Oracle3D().forward(pb, pb.ca, pb.cb, pb.f, r_o, f_o, m_o)
    _same(r, r_o, "receivers")
    for name, a, b in zip("Ex Ey Ez Hx Hy Hz".split(), g.fields, f_o):
        _same(a, b, name)
    for name, a, b in zip(em3d.MEM_NAMES, _unpack(pb, g.memories, em3d.MEM_AXES), m_o):
        _same(a, b, name)
    assert nat.device_status(cuda_device) == 0


def _fwd_store(pb, dev, fmt, mode=stg.STORAGE_DEVICE):
    g = _to(pb, dev)
    sn = em3d.allocate_snapshots(g, mode, fmt, True, True)
    for t in sn.dev + sn.host:
        t.zero_()
    r = torch.zeros((g.nt, g.n_shots, g.n_rec), device=dev, dtype=g.dtype)
    em3d.native_forward_storage(g, g.ca, g.cb, g.f, r, sn, True, True)
    torch.cuda.synchronize()
    return g, r, sn


@pytest.mark.parametrize("fmt", [0, 1])
@pytest.mark.parametrize("k", [1, 3])
def test_snapshots_bitwise(cuda_device, fmt, k):
    pb = _problem(21, 8, 9, 10, 2, 30, k=k)
    g, r, sn = _fwd_store(pb, cuda_device, fmt)
    n_store = (pb.nt + k - 1) // k
    sdt = torch.bfloat16 if fmt else torch.float32
    st_o = [torch.zeros((n_store, pb.n_shots, pb.nz, pb.ny, pb.nx), dtype=sdt) for _ in range(6)]
    r_o = torch.zeros((pb.nt, pb.n_shots, pb.n_rec))
    f_o, m_o = Oracle3D.full_state(pb)
    Oracle3D().forward(pb, pb.ca, pb.cb, pb.f, r_o, f_o, m_o, store=st_o, k=k, fmt=fmt)
    _same(r, r_o, "receivers with storage")
    for c in range(6):
        assert torch.equal(sn.dev[c].cpu(), st_o[c]), f"snapshot component {c}"


def test_cpu_offload_equals_device(cuda_device):
    pb = _problem(22, 8, 9, 10, 2, 20)
    _, r_d, sd = _fwd_store(pb, cuda_device, 0, stg.STORAGE_DEVICE)
    _, r_c, sc = _fwd_store(pb, cuda_device, 0, stg.STORAGE_CPU)
    assert torch.equal(r_d.cpu(), r_c.cpu())
    for c in range(6):
        assert torch.equal(sd.dev[c].cpu().reshape(-1), sc.host[c].reshape(-1))


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("batched,shots", [(False, 1), (False, 3), (True, 2)])
@pytest.mark.parametrize("k", [1, 2])
def test_backward_bitwise_vs_oracle(cuda_device, dtype, batched, shots, k):
    pb = _problem(31 + shots, 9, 10, 11, shots, 36, dtype=dtype, batched=batched, k=k,
                  comps=("ex", "ez"))
    g, r, sn = _fwd_store(pb, cuda_device, 0)
    grad_r = torch.randn((pb.nt, pb.n_shots, pb.n_rec), generator=torch.Generator().manual_seed(3),
                         dtype=dtype)
    mshape = pb.ca.shape
    geps = torch.zeros(mshape, device=cuda_device, dtype=dtype)
    gsig = torch.zeros(mshape, device=cuda_device, dtype=dtype)
    lam = {"fields": [torch.zeros((pb.n_shots, pb.nz, pb.ny, pb.nx), device=cuda_device, dtype=dtype)
                      for _ in range(6)],
           "mem": [pb.layout.zeros(a, cuda_device, dtype) for a in em3d.ADJ_MEM_AXES]}
    gca, gcb, gf = em3d.native_backward(g, g.ca, g.cb, grad_r.to(cuda_device), sn, True, True, True,
                                        grad_eps=geps, grad_sigma=gsig, lam=lam)
    torch.cuda.synchronize()
    # oracle: same forward with stored history, then the adjoint
    n_store = (pb.nt + k - 1) // k
    st_o = [torch.zeros((n_store, pb.n_shots, pb.nz, pb.ny, pb.nx), dtype=dtype) for _ in range(6)]
    r_o = torch.zeros((pb.nt, pb.n_shots, pb.n_rec), dtype=dtype)
    f_o, m_o = Oracle3D.full_state(pb)
    o = Oracle3D()
    o.forward(pb, pb.ca, pb.cb, pb.f, r_o, f_o, m_o, store=st_o, k=k)
    oca, ocb, ogf, ol, olm, oeps, osig = o.backward(pb, pb.ca, pb.cb, grad_r, st_o, k=k,
                                                   eps_sigma=True)
    _same(r, r_o, "receivers")
    _same(gca.reshape(oca.shape), oca, "grad ca")
    _same(gcb.reshape(ocb.shape), ocb, "grad cb")
    _same(gf.reshape(ogf.shape), ogf, "grad f")
    _same(geps.reshape(oeps.shape), oeps, "grad eps")
    _same(gsig.reshape(osig.shape), osig, "grad sigma")
    for name, a, b in zip("lEx lEy lEz lHx lHy lHz".split(), lam["fields"], ol):
        _same(a, b, name)
    for i, (a, b) in enumerate(zip(_unpack(pb, lam["mem"], em3d.ADJ_MEM_AXES), olm)):
        _same(a, b, f"adjoint memory {i}")
    assert nat.device_status(cuda_device) == 0


def test_public_api_fp64_vs_reference_golden(cuda_device):
    """tide_b200.em3d.maxwell3d in FP64 against the reference's functional
    API (golden fixture): receivers and epsilon/sigma gradients."""
    z = np.load(GOLDEN / "em3d_case.npz")
    dev = cuda_device
    eps = torch.from_numpy(z["eps"]).to(dev).requires_grad_(True)
    sig = torch.from_numpy(z["sig"]).to(dev).requires_grad_(True)
    mu = torch.from_numpy(z["mu"]).to(dev)
    out = em3d.maxwell3d(eps, sig, mu, float(z["dx"]), float(z["dt"]),
                         torch.from_numpy(z["amp"]).to(dev), torch.from_numpy(z["src"]).to(dev),
                         torch.from_numpy(z["rec"]).to(dev), pml_width=int(z["pml"]))
    r = out[-1]
    assert rel_l2(r, torch.from_numpy(z["r_native_f64"])) < 1e-13
    w = torch.randn(r.shape, generator=torch.Generator().manual_seed(5), dtype=r.dtype).to(dev)
    (r * w).sum().backward()
    assert rel_l2(eps.grad, torch.from_numpy(z["geps_python_f64"])) < 1e-9
    assert rel_l2(sig.grad, torch.from_numpy(z["gsig_python_f64"])) < 1e-9


def test_bad_arguments_raise_not_exit(cuda_device):
    pb = _problem(41, 6, 6, 6, 1, 5)
    g = _to(pb, cuda_device)
    g.src_comp = 5
    with pytest.raises(nat.NativeError, match="component"):
        em3d.native_forward(g, g.ca, g.cb, g.f, torch.zeros((5, 1, g.n_rec), device=cuda_device),
                            0, 5)


# ------------------------------------------------------- stencil orders 4, 6, 8
@pytest.mark.parametrize("stencil", [4, 6, 8])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("batched", [False, True])
@pytest.mark.parametrize("shape", [(9, 11, 13, 2), (5, 4, 40, 3)])
def test_high_order_forward_bitwise_vs_oracle(cuda_device, stencil, dtype, batched, shape):
    nz, ny, nx, pml = shape
    pb = _problem(7 + nz + stencil, nz, ny, nx, 2, 40, pml=pml, dtype=dtype, batched=batched,
                  comps=("ez", "ex") if nz == 5 else ("ey", "ey"), stencil=stencil)
    g = _to(pb, cuda_device)
    r = torch.zeros((g.nt, g.n_shots, g.n_rec), device=cuda_device, dtype=dtype)
    em3d.native_forward(g, g.ca, g.cb, g.f, r, 0, g.nt)
    torch.cuda.synchronize()
    r_o = torch.zeros((pb.nt, pb.n_shots, pb.n_rec), dtype=dtype)
    f_o, m_o = Oracle3D.full_state(pb)
    Oracle3D().forward(pb, pb.ca, pb.cb, pb.f, r_o, f_o, m_o)
    assert float(r_o.abs().max()) > 0
    _same(r, r_o, "receivers")
    for name, a, b in zip("Ex Ey Ez Hx Hy Hz".split(), g.fields, f_o):
        _same(a, b, name)
    for name, a, b in zip(em3d.MEM_NAMES, _unpack(pb, g.memories, em3d.MEM_AXES), m_o):
        _same(a, b, name)
    assert nat.device_status(cuda_device) == 0


@pytest.mark.parametrize("stencil", [4, 8])
@pytest.mark.parametrize("fmt", [0, 1])
def test_high_order_snapshots_bitwise(cuda_device, stencil, fmt):
    k = 2
    pb = _problem(23, 8, 9, 10, 2, 24, k=k, stencil=stencil)
    g, r, sn = _fwd_store(pb, cuda_device, fmt)
    n_store = (pb.nt + k - 1) // k
    sdt = torch.bfloat16 if fmt else torch.float32
    st_o = [torch.zeros((n_store, pb.n_shots, pb.nz, pb.ny, pb.nx), dtype=sdt) for _ in range(6)]
    r_o = torch.zeros((pb.nt, pb.n_shots, pb.n_rec))
    f_o, m_o = Oracle3D.full_state(pb)
    Oracle3D().forward(pb, pb.ca, pb.cb, pb.f, r_o, f_o, m_o, store=st_o, k=k, fmt=fmt)
    _same(r, r_o, "receivers with storage")
    for c in range(6):
        assert torch.equal(sn.dev[c].cpu(), st_o[c]), f"snapshot component {c}"


@pytest.mark.parametrize("stencil", [4, 6, 8])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("batched,shots,k", [(False, 1, 1), (False, 3, 2), (True, 2, 1)])
def test_high_order_backward_bitwise_vs_oracle(cuda_device, stencil, dtype, batched, shots, k):
    pb = _problem(31 + shots + stencil, 9, 10, 11, shots, 30, dtype=dtype, batched=batched, k=k,
                  comps=("ex", "ez"), stencil=stencil)
    g, r, sn = _fwd_store(pb, cuda_device, 0)
    grad_r = torch.randn((pb.nt, pb.n_shots, pb.n_rec), generator=torch.Generator().manual_seed(3),
                         dtype=dtype)
    mshape = pb.ca.shape
    geps = torch.zeros(mshape, device=cuda_device, dtype=dtype)
    gsig = torch.zeros(mshape, device=cuda_device, dtype=dtype)
    lam = {"fields": [torch.zeros((pb.n_shots, pb.nz, pb.ny, pb.nx), device=cuda_device, dtype=dtype)
                      for _ in range(6)],
           "mem": [pb.layout.zeros(a, cuda_device, dtype) for a in em3d.ADJ_MEM_AXES]}
    gca, gcb, gf = em3d.native_backward(g, g.ca, g.cb, grad_r.to(cuda_device), sn, True, True, True,
                                        grad_eps=geps, grad_sigma=gsig, lam=lam)
    torch.cuda.synchronize()
    n_store = (pb.nt + k - 1) // k
    st_o = [torch.zeros((n_store, pb.n_shots, pb.nz, pb.ny, pb.nx), dtype=dtype) for _ in range(6)]
    r_o = torch.zeros((pb.nt, pb.n_shots, pb.n_rec), dtype=dtype)
    f_o, m_o = Oracle3D.full_state(pb)
    o = Oracle3D()
    o.forward(pb, pb.ca, pb.cb, pb.f, r_o, f_o, m_o, store=st_o, k=k)
    oca, ocb, ogf, ol, olm, oeps, osig = o.backward(pb, pb.ca, pb.cb, grad_r, st_o, k=k,
                                                   eps_sigma=True)
    assert float(oca.abs().max()) > 0
    _same(r, r_o, "receivers")
    _same(gca.reshape(oca.shape), oca, "grad ca")
    _same(gcb.reshape(ocb.shape), ocb, "grad cb")
    _same(gf.reshape(ogf.shape), ogf, "grad f")
    _same(geps.reshape(oeps.shape), oeps, "grad eps")
    _same(gsig.reshape(osig.shape), osig, "grad sigma")
    for name, a, b in zip("lEx lEy lEz lHx lHy lHz".split(), lam["fields"], ol):
        _same(a, b, name)
    for i, (a, b) in enumerate(zip(_unpack(pb, lam["mem"], em3d.ADJ_MEM_AXES), olm)):
        _same(a, b, f"adjoint memory {i}")
    assert nat.device_status(cuda_device) == 0


@pytest.mark.parametrize("stencil", [4, 6, 8])
def test_high_order_public_api_fp64_vs_reference_golden(cuda_device, stencil):
    """tide_b200.em3d.maxwell3d at orders 4 to 8 in FP64 against the
    reference's functional API (golden fixture): receivers and gradients."""
    z = np.load(GOLDEN / "em3d_case.npz")
    hi = np.load(GOLDEN / "em3d_hi_case.npz")
    dev = cuda_device
    eps = torch.from_numpy(z["eps"]).to(dev).requires_grad_(True)
    sig = torch.from_numpy(z["sig"]).to(dev).requires_grad_(True)
    mu = torch.from_numpy(z["mu"]).to(dev)
    out = em3d.maxwell3d(eps, sig, mu, float(z["dx"]), float(hi["dt"]),
                         torch.from_numpy(hi["amp"]).to(dev), torch.from_numpy(z["src"]).to(dev),
                         torch.from_numpy(z["rec"]).to(dev), pml_width=int(z["pml"]),
                         stencil=stencil)
    r = out[-1]
    assert rel_l2(r, torch.from_numpy(hi[f"r_python_s{stencil}"])) < 1e-13
    w = torch.randn(r.shape, generator=torch.Generator().manual_seed(5), dtype=r.dtype).to(dev)
    (r * w).sum().backward()
    assert rel_l2(eps.grad, torch.from_numpy(hi[f"geps_s{stencil}"])) < 1e-9
    assert rel_l2(sig.grad, torch.from_numpy(hi[f"gsig_s{stencil}"])) < 1e-9
