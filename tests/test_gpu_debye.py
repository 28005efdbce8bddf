"""Debye media on the GPU: forward with storage and exact adjoint against the
Debye CPU oracle (bit for bit), and the public API against the reference.

The CUDA sweeps keep the oracle's operation order without FMA contraction, so
receivers, fields, polarisation, every snapshot, the adjoint state and the
gradients of ca, cb, a, b, cp and of the source amplitudes are bit-identical
to it (FP32 and FP64, stencils 2 and 4, sampling intervals 1 and 3, BF16
snapshots).  The FP32 bar (relative L2 <= 1e-5) is asserted next to every
equality.  End to end, tide_b200.maxwelltm with a DebyeDispersion gives the
reference CPU backend's receivers and the reference's autograd gradients
with respect to epsilon, sigma, delta_epsilon and tau (FP64, <= 1e-12), with
the snapshot history on the device or by checkpoint segments.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from cases import clone_problem
from conftest import GOLDEN
from oracle_harness import rel_l2
from test_debye_oracle import _load, _problem, run_oracle
from tide_b200 import _native as nat
from tide_b200 import debye as dby

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _same(a, b, what):
    a, b = a.detach().cpu(), b.detach().cpu()
    if a.dtype == torch.bfloat16:
        assert torch.equal(a, b), what
        return
    err = rel_l2(a, b)
    assert err <= TOL, f"{what}: rel l2 {err}"
    assert torch.equal(a, b), f"{what}: not bit-identical (rel l2 {err})"


def _gpu_run(pb_cpu, dev, k, fmt, grad_r):
    g = clone_problem(pb_cpu, dev)
    d = g.debye
    sdt = torch.bfloat16 if fmt else g.dtype
    snaps = dby.Snapshots(-(-g.nt // k), g, sdt, True, True, True, True)
    for t in (snaps.ey, snaps.curl, snaps.pol, snaps.esum):
        t.zero_()
    r = torch.zeros((g.nt, g.n_shots, g.n_rec), device=dev, dtype=g.dtype)
    dby.native_forward_storage(g, g.ca, g.cb, g.f, r, d["a"], d["b"], d["cp"], snaps, 0, g.nt,
                               k, fmt)
    st = dby.AdjointState(g, {n: True for n in ("ca", "cb", "cp", "a", "b")})
    dby.native_backward(g, g.ca, g.cb, d["a"], d["b"], d["cp"], grad_r.to(dev), st, snaps, g.nt,
                        g.nt, k, fmt)
    torch.cuda.synchronize()
    return g, r, st, snaps


def _dom_mask(pb, stencil):
    p = stencil // 2
    m = torch.zeros((pb.ny, pb.nx), dtype=torch.bool)
    m[p:pb.ny - p + 1, p:pb.nx - p + 1] = True
    return m


@pytest.mark.parametrize("dtype,fmt", [(torch.float32, 0), (torch.float64, 0),
                                       (torch.float32, 1)])
@pytest.mark.parametrize("stencil,k", [(2, 1), (4, 1), (2, 3)])
def test_storage_and_adjoint_bitwise_vs_oracle(cuda_device, dtype, fmt, stencil, k):
    _, c, _ = _load(dtype)
    pb, _ = _problem(c, stencil=stencil, k=k)
    grad_r = c["w"].contiguous()
    o_pb = clone_problem(pb)
    r_o, st_o, sn_o = run_oracle(o_pb, k=k, fmt=fmt, grad_r=grad_r)
    g, r, st, sn = _gpu_run(pb, cuda_device, k, fmt, grad_r)
    _same(r, r_o, "receivers")
    for name, a, b in zip("Ey Hx Hz mEyx mEyz mHxz mHzx".split(), g.fields, o_pb.fields):
        _same(a, b, name)
    _same(dby.polarization(g), dby.polarization(o_pb), "polarisation")
    dom = _dom_mask(pb, stencil)
    for name, a, b in (("ey", sn.ey, sn_o.ey), ("curl", sn.curl, sn_o.curl),
                       ("esum", sn.esum, sn_o.esum)):
        _same(a.cpu()[..., dom], b[..., dom], f"{name} snapshots")
    _same(sn.pol.cpu()[..., dom], sn_o.pol[..., dom], "pol snapshots")
    for i, (a, b) in enumerate(zip(st.lam, st_o.lam)):
        _same(a, b, f"adjoint field {i}")
    _same(st.lam_pol, st_o.lam_pol, "polarisation adjoint")
    _same(st.grad_f, st_o.grad_f, "source gradient")
    for n in ("ca", "cb", "cp", "a", "b"):
        _same(st.g[n], st_o.g[n], f"grad {n}")
    assert nat.device_status(cuda_device) == 0


@pytest.mark.parametrize("mode", ["device", "checkpoint"])
def test_public_api_fp64_vs_reference(cuda_device, mode):
    import tide_b200 as tide

    z, c, _ = _load(torch.float64)
    dev = cuda_device
    leaves = {n: c[n].to(dev).requires_grad_(True) for n in ("eps", "sig", "deps", "tau")}
    out = tide.maxwelltm(leaves["eps"], leaves["sig"], c["mu"].to(dev), c["dx"], c["dt"],
                         c["amp"].to(dev), c["src"].to(dev), c["rec"].to(dev),
                         pml_width=c["pml"], storage_mode=mode, storage_chunk_steps=17,
                         dispersion=tide.DebyeDispersion(leaves["deps"], leaves["tau"]))
    r = out[-1]
    assert rel_l2(r, torch.from_numpy(z["r_native_f64"])) <= 1e-13
    grads = torch.autograd.grad((r * c["w"].to(dev)).sum(),
                                [leaves[n] for n in ("eps", "sig", "deps", "tau")])
    for name, gv, key in zip(("eps", "sigma", "delta_eps", "tau"), grads,
                             ("geps_f64", "gsig_f64", "gdeps_f64", "gtau_f64")):
        err = rel_l2(gv, torch.from_numpy(z[key]))
        assert err <= 1e-12, f"{name}: rel l2 {err}"


def test_public_api_fp32_receivers_and_checkpoint_equal_device(cuda_device):
    """FP32: receivers equal the reference CPU backend's bit for bit, and the
    checkpointed gradient equals the device-history gradient bit for bit."""
    import tide_b200 as tide

    z, c, _ = _load(torch.float32)
    dev = cuda_device

    def run(mode):
        eps = c["eps"].to(dev).requires_grad_(True)
        sig = c["sig"].to(dev).requires_grad_(True)
        out = tide.maxwelltm(eps, sig, c["mu"].to(dev), c["dx"], c["dt"], c["amp"].to(dev),
                             c["src"].to(dev), c["rec"].to(dev), pml_width=c["pml"],
                             storage_mode=mode, storage_chunk_steps=23,
                             dispersion=tide.DebyeDispersion(c["deps"].to(dev), c["tau"].to(dev)))
        g = torch.autograd.grad((out[-1] * c["w"].to(dev)).sum(), [eps, sig])
        return out[-1].detach(), g

    r_d, g_d = run("device")
    r_c, g_c = run("checkpoint")
    _same(r_d, torch.from_numpy(z["r_native_f32"]), "receivers vs reference CPU")
    _same(r_c, r_d, "checkpoint receivers")
    for a, b, n in zip(g_c, g_d, ("eps", "sigma")):
        _same(a, b, f"checkpoint grad {n}")


def test_plain_forward_matches_reference(cuda_device):
    """The Debye forward without gradients (per-call forward entry point)."""
    import tide_b200 as tide

    z, c, _ = _load(torch.float64)
    dev = cuda_device
    out = tide.maxwelltm(c["eps"].to(dev), c["sig"].to(dev), c["mu"].to(dev), c["dx"], c["dt"],
                         c["amp"].to(dev), c["src"].to(dev), c["rec"].to(dev),
                         pml_width=c["pml"],
                         dispersion=tide.DebyeDispersion(c["deps"].to(dev), c["tau"].to(dev)))
    ref = torch.from_numpy(z["r_native_f64"])
    assert rel_l2(out[-1], ref) <= 1e-13
    assert torch.equal(out[-1].cpu(), ref)
