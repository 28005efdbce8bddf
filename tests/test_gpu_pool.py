"""The device snapshot history is reused across gradient evaluations on
different streams without a race.

A gradient evaluation keeps its snapshot history until its adjoint has run;
released histories are kept for the next request of the same shape
(`tide_b200.storage._HistoryPool`).  Here evaluation A runs on stream 1 and
is released while its adjoint may still be queued; evaluation B on stream 2
then takes the same buffer for its storing forward.  Both gradients must
equal the ones of the same evaluations run alone on the default stream
(bit-identical: same kernels, same inputs).
"""

from __future__ import annotations

import gc

import pytest
import torch

import tide_b200 as tide
from tide_b200 import storage as stg

pytestmark = pytest.mark.gpu


def _inputs(seed, dev, ny=160, nx=240, shots=4, nt=500):
    g = torch.Generator().manual_seed(seed)
    eps = (4.0 + 6.0 * torch.rand((ny, nx), generator=g)).to(dev)
    sig = (0.004 * torch.rand((ny, nx), generator=g)).to(dev)
    mu = torch.ones((ny, nx), device=dev)
    dt = 4e-11
    amp = tide.ricker(600e6, nt, dt).view(1, 1, nt).repeat(shots, 1, 1).to(dev)
    src = torch.tensor([[[12, 20 + 50 * i + seed % 7]] for i in range(shots)], device=dev)
    rec = torch.tensor([[[12, 4 + 8 * j] for j in range(28)]] * shots, device=dev)
    return eps, sig, mu, 0.02, dt, amp, src, rec


def _grad(inp):
    eps, sig, mu, dx, dt, amp, src, rec = inp
    e = eps.detach().clone().requires_grad_(True)
    s = sig.detach().clone().requires_grad_(True)
    out = tide.maxwelltm(e, s, mu, dx, dt, amp, src, rec, stencil=2, pml_width=10,
                         storage_mode="device")
    r = out[-1]
    (0.5 * (r * r).sum()).backward()
    return e.grad, s.grad


def test_history_reuse_across_streams(cuda_device):
    dev = cuda_device
    a_in, b_in = _inputs(1, dev), _inputs(2, dev)
    stg.release_history_pool()
    ga_ref = _grad(a_in)
    gc.collect()
    gb_ref = _grad(b_in)
    torch.cuda.synchronize()
    gc.collect()
    s1, s2 = torch.cuda.Stream(dev), torch.cuda.Stream(dev)
    for _ in range(3):
        with torch.cuda.stream(s1):
            ga = _grad(a_in)
        gc.collect()  # A's history goes back to the pool, its adjoint possibly still queued
        with torch.cuda.stream(s2):
            gb = _grad(b_in)
        torch.cuda.synchronize()
        for got, ref in ((ga, ga_ref), (gb, gb_ref)):
            for x, y in zip(got, ref):
                assert torch.equal(x, y)
        gc.collect()
    stg.release_history_pool()
