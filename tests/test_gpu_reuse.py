"""maxwell_tm_*_background_vjp_reuse: the exact adjoint of n_shots shots
against a snapshot history of background_n_shots shots (shot s images
against snapshot shot s % background_n_shots), as the reference's Born
autograd calls it when the background is shared
(src/tide/maxwell/tm2d_born_autograd.py:886-960).

Check: the reuse call equals the ordinary backward over the history with
its shots repeated to n_shots, bit for bit (the same image terms summed in
the same order), on both stencil-2 paths (TMA one-sweep and per-call
kernels), for one and two background shots, FP32 and BF16 snapshots.
"""

from __future__ import annotations

import pytest
import torch

from cases import clone_problem, random_problem
from oracle_harness import rel_l2
from tide_b200 import _native as nat
from tide_b200 import storage as stg
from tide_b200 import tm2d

pytestmark = pytest.mark.gpu


def _history(pb_cpu, dev, fmt):
    g = clone_problem(pb_cpu, dev)
    sdt = torch.bfloat16 if fmt else torch.float32
    snaps = stg.allocate(stg.STORAGE_DEVICE, sdt, fmt, g.nt, g.n_shots, g.ny, g.nx, dev, True, True)
    snaps.ey_dev.zero_()
    snaps.curl_dev.zero_()
    r = torch.zeros((g.nt, g.n_shots, g.n_rec), device=dev)
    tm2d._run_forward_storage(g, g.ca, g.cb, g.f, r, snaps, True, True, None, 0)
    return snaps


@pytest.mark.parametrize("tma", [2, 0])
@pytest.mark.parametrize("bg,fmt", [(1, 0), (2, 0), (2, 1)])
def test_reuse_equals_backward_on_repeated_history(cuda_device, tma, bg, fmt):
    prev = nat.set_tma_mode(tma)
    try:
        S = 4
        pbg = random_problem(61, 40, 150, bg, 50, pml=6, n_rec=5)
        pb = random_problem(61, 40, 150, S, 50, pml=6, n_rec=5)
        assert torch.equal(pbg.ca, pb.ca) and torch.equal(pbg.cb, pb.cb)
        h_bg = _history(pbg, cuda_device, fmt)
        rep = [s % bg for s in range(S)]
        h_full = _history(pbg, cuda_device, fmt)
        h_full.ey_dev = h_bg.ey_dev[:, rep].contiguous()
        h_full.curl_dev = h_bg.curl_dev[:, rep].contiguous()
        grad_r = torch.randn((pb.nt, S, pb.n_rec), generator=torch.Generator().manual_seed(7))
        g1 = clone_problem(pb, cuda_device)
        a = tm2d._run_backward(g1, g1.ca, g1.cb, grad_r.to(cuda_device), h_bg, True, True, True,
                               {}, bg_shots=bg)
        g2 = clone_problem(pb, cuda_device)
        b = tm2d._run_backward(g2, g2.ca, g2.cb, grad_r.to(cuda_device), h_full, True, True, True,
                               {})
        torch.cuda.synchronize()
    finally:
        nat.set_tma_mode(prev)
    for x, y, name in zip(a, b, ("grad_ca", "grad_cb", "grad_f")):
        assert rel_l2(x, y) <= 1e-5, name
        assert torch.equal(x.cpu(), y.cpu()), f"{name} not bit-identical"
    assert float(a[0].abs().sum()) > 0


def test_reuse_rejects_incompatible_shot_counts(cuda_device):
    pb = random_problem(62, 20, 30, 3, 10, pml=4, n_rec=3)
    g = clone_problem(pb, cuda_device)
    h = _history(random_problem(62, 20, 30, 2, 10, pml=4, n_rec=3), cuda_device, 0)
    grad_r = torch.zeros((pb.nt, 3, pb.n_rec), device=cuda_device)
    with pytest.raises(nat.NativeError, match="multiple of background_n_shots"):
        tm2d._run_backward(g, g.ca, g.cb, grad_r, h, True, True, True, {}, bg_shots=2)
