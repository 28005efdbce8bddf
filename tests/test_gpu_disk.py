"""Disk storage mode of the TM2D gradient (storage_mode='disk').

The snapshot history goes to one temporary file per snapshot kind through a
3-slot pinned staging ring and a writer thread, and is read back in the
adjoint; gradients, receivers and source gradients must be bit-identical to
the device-history mode (FP32 and BF16 snapshots, sampling intervals 1 and
3, a backward split into several calls, the public API), and the files must
be removed when the history is released.  Tolerance: bit-identical (the FP32
bar, relative L2 <= 1e-5, is asserted alongside).
"""

from __future__ import annotations

import gc
import os

import pytest
import torch

import tide_b200 as tide
from cases import clone_problem, random_problem
from oracle_harness import rel_l2
from tide_b200 import storage as stg
from tide_b200 import tm2d

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _same(a, b, what):
    a, b = a.detach().cpu(), b.detach().cpu()
    assert rel_l2(a, b) <= TOL, what
    assert torch.equal(a, b), f"{what}: not bit-identical"


def _gradients(pb_cpu, dev, grad_r, mode, fmt=0, k=1, opts=None, path="."):
    g = clone_problem(pb_cpu, dev)
    g.grad_interval = k
    S, ny, nx, nt = g.n_shots, g.ny, g.nx, g.nt
    sdt = torch.bfloat16 if fmt else g.dtype
    n_store = (nt + k - 1) // k
    snaps = stg.allocate(mode, sdt, fmt, n_store, S, ny, nx, dev, True, True, path=path)
    files = list(snaps.files.paths) if snaps.files is not None else []
    r = torch.zeros((g.nt, g.n_shots, g.n_rec), device=dev, dtype=g.dtype)
    tm2d._run_forward_storage(g, g.ca, g.cb, g.f, r, snaps, True, True, None, 0)
    if files:
        step = g.n_shots * g.ny * g.nx * sdt.itemsize
        for f in files:
            assert os.path.getsize(f) == n_store * step
    out = tm2d._run_backward(g, g.ca, g.cb, grad_r.to(dev), snaps, True, True, True, opts or {})
    torch.cuda.synchronize()
    return (r, *out), files, snaps


@pytest.mark.parametrize("fmt,k", [(0, 1), (1, 1), (0, 3)])
def test_disk_equals_device(cuda_device, tmp_path, fmt, k):
    pb = random_problem(61 + k, 35, 45, 2, 80)
    grad_r = torch.randn((pb.nt, pb.n_shots, pb.n_rec), generator=torch.Generator().manual_seed(3))
    a, _, _ = _gradients(pb, cuda_device, grad_r, stg.STORAGE_DEVICE, fmt, k)
    b, files, snaps = _gradients(pb, cuda_device, grad_r, stg.STORAGE_DISK, fmt, k,
                                 path=str(tmp_path))
    assert len(files) == 2 and all(os.path.dirname(f) == str(tmp_path) for f in files)
    for x, y, n in zip(a, b, ("r", "gca", "gcb", "gf")):
        _same(x, y, n)
    del snaps
    gc.collect()
    assert not any(os.path.exists(f) for f in files), "snapshot files not removed"


def test_disk_chunked_backward(cuda_device, tmp_path):
    """Backward split into callback chunks reads the same file across calls."""
    pb = random_problem(71, 30, 40, 2, 75)
    grad_r = torch.randn((pb.nt, pb.n_shots, pb.n_rec), generator=torch.Generator().manual_seed(4))
    a, _, _ = _gradients(pb, cuda_device, grad_r, stg.STORAGE_DEVICE)
    seen = []
    b, _, _ = _gradients(pb, cuda_device, grad_r, stg.STORAGE_DISK, path=str(tmp_path),
                         opts={"backward_callback": lambda s: seen.append(s.step),
                               "callback_frequency": 16})
    assert seen == [59, 43, 27, 11, 0]
    for x, y, n in zip(a, b, ("r", "gca", "gcb", "gf")):
        _same(x, y, n)


def test_disk_mode_public_api(cuda_device, tmp_path):
    dev = cuda_device
    g = torch.Generator().manual_seed(8)
    ny, nx, S, nt = 28, 40, 2, 60
    eps = (2.0 + 4.0 * torch.rand((ny, nx), generator=g, dtype=torch.float64)).float().to(dev)
    sig = (0.005 * torch.rand((ny, nx), generator=g, dtype=torch.float64)).float().to(dev)
    mu = torch.ones((ny, nx), device=dev)
    dx = 0.02
    dt = 0.9 * dx / (tide.C0 / float(eps.min().sqrt()) * 2 ** 0.5)
    amp = tide.ricker(500e6, nt, dt, dtype=torch.float32).view(1, 1, nt).repeat(S, 1, 1).to(dev)
    src = torch.tensor([[[10, 12]], [[15, 30]]], device=dev)
    rec = torch.tensor([[[5, 5 + 3 * j] for j in range(10)]] * S, device=dev)
    grads = {}
    for mode in ("device", "disk"):
        e = eps.clone().requires_grad_(True)
        s_ = sig.clone().requires_grad_(True)
        out = tide.maxwelltm(e, s_, mu, dx, dt, amp, src, rec, pml_width=8, storage_mode=mode,
                             storage_path=str(tmp_path), storage_compression=True)
        (out[-1] ** 2).sum().backward()
        grads[mode] = (e.grad, s_.grad)
        del out
    gc.collect()
    _same(grads["disk"][0], grads["device"][0], "grad eps")
    _same(grads["disk"][1], grads["device"][1], "grad sigma")
    assert not list(tmp_path.iterdir()), "snapshot files left behind"
