"""Parity of the one-sweep TMA time steps (stencil 2, FP32).

The library runs them on grids of at least 64 tiles; these tests force them
on (tide_b200_set_tma_mode(2)) for small grids so that interior, CPML-strip
and edge tiles, tiles cut by the grid edge, point tiles, and the persistent
schedule are all exercised.  The number of persistent CTAs is capped
(tide_b200_set_tma_ctas) so that tiles are split between neighbouring CTAs
and the coefficient-gradient running sums are handed over: forward fields,
receivers, snapshots and the adjoint's ca / cb / source gradients must be
bit-identical to the CPU oracle (gradient in the kernels' step-major shot
order), with the FP32 bar (relative L2 <= 1e-5) asserted alongside.
"""

from __future__ import annotations

import pytest
import torch

from cases import clone_problem, random_problem
from oracle_harness import rel_l2, set_grad_order
from tide_b200 import _native as nat
from tide_b200 import storage as stg
from tide_b200 import tm2d

pytestmark = pytest.mark.gpu
TOL = 1e-5
FIELDS = ("Ey", "Hx", "Hz", "mEyx", "mEyz", "mHxz", "mHzx")

# (model ny, model nx, CPML width): several tiles with strips; no CPML; a
# single partial tile; odd widths; many tiles; per-side widths.
SHAPES = [(45, 71, 8), (20, 24, 2), (8, 9, 0), (3, 5, 1), (64, 129, 5), (130, 300, 20),
          (33, 260, [3, 11, 0, 6])]


@pytest.fixture(params=[0, 3])
def tma(request, cuda_device):
    prev_m = nat.set_tma_mode(2)
    prev_c = nat.set_tma_ctas(request.param)
    yield request.param
    nat.set_tma_mode(prev_m)
    nat.set_tma_ctas(prev_c)


def _zeros_r(pb, device="cpu"):
    return torch.zeros((pb.nt, pb.n_shots, pb.n_rec), dtype=pb.dtype, device=device)


def _same(a, b, what):
    a, b = a.detach().cpu(), b.detach().cpu()
    err = rel_l2(a, b)
    assert err <= TOL, f"{what}: rel l2 {err}"
    assert torch.equal(a, b), f"{what}: not bit-identical (rel l2 {err})"


@pytest.mark.parametrize("shape", SHAPES)
def test_forward_bitwise(oracle, cuda_device, tma, shape):
    ny, nx, pml = shape
    pb = random_problem(400 + ny, ny, nx, 3, 60, pml=pml, n_rec=9)
    g = clone_problem(pb, cuda_device)
    r_gpu = _zeros_r(g, cuda_device)
    tm2d.native_forward(g, g.ca, g.cb, g.f, r_gpu, 0, g.nt)
    torch.cuda.synchronize()
    r = _zeros_r(pb)
    oracle.forward(pb, pb.ca, pb.cb, pb.f, r)
    _same(r_gpu, r, "receivers")
    for name, a, b in zip(FIELDS, g.fields, pb.fields):
        _same(a, b, name)
    assert nat.device_status(cuda_device) == 0


def _gradients(pb, dev, grad_r, fmt=0, mode=stg.STORAGE_DEVICE):
    g = clone_problem(pb, dev)
    S, ny, nx, nt, k = g.n_shots, g.ny, g.nx, g.nt, g.grad_interval
    sdt = torch.bfloat16 if fmt else torch.float32
    n_store = (nt + k - 1) // k
    snaps = stg.allocate(mode, sdt, fmt, n_store, S, ny, nx, dev, True, True)
    for t in (snaps.ey_dev, snaps.curl_dev, snaps.ey_host, snaps.curl_host):
        if t.numel():
            t.zero_()
    r = _zeros_r(g, dev)
    tm2d._run_forward_storage(g, g.ca, g.cb, g.f, r, snaps, True, True, None, 0)
    gca, gcb, gf = tm2d._run_backward(g, g.ca, g.cb, grad_r.to(dev), snaps, True, True, True, {})
    torch.cuda.synchronize()
    return r, gca, gcb, gf, snaps, g


def _oracle_gradients(oracle, pb, grad_r, fmt=0):
    q = clone_problem(pb)
    S, ny, nx, nt, k = q.n_shots, q.ny, q.nx, q.nt, q.grad_interval
    n_store = (nt + k - 1) // k
    sdt = torch.bfloat16 if fmt else torch.float32
    store = (torch.zeros((n_store, S, ny, nx), dtype=sdt), torch.zeros((n_store, S, ny, nx), dtype=sdt))
    r = _zeros_r(q)
    oracle.forward(q, q.ca, q.cb, q.f, r, store=store, k=k, fmt=fmt, need_ca=True, need_cb=True)
    set_grad_order(oracle, 1)
    try:
        oca, ocb, ogf, _ = oracle.backward(q, q.ca, q.cb, grad_r, store, k=k, fmt=fmt)
    finally:
        set_grad_order(oracle, 0)
    return r, oca, ocb, ogf, store, q


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("fmt,k", [(0, 1), (1, 3)])
def test_gradient_bitwise(oracle, cuda_device, tma, shape, fmt, k):
    ny, nx, pml = shape
    pb = random_problem(500 + nx, ny, nx, 5, 48, pml=pml, n_rec=7, k=k)
    grad_r = torch.randn((pb.nt, pb.n_shots, pb.n_rec), generator=torch.Generator().manual_seed(ny))
    r, gca, gcb, gf, snaps, g = _gradients(pb, cuda_device, grad_r, fmt)
    r_o, oca, ocb, ogf, store, q = _oracle_gradients(oracle, pb, grad_r, fmt)
    _same(r, r_o, "receivers")
    assert torch.equal(snaps.ey_dev.cpu(), store[0]), "Ey snapshots"
    assert torch.equal(snaps.curl_dev.cpu(), store[1]), "curl H snapshots"
    for name, a, b in zip(FIELDS, g.fields, q.fields):
        _same(a, b, f"final {name}")
    _same(gca[0], oca, "grad ca")
    _same(gcb[0], ocb, "grad cb")
    _same(gf.reshape(ogf.shape), ogf, "grad f")
    assert nat.device_status(cuda_device) == 0


@pytest.mark.parametrize("ctas", [1, 2, 5, 7])
def test_gradient_split_tiles(oracle, cuda_device, ctas):
    """Many shots over few CTAs: every CTA range starts and ends inside a
    tile, so the running sums are handed over at every boundary."""
    prev_m, prev_c = nat.set_tma_mode(2), nat.set_tma_ctas(ctas)
    try:
        pb = random_problem(77, 70, 190, 7, 30, pml=6, n_rec=5)
        grad_r = torch.randn((pb.nt, pb.n_shots, pb.n_rec), generator=torch.Generator().manual_seed(3))
        _, gca, gcb, gf, _, _ = _gradients(pb, cuda_device, grad_r)
    finally:
        nat.set_tma_mode(prev_m)
        nat.set_tma_ctas(prev_c)
    _, oca, ocb, ogf, _, _ = _oracle_gradients(oracle, pb, grad_r)
    _same(gca[0], oca, "grad ca")
    _same(gcb[0], ocb, "grad cb")
    _same(gf.reshape(ogf.shape), ogf, "grad f")
    assert nat.device_status(cuda_device) == 0


def test_edge_case_points(oracle, cuda_device, tma):
    """Duplicate, negative and out-of-domain sources and receivers, forward
    and adjoint."""
    pb = random_problem(71, 26, 140, 2, 40, n_rec=6, pml=4)
    N = pb.ny * pb.nx
    si = torch.cat([pb.sources_i, pb.sources_i, torch.tensor([[-1], [pb.nx + 0]])], dim=1)
    pb.sources_i = si.contiguous()
    pb.n_src = 3
    f = torch.randn((pb.nt, pb.n_shots, 3), generator=torch.Generator().manual_seed(9))
    pb.f = f.reshape(-1).contiguous()
    ri = pb.receivers_i.clone()
    ri[0, 1] = ri[0, 0]
    ri[1, 2] = -1
    ri[1, 3] = N - 1
    ri[0, 4] = 0
    pb.receivers_i = ri.contiguous()
    grad_r = torch.randn((pb.nt, pb.n_shots, pb.n_rec), generator=torch.Generator().manual_seed(8))
    r, gca, gcb, gf, _, g = _gradients(pb, cuda_device, grad_r)
    r_o, oca, ocb, ogf, _, q = _oracle_gradients(oracle, pb, grad_r)
    _same(r, r_o, "receivers")
    _same(g.fields[0], q.fields[0], "Ey")
    _same(gca[0], oca, "grad ca")
    _same(gcb[0], ocb, "grad cb")
    _same(gf.reshape(ogf.shape), ogf, "grad f")


def test_cpu_offload_equals_device(cuda_device, tma):
    pb = random_problem(23, 40, 150, 3, 30, pml=5)
    grad_r = torch.randn((pb.nt, pb.n_shots, pb.n_rec), generator=torch.Generator().manual_seed(4))
    a = _gradients(pb, cuda_device, grad_r, mode=stg.STORAGE_DEVICE)
    b = _gradients(pb, cuda_device, grad_r, mode=stg.STORAGE_CPU)
    for x, y, n in zip(a[:4], b[:4], ("r", "gca", "gcb", "gf")):
        _same(x, y, n)


def test_tma_equals_per_call_kernels_config2_slice(cuda_device):
    """Config-2 padded geometry (553 x 1065, CPML 20), 4 shots, 30 steps:
    the TMA path (auto mode: 306 tiles) against the per-call kernels."""
    pb = random_problem(5, 512, 1024, 4, 30, pml=20, n_rec=256)
    grad_r = torch.randn((pb.nt, pb.n_shots, pb.n_rec), generator=torch.Generator().manual_seed(5))
    res = {}
    for mode in (1, 0):
        prev = nat.set_tma_mode(mode)
        try:
            r, gca, gcb, gf, _, g = _gradients(pb, cuda_device, grad_r)
            res[mode] = [r.cpu(), gca.cpu(), gcb.cpu(), gf.cpu()] + [t.cpu() for t in g.fields]
        finally:
            nat.set_tma_mode(prev)
    for a, b, name in zip(res[1], res[0], ("r", "gca", "gcb", "gf") + FIELDS):
        _same(a, b, f"config-2 slice {name}")
