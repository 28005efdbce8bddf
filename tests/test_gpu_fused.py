"""Parity of the fused stencil-2 FP32 forward (one launch per step).

The library picks the fused kernel only for calls whose fields exceed about
half of L2 (tide_b200_set_fused_threshold); these tests force it on small
grids so every part of its decomposition -- interior and band rows of the
column band, side columns with CPML strips and edges, padding lanes, point
tiles -- is checked bit for bit against the CPU oracle, over grid shapes
that give empty, partial and full parts.  Tolerance: bit-identical (the FP32
bar, relative L2 <= 1e-5, is asserted alongside).
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


@pytest.fixture(params=["fused", "two_kernel"])
def mode(request, cuda_device):
    prev = nat.set_fused_threshold(0 if request.param == "fused" else -1)
    yield request.param
    nat.set_fused_threshold(prev)


@pytest.fixture
def fused(cuda_device):
    prev = nat.set_fused_threshold(0)
    yield
    nat.set_fused_threshold(prev)


def _zeros_r(pb, device="cpu"):
    return torch.zeros((pb.nt, pb.n_shots, pb.n_rec), dtype=pb.dtype, device=device)


def _same(a, b, what):
    a, b = a.detach().cpu(), b.detach().cpu()
    err = rel_l2(a, b)
    assert err <= TOL, f"{what}: rel l2 {err}"
    assert torch.equal(a, b), f"{what}: not bit-identical (rel l2 {err})"


FIELDS = ("Ey", "Hx", "Hz", "mEyx", "mEyz", "mHxz", "mHzx")

# (model ny, model nx, CPML width): interior + band + side; no CPML; grids too
# small for an interior (side part only); wide grids with several column warps.
SHAPES = [(45, 71, 8), (20, 24, 2), (8, 9, 0), (3, 5, 1), (64, 129, 5), (130, 300, 20),
          (33, 260, [3, 11, 0, 6])]


@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("batched", [False, True])
def test_forward_bitwise(oracle, cuda_device, mode, shape, batched):
    ny, nx, pml = shape
    pb = random_problem(300 + ny, ny, nx, 3, 60, pml=pml, batched=batched, n_rec=9)
    g = clone_problem(pb, cuda_device)
    r_gpu = _zeros_r(g, cuda_device)
    tm2d.native_forward(g, g.ca, g.cb, g.f, r_gpu, 0, g.nt)
    torch.cuda.synchronize()
    r = _zeros_r(pb)
    oracle.forward(pb, pb.ca, pb.cb, pb.f, r)
    _same(r_gpu, r, f"{mode} receivers")
    for name, a, b in zip(FIELDS, g.fields, pb.fields):
        _same(a, b, f"{mode} {name}")
    assert nat.device_status(cuda_device) == 0


@pytest.mark.parametrize("fmt", [0, 1])
@pytest.mark.parametrize("k", [1, 3])
def test_storage_snapshots_bitwise(oracle, cuda_device, fused, fmt, k):
    pb = random_problem(17 + k, 37, 150, 2, 45, pml=6, k=k)
    S, ny, nx, nt = pb.n_shots, pb.ny, pb.nx, pb.nt
    n_store = (nt + k - 1) // k
    sdt = torch.bfloat16 if fmt else torch.float32
    st_o = (torch.zeros((n_store, S, ny, nx), dtype=sdt), torch.zeros((n_store, S, ny, nx), dtype=sdt))
    q = clone_problem(pb)
    r_o = _zeros_r(q)
    oracle.forward(q, q.ca, q.cb, q.f, r_o, store=st_o, k=k, fmt=fmt, need_ca=True, need_cb=True)
    g = clone_problem(pb, cuda_device)
    snaps = stg.allocate(stg.STORAGE_DEVICE, sdt, fmt, n_store, S, ny, nx, cuda_device, True, True)
    snaps.ey_dev.zero_()
    snaps.curl_dev.zero_()
    r = _zeros_r(g, cuda_device)
    tm2d._run_forward_storage(g, g.ca, g.cb, g.f, r, snaps, True, True, None, 0)
    torch.cuda.synchronize()
    _same(r, r_o, "receivers with storage")
    assert torch.equal(snaps.ey_dev.cpu(), st_o[0]), "Ey snapshots"
    assert torch.equal(snaps.curl_dev.cpu(), st_o[1]), "curl H snapshots"
    for name, a, b in zip(FIELDS, g.fields, q.fields):
        _same(a, b, f"final {name}")


def test_cpu_offload_equals_device(cuda_device, fused):
    pb = random_problem(23, 40, 90, 2, 30, pml=5)
    out = {}
    for mode in (stg.STORAGE_DEVICE, stg.STORAGE_CPU):
        g = clone_problem(pb, cuda_device)
        snaps = stg.allocate(mode, torch.float32, 0, g.nt, g.n_shots, g.ny, g.nx, cuda_device,
                             True, True)
        for t in (snaps.ey_dev, snaps.ey_host, snaps.curl_dev, snaps.curl_host):
            t.zero_()  # cells outside the update domain are never written
        r = _zeros_r(g, cuda_device)
        tm2d._run_forward_storage(g, g.ca, g.cb, g.f, r, snaps, True, True, None, 0)
        torch.cuda.synchronize()
        ey = snaps.ey_dev if mode == stg.STORAGE_DEVICE else snaps.ey_host
        out[mode] = (r.cpu(), ey.cpu().reshape(-1))
    assert torch.equal(out[stg.STORAGE_DEVICE][0], out[stg.STORAGE_CPU][0])
    assert torch.equal(out[stg.STORAGE_DEVICE][1], out[stg.STORAGE_CPU][1])


def test_edge_case_points(oracle, cuda_device, fused):
    """Duplicate, negative and out-of-domain sources and receivers."""
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
    g = clone_problem(pb, cuda_device)
    r_gpu = _zeros_r(g, cuda_device)
    tm2d.native_forward(g, g.ca, g.cb, g.f, r_gpu, 0, g.nt)
    torch.cuda.synchronize()
    r = _zeros_r(pb)
    oracle.forward(pb, pb.ca, pb.cb, pb.f, r)
    _same(r_gpu, r, "receivers with edge-case points")
    _same(g.fields[0], pb.fields[0], "Ey with edge-case points")


def test_gradient_after_fused_forward(oracle, cuda_device, fused):
    pb = random_problem(123, 40, 140, 2, 50, pml=6)
    g = clone_problem(pb, cuda_device)
    S, ny, nx, nt = g.n_shots, g.ny, g.nx, g.nt
    snaps = stg.allocate(stg.STORAGE_DEVICE, torch.float32, 0, nt, S, ny, nx, cuda_device, True,
                         True)
    r = _zeros_r(g, cuda_device)
    tm2d._run_forward_storage(g, g.ca, g.cb, g.f, r, snaps, True, True, None, 0)
    grad_r = torch.randn((nt, S, g.n_rec), generator=torch.Generator().manual_seed(0))
    gca, gcb, gf = tm2d._run_backward(g, g.ca, g.cb, grad_r.to(cuda_device), snaps, True, True,
                                      True, {})
    torch.cuda.synchronize()
    q = clone_problem(pb)
    store = (torch.zeros((nt, S, ny, nx)), torch.zeros((nt, S, ny, nx)))
    r_o = _zeros_r(q)
    oracle.forward(q, q.ca, q.cb, q.f, r_o, store=store, need_ca=True, need_cb=True)
    set_grad_order(oracle, 1)
    try:
        oca, ocb, ogf, _ = oracle.backward(q, q.ca, q.cb, grad_r, store)
    finally:
        set_grad_order(oracle, 0)
    _same(r, r_o, "receivers")
    _same(gca[0], oca, "grad ca")
    _same(gcb[0], ocb, "grad cb")
    _same(gf.reshape(ogf.shape), ogf, "grad f")


def test_fused_equals_two_kernel_config2_slice(cuda_device):
    """Config-2 padded geometry (553 x 1065, CPML 20), 4 shots, 30 steps."""
    pb = random_problem(5, 512, 1024, 4, 30, pml=20, n_rec=256)
    res = {}
    for thr in (0, -1):
        prev = nat.set_fused_threshold(thr)
        try:
            g = clone_problem(pb, cuda_device)
            r = _zeros_r(g, cuda_device)
            tm2d.native_forward(g, g.ca, g.cb, g.f, r, 0, g.nt)
            torch.cuda.synchronize()
            res[thr] = [r.cpu()] + [t.cpu() for t in g.fields]
        finally:
            nat.set_fused_threshold(prev)
    for a, b, name in zip(res[0], res[-1], ("receivers",) + FIELDS):
        _same(a, b, f"config-2 slice {name}")
