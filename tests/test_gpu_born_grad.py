"""Gradients through the Born pass on the GPU.

* ``born_forward_with_storage`` advances both states exactly as
  ``born_forward`` (receivers and states bit-identical), stores the same
  background history as ``forward_with_storage`` (bit for bit, FULL and BF16,
  sampling intervals 1 and 2), and its scattered history holds dEy^n and
  dcurl H^n of the scattered state;
* ``born_backward`` returns backward's gradients bit for bit on that
  history (the scattered update is linear in (dca, dcb, df) with the
  background factors of (ca, cb, f));
* through ``borntm``: the adjoint dot-product test <J v, w> = <v, J^T w> in
  (depsilon, dsigma) (FP64, 1e-12), the depsilon gradient against the
  epsilon gradient of ``maxwelltm`` on interior cells (FP64, 1e-10), the
  background-receiver gradient equal to ``maxwelltm``'s bit for bit, and
  cpu / disk storage giving the device mode's gradients bit for bit;
* the second-order term (scattered receivers in the background model):
  ``born_backward_bggrad`` bit-identical to the oracle's joint adjoint
  (gradients in ca, cb, dca, dcb, f0, df; stencils 2, 4, 6; FP32 and FP64;
  sampling intervals 1 and 2), and ``borntm``'s gradients in epsilon, sigma,
  depsilon, dsigma equal the reference Python path's autograd (FP64, 1e-9,
  golden born_bggrad.npz);
* the second-order term in cpu storage mode and checkpoint storage raise.
"""

from __future__ import annotations

import pytest
import torch

import tide_b200 as tide
from cases import clone_problem, random_problem
from oracle_harness import rel_l2
from tide_b200 import born as bn
from tide_b200 import storage as stg
from tide_b200 import tm2d

pytestmark = pytest.mark.gpu


def _perturbation(pb, seed, dev):
    g = torch.Generator().manual_seed(seed)
    shape = (1, pb.ny, pb.nx)
    dca = (1e-3 * torch.randn(shape, generator=g, dtype=torch.float64)).to(pb.dtype)
    dcb = (1e-3 * torch.randn(shape, generator=g, dtype=torch.float64)).to(pb.dtype) * pb.cb
    df = (torch.randn(pb.f.shape, generator=g, dtype=torch.float64).to(pb.dtype) * 0.1
          * pb.f.abs().max())
    return [t.contiguous().to(dev) for t in (dca, dcb, df)]


def _born(q, d, snaps=None, direct=(0, 0)):
    tan = [torch.zeros_like(t) for t in q.fields]
    r = torch.zeros((q.nt, q.n_shots, q.n_rec), device=q.device, dtype=q.dtype)
    bg = torch.zeros_like(r)
    need = (snaps is not None and snaps.ey_dev.numel() > 0,
            snaps is not None and snaps.curl_dev.numel() > 0)
    bn._born_forward_call(q, d[0], d[1], d[2], q.f, tan, r, bg, snaps, need, None, direct)
    torch.cuda.synchronize()
    return r, bg, q.fields, tan


def _history(q, fmt, sdtype, n_store, mode=stg.STORAGE_DEVICE, path="."):
    """A history whose cells outside the update domain (never written) are 0."""
    h = stg.allocate(mode, sdtype, fmt, n_store, q.n_shots, q.ny, q.nx, q.device, True, True,
                     path=path)
    h.ey_dev.zero_()
    h.curl_dev.zero_()
    return h


@pytest.mark.parametrize("stencil,k,bf16", [(2, 1, False), (4, 2, False), (2, 1, True),
                                            (8, 3, True)])
def test_born_storage_forward_matches_born_and_storage_forward(cuda_device, stencil, k, bf16):
    dev = cuda_device
    pb = random_problem(810 + stencil, 33, 47, 3, 41, stencil=stencil, pml=6, k=k)
    d = _perturbation(pb, 5, dev)
    fmt, sdtype = (1, torch.bfloat16) if bf16 else (0, torch.float32)
    n_store = (pb.nt + k - 1) // k
    ref = _born(clone_problem(pb, dev), d)
    q = clone_problem(pb, dev)
    snaps = _history(q, fmt, sdtype, n_store)
    got = _born(q, d, snaps)
    for a, b in zip((ref[0], ref[1], *ref[2], *ref[3]), (got[0], got[1], *got[2], *got[3])):
        assert torch.equal(a, b)
    # the same history as the plain storing forward
    p = clone_problem(pb, dev)
    plain = _history(p, fmt, sdtype, n_store)
    r = torch.zeros((p.nt, p.n_shots, p.n_rec), device=dev, dtype=p.dtype)
    tm2d._storage_call(p, p.ca, p.cb, p.f, r.data_ptr(), tm2d._snap_ptrs(plain), 0, fmt,
                       plain.shot_bytes, True, True, 0, p.nt)
    torch.cuda.synchronize()
    assert torch.equal(r, got[1])
    assert torch.equal(plain.ey_dev, snaps.ey_dev)
    assert torch.equal(plain.curl_dev, snaps.curl_dev)


def test_born_storage_scattered_history(cuda_device):
    """dey_store[q] is the scattered Ey after q*k steps; dcurl_store[q] is the
    curl a plain storing step computes from that scattered state."""
    dev = cuda_device
    k = 2
    pb = random_problem(833, 31, 45, 2, 30, pml=6, k=k)
    d = _perturbation(pb, 7, dev)
    n_store = (pb.nt + k - 1) // k
    q = clone_problem(pb, dev)
    snaps = _history(q, 0, torch.float32, n_store)
    dey_h = torch.zeros((n_store, q.n_shots, q.ny, q.nx), device=dev, dtype=q.dtype)
    dcurl_h = torch.zeros_like(dey_h)
    _born(q, d, snaps, (dey_h.data_ptr(), dcurl_h.data_ptr()))
    for qi in (3, n_store - 1):
        t = qi * k
        p = clone_problem(pb, dev)
        p.nt = t
        p.f = p.f[: t * p.n_shots * p.n_src].contiguous()
        dp = [d[0], d[1], d[2][: t * p.n_shots * p.n_src].contiguous()]
        _, _, _, tan = _born(p, dp)
        assert torch.equal(tan[0], dey_h[qi])
        # one plain storing step from the scattered state gives its curl
        s = clone_problem(pb, dev)
        for a, b in zip(s.fields, tan):
            a.copy_(b)
        one = _history(s, 0, torch.float32, 1)
        r = torch.zeros((1, s.n_shots, s.n_rec), device=dev, dtype=s.dtype)
        s.f = torch.zeros_like(s.f[: s.n_shots * s.n_src])
        tm2d._storage_call(s, s.ca, s.cb, s.f, r.data_ptr(), tm2d._snap_ptrs(one), 0, 0,
                           one.shot_bytes, True, True, 0, 1)
        torch.cuda.synchronize()
        assert torch.equal(one.curl_dev[0], dcurl_h[qi])


@pytest.mark.parametrize("stencil,k", [(2, 1), (4, 2)])
def test_born_backward_equals_backward(cuda_device, stencil, k):
    dev = cuda_device
    pb = random_problem(850 + stencil, 35, 49, 3, 44, stencil=stencil, pml=6, k=k)
    d = _perturbation(pb, 9, dev)
    q = clone_problem(pb, dev)
    snaps = _history(q, 0, torch.float32, (pb.nt + k - 1) // k)
    _born(q, d, snaps)
    g = torch.Generator().manual_seed(4)
    grad_r = torch.randn((pb.nt, pb.n_shots, pb.n_rec), generator=g).to(dev)
    st = tm2d._AdjointState(q, True, True, scratch=False)
    bn._born_backward_call(q, grad_r, st, snaps, True, True)
    ref = tm2d._AdjointState(q, True, True)
    tm2d._backward_call(q, q.ca, q.cb, grad_r, ref, tm2d._snap_ptrs(snaps), 0, 0,
                        snaps.shot_bytes, True, True, pb.nt, pb.nt)
    torch.cuda.synchronize()
    for a, b in zip(st.result(q, True, True, True), ref.result(q, True, True, True)):
        assert torch.equal(a, b)
    assert float(st.grad_ca.abs().max()) > 0 and float(st.grad_cb.abs().max()) > 0


def _case(dev, dtype=torch.float64, seed=3, stencil=2):
    g = torch.Generator().manual_seed(seed)
    ny, nx, S, nt = 30, 44, 2, 70
    eps = (2.0 + 4.0 * torch.rand((ny, nx), generator=g, dtype=torch.float64)).to(dtype).to(dev)
    sig = (0.005 * torch.rand((ny, nx), generator=g, dtype=torch.float64)).to(dtype).to(dev)
    mu = torch.ones((ny, nx), device=dev, dtype=dtype)
    dx = 0.02
    dt = 0.9 * dx / (tide.C0 / float(eps.min().sqrt()) * 2 ** 0.5)
    amp = tide.ricker(500e6, nt, dt, dtype=dtype).view(1, 1, nt).repeat(S, 1, 1).to(dev)
    src = torch.tensor([[[10, 12]], [[15, 30]]], device=dev)
    rec = torch.tensor([[[5, 5 + 3 * j] for j in range(10)]] * S, device=dev)
    deps = (0.3 * torch.randn((ny, nx), generator=g, dtype=torch.float64)).to(dtype).to(dev)
    dsig = (1e-3 * torch.randn((ny, nx), generator=g, dtype=torch.float64)).to(dtype).to(dev)
    w = torch.randn((nt, S, 10), generator=g, dtype=torch.float64).to(dtype).to(dev)
    return dict(eps=eps, sig=sig, mu=mu, dx=dx, dt=dt, amp=amp, src=src, rec=rec, deps=deps,
                dsig=dsig, w=w, stencil=stencil)


def _borntm(c, deps, dsig, eps=None, **kw):
    return tide.borntm(c["eps"] if eps is None else eps, c["sig"], c["mu"], c["dx"], c["dt"],
                       c["amp"], c["src"], c["rec"], c["rec"], depsilon=deps, dsigma=dsig,
                       stencil=c["stencil"], pml_width=8, **kw)


def _born_grads(c, **kw):
    deps = c["deps"].clone().requires_grad_()
    dsig = c["dsig"].clone().requires_grad_()
    r = _borntm(c, deps, dsig, **kw)[-1]
    (r * c["w"]).sum().backward()
    return r.detach(), deps.grad, dsig.grad


def test_borntm_adjoint_dot_product(cuda_device):
    c = _case(cuda_device)
    r, g_eps, g_sig = _born_grads(c)
    lhs = float((r * c["w"]).sum())
    rhs = float((g_eps * c["deps"]).sum() + (g_sig * c["dsig"]).sum())
    assert abs(lhs) > 0
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


@pytest.mark.parametrize("stencil", [2, 4])
def test_borntm_gradient_matches_maxwelltm_gradient(cuda_device, stencil):
    """d<r_born(v), w>/dv = J^T w = d<r(eps), w>/d eps (interior cells: the
    Born perturbation is zero-padded, the model replicate-padded)."""
    c = _case(cuda_device, stencil=stencil)
    _, g_eps, g_sig = _born_grads(c)
    eps = c["eps"].clone().requires_grad_()
    sig = c["sig"].clone().requires_grad_()
    r = tide.maxwelltm(eps, sig, c["mu"], c["dx"], c["dt"], c["amp"], c["src"], c["rec"],
                       stencil=stencil, pml_width=8)[-1]
    (r * c["w"]).sum().backward()
    inner = (slice(1, -1), slice(1, -1))
    assert rel_l2(g_eps[inner], eps.grad[inner]) <= 1e-10
    assert rel_l2(g_sig[inner], sig.grad[inner]) <= 1e-10


def test_borntm_background_receiver_gradient_equals_maxwelltm(cuda_device):
    c = _case(cuda_device)
    eps = c["eps"].clone().requires_grad_()
    bg_r = _borntm(c, c["deps"], c["dsig"], eps=eps)[-2]
    (bg_r * c["w"]).sum().backward()
    eps2 = c["eps"].clone().requires_grad_()
    r = tide.maxwelltm(eps2, c["sig"], c["mu"], c["dx"], c["dt"], c["amp"], c["src"], c["rec"],
                       pml_width=8)[-1]
    assert torch.equal(bg_r.detach(), r.detach())
    (r * c["w"]).sum().backward()
    assert torch.equal(eps.grad, eps2.grad)


@pytest.mark.parametrize("mode", ["cpu", "disk"])
@pytest.mark.parametrize("compression", [False, "bf16"])
def test_borntm_host_and_disk_storage_match_device(cuda_device, tmp_path, mode, compression):
    c = _case(cuda_device, dtype=torch.float32)
    ref = _born_grads(c, storage_compression=compression)
    got = _born_grads(c, storage_mode=mode, storage_path=str(tmp_path),
                      storage_compression=compression)
    for a, b in zip(ref, got):
        assert torch.equal(a, b)
    assert list(tmp_path.iterdir()) == [] or mode == "cpu"


def test_borntm_unbuilt_parts_raise(cuda_device):
    c = _case(cuda_device)
    eps = c["eps"].clone().requires_grad_()
    deps = c["deps"].clone().requires_grad_()
    r = _borntm(c, deps, c["dsig"], eps=eps, storage_mode="cpu")[-1]
    with pytest.raises(NotImplementedError, match="second"):
        (r * c["w"]).sum().backward()
    with pytest.raises(NotImplementedError, match="checkpoint"):
        _borntm(c, deps, c["dsig"], storage_mode="checkpoint")


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("stencil", [2, 4])
def test_jvp_from_kept_history_equals_born_pass(cuda_device, dtype, stencil):
    """MaxwellTM.linearize(...).jvp reads the primal's device history
    (born_tangent_forward_with_storage) instead of recomputing the
    background: bit-identical to the full Born pass."""
    c = _case(cuda_device, dtype=dtype, stencil=stencil)
    op = tide.MaxwellTM(tide.Discretization(c["dx"], c["dt"], stencil=stencil,
                                            boundary=tide.CPML(8)),
                        tide.Experiment(tide.Acquisition(c["src"], c["rec"]), c["amp"]))
    lin = op.linearize(tide.EMModel(c["eps"], c["sig"], c["mu"]))
    v = tide.EMDirection(c["deps"], c["dsig"])
    fast = lin._jvp_from_history(v)
    assert fast is not None
    with torch.no_grad():
        full = _borntm(c, c["deps"], c["dsig"])
    assert torch.equal(fast.receiver_data, full[-1])
    assert torch.equal(lin.jvp(v).receiver_data, full[-1])
    st = fast.final_state
    for a, b in zip((st.Ey, st.Hx, st.Hz, st.m_Ey_x, st.m_Ey_z, st.m_Hx_z, st.m_Hz_x),
                    full[7:14]):
        assert torch.equal(a, b)


def test_tangent_pass_direction_batches(cuda_device):
    """n_shots = directions x background shots: scattered shot s reads
    background shot s % background_n_shots; each direction block equals a
    separate tangent pass."""
    from tide_b200 import _native as nat
    from tide_b200.tm2d import _PROFILE_ORDER

    dev = cuda_device
    pb = random_problem(871, 29, 41, 2, 36, pml=6, dtype=torch.float64)
    q = clone_problem(pb, dev)
    snaps = _history(q, 0, torch.float64, pb.nt)
    d = _perturbation(pb, 11, dev)
    _born(q, d, snaps)
    S, n_dir = pb.n_shots, 3
    g = torch.Generator().manual_seed(12)
    dirs = [(1e-3 * torch.randn((1, pb.ny, pb.nx), generator=g, dtype=torch.float64)).to(dev)
            for _ in range(n_dir)]

    def tangent(dca, dcb, shots, bg_shots, src_i, rec_i, df):
        tan = [torch.zeros((shots, pb.ny, pb.nx), device=dev, dtype=pb.dtype) for _ in range(7)]
        r = torch.zeros((pb.nt, shots, pb.n_rec), device=dev, dtype=pb.dtype)
        batched = dca.shape[0] > 1
        ca = q.ca.expand(shots, -1, -1).contiguous() if batched else q.ca
        cb = q.cb.expand(shots, -1, -1).contiguous() if batched else q.cb
        cq = q.cq.expand(shots, -1, -1).contiguous() if batched else q.cq
        fn = nat.get_backend_function("maxwell_tm", "born_tangent_forward_with_storage", 2,
                                      pb.dtype, dev)
        fn(nat.ptr(ca), nat.ptr(cb), nat.ptr(cq), nat.ptr(dca), nat.ptr(dcb), nat.ptr(df),
           *[nat.ptr(t) for t in tan], nat.ptr(r), nat.ptr(snaps.ey_dev), nat.ptr(snaps.curl_dev),
           0, 0, *[nat.ptr(q.profiles[n]) for n in _PROFILE_ORDER], nat.ptr(src_i),
           nat.ptr(rec_i), q.rdy, q.rdx, q.dt, pb.nt, shots, q.ny, q.nx, q.n_src, q.n_rec, 1, 0,
           bg_shots, batched, batched, batched, 0, q.pml_y0, q.pml_x0, q.pml_y1, q.pml_x1, 0,
           dev.index or 0, torch.cuda.current_stream(dev).cuda_stream)
        nat.check("born_tangent_forward_with_storage")
        torch.cuda.synchronize()
        return r, tan

    df0 = torch.zeros(pb.nt * S * pb.n_src, device=dev, dtype=pb.dtype)
    singles = [tangent(dv, 0.5 * dv, S, S, q.sources_i, q.receivers_i, df0) for dv in dirs]
    dca = torch.cat([dv.expand(S, -1, -1) for dv in dirs]).contiguous()
    src_i = q.sources_i.repeat(n_dir, 1).contiguous()
    rec_i = q.receivers_i.repeat(n_dir, 1).contiguous()
    dfb = torch.zeros(pb.nt * S * n_dir * pb.n_src, device=dev, dtype=pb.dtype)
    rb, tb = tangent(dca, (0.5 * dca).contiguous(), S * n_dir, S, src_i, rec_i, dfb)
    for k, (r1, t1) in enumerate(singles):
        assert torch.equal(rb[:, k * S:(k + 1) * S], r1)
        assert torch.equal(tb[0][k * S:(k + 1) * S], t1[0])
    assert float(rb.abs().max()) > 0


# ------------------------------------------------------------ second order
@pytest.mark.parametrize("stencil", [2, 4, 6])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("k", [1, 2])
def test_born_bggrad_bitwise_vs_oracle(cuda_device, stencil, dtype, k):
    from oracle_harness import Oracle

    dev = cuda_device
    pb = random_problem(900 + stencil + k, 31, 43, 3, 36, stencil=stencil, pml=6, k=k,
                        dtype=dtype)
    d = _perturbation(pb, 19, dev)
    n_store = (pb.nt + k - 1) // k
    q = clone_problem(pb, dev)
    snaps = _history(q, 0, dtype, n_store)
    shape = (n_store, q.n_shots, q.ny, q.nx)
    scat = [torch.zeros(shape, device=dev, dtype=dtype) for _ in range(2)]
    _born(q, d, snaps, direct=tuple(t.data_ptr() for t in scat))
    g = torch.Generator().manual_seed(29)
    grad_r = torch.randn((pb.nt, pb.n_shots, pb.n_rec), generator=g, dtype=torch.float64).to(dtype)
    grad_bg = torch.randn((pb.nt, pb.n_shots, pb.n_rec), generator=g, dtype=torch.float64).to(dtype)
    got = bn._born_bggrad_call(q, tuple(d), grad_r.to(dev), grad_bg.to(dev), snaps, scat)
    torch.cuda.synchronize()
    # oracle: the same Born forward with the four histories, then the joint adjoint
    op = clone_problem(pb)
    tan = [torch.zeros_like(t) for t in op.fields]
    r = torch.zeros((op.nt, op.n_shots, op.n_rec), dtype=dtype)
    bg = torch.zeros_like(r)
    st = [torch.zeros(shape, dtype=dtype) for _ in range(4)]
    dc = [t.cpu() for t in d]
    o = Oracle()
    o.born_forward(op, dc[0], dc[1], op.f, dc[2], tan, r, bg, store=st, k=k)
    for a, b in zip((snaps.ey_dev, snaps.curl_dev, *scat), st):
        assert torch.equal(a.cpu(), b)
    gca, gcb, gdca, gdcb, gf0, gdf, _, _ = o.born_bggrad(op, dc[0], dc[1], grad_r, grad_bg, st, k=k)
    n = pb.nt * pb.n_shots * pb.n_src
    pairs = (("dca", got[0], gdca), ("dcb", got[1], gdcb), ("df", got[2], gdf.reshape(-1)[:n]),
             ("ca", got[3], gca), ("cb", got[4], gcb), ("f0", got[5], gf0.reshape(-1)[:n]))
    for name, a, b in pairs:
        a = a.cpu().reshape(b.shape)
        assert float(b.abs().max()) > 0, name
        assert rel_l2(a, b) <= 1e-5, (name, rel_l2(a, b))
        assert torch.equal(a, b), (name, rel_l2(a, b))


@pytest.mark.parametrize("stencil", [2, 4])
def test_borntm_second_order_gradient_vs_reference_golden(cuda_device, stencil):
    """borntm with the background and the direction all requiring gradients
    (FP64): the gradients of <w, scattered> + <wb, background> receivers in
    epsilon, sigma, depsilon and dsigma against the reference Python path's
    autograd (golden born_bggrad.npz) to 1e-9."""
    import numpy as np

    from cases import hetero_inputs
    from conftest import GOLDEN

    z = np.load(GOLDEN / "born_bggrad.npz")
    dev = cuda_device
    c = hetero_inputs(torch.float64)
    eps = c["eps"].to(dev).requires_grad_(True)
    sig = c["sig"].to(dev).requires_grad_(True)
    deps = torch.from_numpy(z["deps"]).to(dev).requires_grad_(True)
    dsig = torch.from_numpy(z["dsig"]).to(dev).requires_grad_(True)
    rec = c["rec"].to(dev)
    out = tide.borntm(eps, sig, c["mu"].to(dev), c["dx"], c["dt"], c["amp"].to(dev),
                      c["src"].to(dev), rec, rec, depsilon=deps, dsigma=dsig, stencil=stencil,
                      pml_width=c["pml"])
    bg, r = out[-2], out[-1]
    tag = f"s{stencil}"
    assert rel_l2(r.detach().cpu(), torch.from_numpy(z[f"r_{tag}"])) < 1e-13
    w, wb = torch.from_numpy(z[f"w_{tag}"]).to(dev), torch.from_numpy(z[f"wb_{tag}"]).to(dev)
    ((r * w).sum() + (bg * wb).sum()).backward()
    for name, t in (("geps", eps), ("gsig", sig), ("gdeps", deps), ("gdsig", dsig)):
        err = rel_l2(t.grad.cpu(), torch.from_numpy(z[f"{name}_{tag}"]))
        assert err < 1e-9, (name, err)
