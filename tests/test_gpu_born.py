"""Born (tangent) propagation on the GPU: the CUDA Born forward against the CPU
oracle, the public ``borntm`` against the reference's Born (golden fixture),
and ``MaxwellTM.linearize(...).jvp`` against the vjp (adjoint dot-product
test) and against central differences of ``maxwelltm``.  The public API is
compared with the reference golden to relative L2 <= 1e-13 in FP64.

The CUDA kernels keep the reference's operation order without FMA
contraction, so background and scattered receivers and states are
bit-identical to the oracle (pinned to the reference in test_born_oracle.py);
the FP32 bar (relative L2 <= 1e-5) is asserted next to every equality.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

import tide_b200 as tide
from cases import clone_problem, hetero_inputs, random_problem
from conftest import GOLDEN
from oracle_harness import Oracle, rel_l2
from tide_b200 import _native as nat
from tide_b200.tm2d import _PROFILE_ORDER

pytestmark = pytest.mark.gpu
TOL = 1e-5


def _same(a, b, what):
    a, b = a.detach().cpu(), b.detach().cpu()
    err = rel_l2(a, b)
    assert err <= TOL, f"{what}: rel l2 {err}"
    assert torch.equal(a, b), f"{what}: not bit-identical (rel l2 {err})"


def _perturbation(pb, seed):
    g = torch.Generator().manual_seed(seed)
    shape = (1, pb.ny, pb.nx)
    dca = (1e-3 * torch.randn(shape, generator=g, dtype=torch.float64)).to(pb.dtype)
    dcb = (1e-3 * torch.randn(shape, generator=g, dtype=torch.float64)).to(pb.dtype) * pb.cb
    df = (torch.randn(pb.f.shape, generator=g, dtype=torch.float64).to(pb.dtype) * 0.1
          * pb.f.abs().max())
    return dca.contiguous(), dcb.contiguous(), df.contiguous()


def _cuda_born(pb, dca, dcb, df, dev):
    q = clone_problem(pb, dev)
    tan = [torch.zeros_like(t) for t in q.fields]
    r = torch.zeros((q.nt, q.n_shots, q.n_rec), device=dev, dtype=q.dtype)
    bg = torch.zeros_like(r)
    fn = nat.get_backend_function("maxwell_tm", "born_forward", q.stencil, q.dtype, dev)
    d = [x.to(dev) for x in (dca, dcb, df)]
    fn(nat.ptr(q.ca), nat.ptr(q.cb), nat.ptr(q.cq), nat.ptr(d[0]), nat.ptr(d[1]), nat.ptr(q.f),
       nat.ptr(d[2]), *[nat.ptr(t) for t in q.fields], *[nat.ptr(t) for t in tan], nat.ptr(r),
       nat.ptr(bg), *[nat.ptr(q.profiles[n]) for n in _PROFILE_ORDER], nat.ptr(q.sources_i),
       nat.ptr(q.receivers_i), q.rdy, q.rdx, q.dt, q.nt, q.n_shots, q.ny, q.nx, q.n_src, q.n_rec,
       1, q.batched, q.batched, q.batched, 0, q.pml_y0, q.pml_x0, q.pml_y1, q.pml_x1, 0,
       dev.index or 0, torch.cuda.current_stream(dev).cuda_stream)
    nat.check("born_forward")
    torch.cuda.synchronize()
    return r, bg, q.fields, tan


def _oracle_born(pb, dca, dcb, df):
    q = clone_problem(pb)
    tan = [torch.zeros_like(t) for t in q.fields]
    r = torch.zeros((q.nt, q.n_shots, q.n_rec), dtype=q.dtype)
    bg = torch.zeros_like(r)
    Oracle().born_forward(q, dca, dcb, q.f, df, tan, r, bg)
    return r, bg, q.fields, tan


@pytest.mark.parametrize("stencil", [2, 4, 6, 8])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_born_forward_bitwise_vs_oracle(cuda_device, stencil, dtype):
    pb = random_problem(700 + stencil, 37, 53, 3, 60, stencil=stencil, dtype=dtype, pml=7)
    dca, dcb, df = _perturbation(pb, stencil)
    got = _cuda_born(pb, dca, dcb, df, cuda_device)
    ref = _oracle_born(pb, dca, dcb, df)
    _same(got[0], ref[0], "scattered receivers")
    _same(got[1], ref[1], "background receivers")
    for i, (a, b) in enumerate(zip(got[2] + got[3], ref[2] + ref[3])):
        _same(a, b, f"state tensor {i}")
    assert nat.device_status(cuda_device) == 0


def test_born_edge_case_points(cuda_device):
    """Duplicate, negative and out-of-domain sources and receivers."""
    pb = random_problem(71, 26, 34, 2, 40, n_rec=6)
    N = pb.ny * pb.nx
    pb.sources_i = torch.cat([pb.sources_i, pb.sources_i, torch.tensor([[-1], [pb.nx]])],
                             dim=1).contiguous()
    pb.n_src = 3
    f = torch.randn((pb.nt, pb.n_shots, 3), generator=torch.Generator().manual_seed(9))
    pb.f = f.reshape(-1).contiguous()
    ri = pb.receivers_i.clone()
    ri[0, 1] = ri[0, 0]
    ri[1, 2] = -1
    ri[1, 3] = N - 1
    pb.receivers_i = ri.contiguous()
    dca, dcb, df = _perturbation(pb, 4)
    got = _cuda_born(pb, dca, dcb, df, cuda_device)
    ref = _oracle_born(pb, dca, dcb, df)
    _same(got[0], ref[0], "scattered receivers")
    _same(got[1], ref[1], "background receivers")


@pytest.mark.parametrize("stencil", [2, 4])
@pytest.mark.parametrize("lin", [True, False])
def test_borntm_public_api_vs_reference_golden(cuda_device, stencil, lin):
    z = np.load(GOLDEN / "born_case.npz")
    c = hetero_inputs(torch.float64)
    dev = cuda_device
    out = tide.borntm(
        c["eps"].to(dev), c["sig"].to(dev), c["mu"].to(dev), c["dx"], c["dt"], c["amp"].to(dev),
        c["src"].to(dev), c["rec"].to(dev), c["rec"].to(dev),
        depsilon=torch.from_numpy(z["deps"]).to(dev), dsigma=torch.from_numpy(z["dsig"]).to(dev),
        stencil=stencil, pml_width=c["pml"], linearize_source=lin,
    )
    tag = f"s{stencil}_{'lin' if lin else 'nolin'}"
    assert len(out) == 16
    # the host preparation (padding, dca/dcb, source values) runs as torch ops
    # on the GPU, whose scalar arithmetic may round differently from the
    # reference's CPU torch: FP64 agreement to 1e-13 (the kernels themselves
    # are bit-identical to the oracle, test_born_forward_bitwise_vs_oracle)
    for got, key in ((out[-1], f"r_{tag}"), (out[-2], f"bg_r_{tag}"), (out[7], f"dey_{tag}")):
        ref = torch.from_numpy(z[key])
        assert rel_l2(got, ref) <= 1e-13, key


def _operator(dev, dtype=torch.float64, seed=3, stencil=2):
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
    op = tide.MaxwellTM(tide.Discretization(dx, dt, stencil=stencil, boundary=tide.CPML(8)),
                        tide.Experiment(tide.Acquisition(src, rec), amp))
    # The Born perturbation is zero-padded into the CPML region (as the
    # reference's), the forward model replicate-padded: directions that vanish
    # on the outer model cells make the two maps' derivatives agree exactly.
    mask = torch.zeros((ny, nx), dtype=torch.float64)
    mask[2:-2, 2:-2] = 1.0
    d_eps = 0.3 * mask * torch.randn((ny, nx), generator=g, dtype=torch.float64)
    d_sig = 1e-3 * mask * torch.randn((ny, nx), generator=g, dtype=torch.float64)
    return (op, tide.EMModel(eps, sig, mu),
            tide.EMDirection(d_eps.to(dtype).to(dev), d_sig.to(dtype).to(dev)))


def test_jvp_adjoint_dot_product(cuda_device):
    """<J v, w> = <v, J^T w>: the Born jvp against the exact adjoint vjp (FP64)."""
    op, model, v = _operator(cuda_device)
    lin = op.linearize(model)
    jv = lin.jvp(v)
    w = torch.randn(jv.receiver_data.shape, generator=torch.Generator().manual_seed(2),
                    dtype=torch.float64).to(cuda_device)
    g = lin.vjp(w)
    lhs = float((jv.receiver_data * w).sum())
    rhs = float((g.epsilon * v.epsilon).sum() + (g.sigma * v.sigma).sum())
    assert abs(lhs - rhs) <= 1e-10 * max(abs(lhs), abs(rhs))
    assert abs(lhs) > 0
    # linear in the direction
    jv2 = lin.jvp(tide.EMDirection(2 * v.epsilon, 2 * v.sigma))
    assert rel_l2(jv2.receiver_data, 2 * jv.receiver_data) <= 1e-12


def test_jvp_matches_central_difference(cuda_device):
    op, model, v = _operator(cuda_device, stencil=4)
    lin = op.linearize(model)
    jv = lin.jvp(v).receiver_data
    h = 1e-4

    def data(s):
        m = tide.EMModel(model.epsilon + s * v.epsilon, model.sigma + s * v.sigma, model.mu)
        return op(m).receiver_data

    fd = (data(h) - data(-h)) / (2 * h)
    assert rel_l2(jv, fd) < 1e-6


def test_jvp_fp32_equals_fp64_within_tolerance(cuda_device):
    op64, m64, v64 = _operator(cuda_device, torch.float64)
    op32, m32, v32 = _operator(cuda_device, torch.float32)
    j64 = op64.linearize(m64).jvp(v64).receiver_data
    j32 = op32.linearize(m32).jvp(v32).receiver_data
    assert rel_l2(j32, j64) < 1e-4


def test_unbuilt_linearization_parts_raise(cuda_device):
    op, model, v = _operator(cuda_device)
    lin = op.linearize(model)
    with pytest.raises(NotImplementedError):
        lin.jvp(tide.EMDirection(mu=torch.ones_like(model.mu)))
    with pytest.raises(NotImplementedError):
        lin.second_vjp(tide.EMDirection(mu=torch.ones_like(model.mu)),
                       torch.zeros_like(lin.primal.receiver_data))


def test_second_vjp_matches_central_difference_of_jvp(cuda_device):
    """<second_vjp(v, w), u> = d/ds <w, J(m + s u) v> at s = 0: the
    second-order Born adjoint against a central difference of the Born jvp
    (FP64)."""
    op, model, v = _operator(cuda_device, stencil=2)
    lin = op.linearize(model)
    w = torch.randn(lin.primal.receiver_data.shape, generator=torch.Generator().manual_seed(4),
                    dtype=torch.float64).to(cuda_device)
    g = lin.second_vjp(v, w)
    gu = torch.Generator().manual_seed(6)
    u_eps = 0.2 * torch.randn(model.epsilon.shape, generator=gu, dtype=torch.float64)
    u_sig = 1e-3 * torch.randn(model.sigma.shape, generator=gu, dtype=torch.float64)
    u_eps, u_sig = u_eps.to(cuda_device), u_sig.to(cuda_device)
    analytic = float((g.epsilon * u_eps).sum() + (g.sigma * u_sig).sum())
    h = 1e-4

    def jw(s):
        m = tide.EMModel(model.epsilon + s * u_eps, model.sigma + s * u_sig, model.mu)
        return float((op.linearize(m).jvp(v).receiver_data * w).sum())

    fd = (jw(h) - jw(-h)) / (2 * h)
    assert abs(fd) > 0
    assert abs(analytic - fd) <= 1e-6 * abs(fd), (analytic, fd)


# ---------------------------------------------------------------------- 3-D
def _born3d_cuda(pb, dca, dcb, df, dev):
    import copy

    from tide_b200 import em3d

    q = copy.copy(pb)
    mv = lambda t: t.detach().to(dev).clone()  # noqa: E731
    q.ca, q.cb, q.cq, q.f = mv(pb.ca), mv(pb.cb), mv(pb.cq), mv(pb.f)
    q.profiles = {k: mv(v) for k, v in pb.profiles.items()}
    q.sources_i, q.receivers_i = mv(pb.sources_i), mv(pb.receivers_i)
    q.fields = [mv(t) for t in pb.fields]
    # full-layout CPML memories on the Born entry point
    q.memories = [mv(pb.layout.unpack(t, a)) for t, a in zip(pb.memories, em3d.MEM_AXES)]
    q.device = torch.device(dev)
    dfields = [torch.zeros_like(t) for t in q.fields]
    dmem = [torch.zeros_like(t) for t in q.memories]
    r = torch.zeros((q.nt, q.n_shots, q.n_rec), device=dev, dtype=q.dtype)
    bg = torch.zeros_like(r)
    d = [x.to(dev) for x in (dca, dcb, df)]
    fn = nat.get_backend_function("maxwell_3d", "born_forward", q.stencil, q.dtype, dev)
    p = nat.ptr
    fn(p(q.ca), p(q.cb), p(q.cq), p(d[0]), p(d[1]), p(q.f), p(d[2]),
       *[p(t) for t in q.fields], *[p(t) for t in q.memories], *[p(t) for t in dfields],
       *[p(t) for t in dmem], p(r), p(bg), *em3d._profile_ptrs(q), p(q.sources_i),
       p(q.receivers_i), q.rdz, q.rdy, q.rdx, q.dt, q.nt, q.n_shots, q.nz, q.ny, q.nx, q.n_src,
       q.n_rec, 1, q.batched, q.batched, q.batched, 0, *q.pml, q.src_comp, q.rec_comp, 0,
       dev.index or 0, 0, torch.cuda.current_stream(dev).cuda_stream)
    nat.check("born_forward 3-D")
    torch.cuda.synchronize()
    full = lambda mems: [m.cpu() for m in mems]  # noqa: E731
    return r, bg, q.fields + full(q.memories), dfields + full(dmem)


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("comps", [("ey", "ey"), ("ex", "ez")])
@pytest.mark.parametrize("stencil", [2, 4, 6, 8])
def test_born3d_forward_bitwise_vs_oracle(cuda_device, dtype, comps, stencil):
    from oracle_harness import Oracle3D
    from test_born_oracle import _case3d, _perturbation3d

    pb = _case3d(dtype, comps, stencil=stencil)
    dca, dcb, df = _perturbation3d(pb, 7)
    got = _born3d_cuda(pb, dca, dcb, df, cuda_device)
    F, M = Oracle3D.full_state(pb)
    DF, DM = [torch.zeros_like(t) for t in F], [torch.zeros_like(t) for t in M]
    r = torch.zeros((pb.nt, pb.n_shots, pb.n_rec), dtype=pb.dtype)
    bg = torch.zeros_like(r)
    Oracle3D().born_forward(pb, dca, dcb, pb.f, df, F, M, DF, DM, r, bg)
    _same(got[0], r, "scattered receivers")
    _same(got[1], bg, "background receivers")
    for i, (a, b) in enumerate(zip(got[2] + got[3], F + M + DF + DM)):
        _same(a, b, f"state tensor {i}")
    assert nat.device_status(cuda_device) == 0


def _operator3d(dev, dtype=torch.float64, seed=5):
    g = torch.Generator().manual_seed(seed)
    nz, ny, nx, S, nt = 10, 12, 11, 2, 50
    eps = (1.5 + 5.0 * torch.rand((nz, ny, nx), generator=g, dtype=torch.float64)).to(dtype).to(dev)
    sig = (0.004 * torch.rand((nz, ny, nx), generator=g, dtype=torch.float64)).to(dtype).to(dev)
    mu = torch.ones((nz, ny, nx), device=dev, dtype=dtype)
    dx = 0.02
    dt = 0.9 * dx / (tide.C0 / float(eps.min().sqrt()) * 3 ** 0.5)
    amp = tide.ricker(600e6, nt, dt, dtype=dtype).view(1, 1, nt).repeat(S, 1, 1).to(dev)
    src = torch.tensor([[[4, 5, 5]], [[6, 7, 4]]], device=dev)
    rec = torch.tensor([[[1, 2 + j, 3] for j in range(6)]] * S, device=dev)
    op = tide.Maxwell3D(tide.Discretization(dx, dt, boundary=tide.CPML(3)),
                        tide.Experiment(tide.Acquisition(src, rec), amp, source_component="ez",
                                        receiver_component="ez"))
    mask = torch.zeros((nz, ny, nx), dtype=torch.float64)
    mask[2:-2, 2:-2, 2:-2] = 1.0
    d_eps = 0.3 * mask * torch.randn((nz, ny, nx), generator=g, dtype=torch.float64)
    d_sig = 1e-3 * mask * torch.randn((nz, ny, nx), generator=g, dtype=torch.float64)
    return (op, tide.EMModel(eps, sig, mu),
            tide.EMDirection(d_eps.to(dtype).to(dev), d_sig.to(dtype).to(dev)))


def test_maxwell3d_jvp_adjoint_dot_product(cuda_device):
    op, model, v = _operator3d(cuda_device)
    lin = op.linearize(model)
    jv = lin.jvp(v)
    assert len(jv.final_state.tensors()) == 18
    w = torch.randn(jv.receiver_data.shape, generator=torch.Generator().manual_seed(2),
                    dtype=torch.float64).to(cuda_device)
    g = lin.vjp(w)
    lhs = float((jv.receiver_data * w).sum())
    rhs = float((g.epsilon * v.epsilon).sum() + (g.sigma * v.sigma).sum())
    assert abs(lhs - rhs) <= 1e-10 * max(abs(lhs), abs(rhs))
    assert abs(lhs) > 0


def test_maxwell3d_jvp_matches_central_difference(cuda_device):
    op, model, v = _operator3d(cuda_device)
    jv = op.linearize(model).jvp(v).receiver_data
    h = 1e-4

    def data(s):
        m = tide.EMModel(model.epsilon + s * v.epsilon, model.sigma + s * v.sigma, model.mu)
        return op(m).receiver_data

    fd = (data(h) - data(-h)) / (2 * h)
    assert rel_l2(jv, fd) < 1e-6


# ------------------------------------------------- 3-D Born storage / backward
def _born3d_store_cuda(pb, dca, dcb, df, dev, k, fmt, scattered=True):
    """maxwell_3d_*_born_forward_with_storage in device mode: background E /
    curl H and (optionally) scattered E / curl snapshots, full memories."""
    import copy

    from tide_b200 import em3d

    q = copy.copy(pb)
    mv = lambda t: t.detach().to(dev).clone()  # noqa: E731
    q.ca, q.cb, q.cq, q.f = mv(pb.ca), mv(pb.cb), mv(pb.cq), mv(pb.f)
    q.profiles = {kk: mv(v) for kk, v in pb.profiles.items()}
    q.sources_i, q.receivers_i = mv(pb.sources_i), mv(pb.receivers_i)
    q.fields = [mv(t) for t in pb.fields]
    q.memories = [mv(pb.layout.unpack(t, a)) for t, a in zip(pb.memories, em3d.MEM_AXES)]
    dfields = [torch.zeros_like(t) for t in q.fields]
    dmem = [torch.zeros_like(t) for t in q.memories]
    n_store = (pb.nt + k - 1) // k
    sdt = torch.bfloat16 if fmt else q.dtype
    shape = (n_store, q.n_shots, q.nz, q.ny, q.nx)
    st = [torch.zeros(shape, device=dev, dtype=sdt) for _ in range(12 if scattered else 6)]
    r = torch.zeros((q.nt, q.n_shots, q.n_rec), device=dev, dtype=q.dtype)
    bg = torch.zeros_like(r)
    d = [x.to(dev) for x in (dca, dcb, df)]
    fn = nat.get_backend_function("maxwell_3d", "born_forward_with_storage", q.stencil, q.dtype,
                                  dev)
    p = nat.ptr
    s18 = []
    for c in range(6):
        s18 += [p(st[c]), 0, 0]
    s6 = [p(st[6 + c]) for c in range(6)] if scattered else [0] * 6
    shot_bytes = q.nz * q.ny * q.nx * (2 if fmt else q.ca.element_size())
    stream = torch.cuda.current_stream(dev).cuda_stream
    fn(p(q.ca), p(q.cb), p(q.cq), p(d[0]), p(d[1]), p(q.f), p(d[2]),
       *[p(t) for t in q.fields], *[p(t) for t in q.memories], *[p(t) for t in dfields],
       *[p(t) for t in dmem], p(r), p(bg), *s18, *s6, *em3d._profile_ptrs(q), p(q.sources_i),
       p(q.receivers_i), q.rdz, q.rdy, q.rdx, q.dt, q.nt, q.n_shots, q.nz, q.ny, q.nx, q.n_src,
       q.n_rec, k, 0, fmt, shot_bytes, True, True, q.batched, q.batched, q.batched, 0, *q.pml,
       q.src_comp, q.rec_comp, 0, dev.index or 0, 0, stream, stream)
    nat.check("born_forward_with_storage 3-D")
    torch.cuda.synchronize()
    return q, r, bg, st, shot_bytes


@pytest.mark.parametrize("stencil", [2, 4])
@pytest.mark.parametrize("dtype,fmt", [(torch.float32, 0), (torch.float32, 1), (torch.float64, 0)])
@pytest.mark.parametrize("k", [1, 2])
def test_born3d_storage_bitwise_vs_oracle(cuda_device, stencil, dtype, fmt, k):
    from oracle_harness import Oracle3D
    from test_born_oracle import _case3d, _perturbation3d

    pb = _case3d(dtype, ("ex", "ez"), stencil=stencil)
    dca, dcb, df = _perturbation3d(pb, 7)
    _, r, bg, st, _ = _born3d_store_cuda(pb, dca, dcb, df, cuda_device, k, fmt)
    F, M = Oracle3D.full_state(pb)
    DF, DM = [torch.zeros_like(t) for t in F], [torch.zeros_like(t) for t in M]
    r_o = torch.zeros((pb.nt, pb.n_shots, pb.n_rec), dtype=pb.dtype)
    bg_o = torch.zeros_like(r_o)
    st_o = [torch.zeros(t.shape, dtype=t.dtype) for t in st]
    Oracle3D().born_forward(pb, dca, dcb, pb.f, df, F, M, DF, DM, r_o, bg_o, store=st_o, k=k,
                            fmt=fmt)
    _same(r, r_o, "scattered receivers")
    _same(bg, bg_o, "background receivers")
    for c in range(12):
        assert torch.equal(st[c].cpu(), st_o[c]), f"snapshot kind {c}"
    assert float(st_o[9].float().abs().max()) > 0
    assert nat.device_status(cuda_device) == 0


@pytest.mark.parametrize("stencil", [2, 6])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("k", [1, 3])
def test_born3d_backward_bitwise_vs_oracle(cuda_device, stencil, dtype, k):
    """maxwell_3d_*_born_backward: the background adjoint imaging against
    the background snapshots of born_forward_with_storage (full memories)
    equals the oracle's exact adjoint with the oracle's background
    snapshots: grad dca, grad dcb, grad f and the adjoint state."""
    from oracle_harness import Oracle3D
    from test_born_oracle import _case3d, _perturbation3d

    from tide_b200 import em3d

    pb = _case3d(dtype, ("ey", "ex"), stencil=stencil)
    dca, dcb, df = _perturbation3d(pb, 11)
    q, r, _, st, shot_bytes = _born3d_store_cuda(pb, dca, dcb, df, cuda_device, k, 0,
                                                 scattered=False)
    dev = cuda_device
    S, shape = q.n_shots, (q.n_shots, q.nz, q.ny, q.nx)
    grad_r = torch.randn((pb.nt, S, pb.n_rec), generator=torch.Generator().manual_seed(4),
                         dtype=dtype)
    lam = [torch.zeros(shape, device=dev, dtype=dtype) for _ in range(6)]
    lmem = [torch.zeros(shape, device=dev, dtype=dtype) for _ in range(12)]
    scratch = torch.empty((12, *shape), device=dev, dtype=dtype)
    mshape = (q.nz, q.ny, q.nx)
    gca = torch.full(mshape, 7.0, device=dev, dtype=dtype)  # zeroed on entry
    gcb = torch.full(mshape, 7.0, device=dev, dtype=dtype)
    gca_s = torch.empty(shape, device=dev, dtype=dtype)
    gcb_s = torch.empty(shape, device=dev, dtype=dtype)
    gf = torch.full((pb.nt * S * q.n_src,), 7.0, device=dev, dtype=dtype)
    fn = nat.get_backend_function("maxwell_3d", "born_backward", q.stencil, dtype, dev)
    p = nat.ptr
    s18 = []
    for c in range(6):
        s18 += [p(st[c]), 0, 0]
    stream = torch.cuda.current_stream(dev).cuda_stream
    fn(p(q.ca), p(q.cb), p(q.cq), p(grad_r.to(dev)), *[p(t) for t in lam],
       *[p(t) for t in lmem], p(scratch), *s18, p(gf), p(gca), p(gcb), p(gca_s), p(gcb_s),
       *em3d._profile_ptrs(q), p(q.sources_i), p(q.receivers_i), q.rdz, q.rdy, q.rdx, q.dt,
       q.nt, S, q.nz, q.ny, q.nx, q.n_src, q.n_rec, k, 0, 0, shot_bytes, True, True, q.batched,
       q.batched, q.batched, q.nt, *q.pml, q.src_comp, q.rec_comp, 0, dev.index or 0, 0, stream,
       stream)
    nat.check("born_backward 3-D")
    torch.cuda.synchronize()
    # oracle: background snapshots from the oracle's own forward, then the adjoint
    n_store = (pb.nt + k - 1) // k
    st_o = [torch.zeros((n_store, S, pb.nz, pb.ny, pb.nx), dtype=dtype) for _ in range(6)]
    r_o = torch.zeros((pb.nt, S, pb.n_rec), dtype=dtype)
    f_o, m_o = Oracle3D.full_state(pb)
    o = Oracle3D()
    o.forward(pb, pb.ca, pb.cb, pb.f, r_o, f_o, m_o, store=st_o, k=k)
    for c in range(6):
        assert torch.equal(st[c].cpu(), st_o[c]), f"background snapshot kind {c}"
    oca, ocb, ogf, ol, olm = o.backward(pb, pb.ca, pb.cb, grad_r, st_o, k=k)
    _same(gca.reshape(oca.shape), oca, "grad dca")
    _same(gcb.reshape(ocb.shape), ocb, "grad dcb")
    _same(gf.reshape(ogf.shape), ogf, "grad f")
    for name, a, b in zip("lEx lEy lEz lHx lHy lHz".split(), lam, ol):
        _same(a, b, name)
    for i, (a, b) in enumerate(zip(lmem, olm)):
        _same(a, b, f"adjoint memory {i}")
    assert float(oca.abs().max()) > 0
    assert nat.device_status(dev) == 0


@pytest.mark.parametrize("stencil", [2, 4])
def test_born3d_public_api_gradient_vs_reference_golden(cuda_device, stencil):
    """tide_b200.em3d.born3d in FP64 with depsilon / dsigma requiring grad:
    scattered receivers and the perturbation gradient of a seeded functional
    against the reference Python path's autograd (born3d_grad.npz)."""
    from tide_b200 import em3d

    z = np.load(GOLDEN / "em3d_case.npz")
    g = np.load(GOLDEN / "born3d_grad.npz")
    dev = cuda_device
    amp = z["amp"] if stencil == 2 else np.load(GOLDEN / "em3d_hi_case.npz")["amp"]
    deps = torch.from_numpy(g["deps"]).to(dev).requires_grad_(True)
    dsig = torch.from_numpy(g["dsig"]).to(dev).requires_grad_(True)
    out = em3d.born3d(torch.from_numpy(z["eps"]).to(dev), torch.from_numpy(z["sig"]).to(dev),
                      torch.from_numpy(z["mu"]).to(dev), float(z["dx"]), float(g[f"dt_s{stencil}"]),
                      torch.from_numpy(amp).to(dev), torch.from_numpy(z["src"]).to(dev),
                      torch.from_numpy(z["rec"]).to(dev), depsilon=deps, dsigma=dsig,
                      stencil=stencil, pml_width=int(z["pml"]))
    r = out[-1]
    assert rel_l2(r.detach().cpu(), torch.from_numpy(g[f"r_s{stencil}"])) < 1e-13
    (r * torch.from_numpy(g[f"w_s{stencil}"]).to(dev)).sum().backward()
    assert rel_l2(deps.grad.cpu(), torch.from_numpy(g[f"geps_s{stencil}"])) < 1e-9
    assert rel_l2(dsig.grad.cpu(), torch.from_numpy(g[f"gsig_s{stencil}"])) < 1e-9
    assert nat.device_status(dev) == 0


@pytest.mark.parametrize("stencil", [2, 4])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("k", [1, 2])
def test_born3d_bggrad_bitwise_vs_oracle(cuda_device, stencil, dtype, k):
    """maxwell_3d_*_born_backward_bggrad over born_forward_with_storage's
    background and scattered histories equals the oracle's 3-D joint adjoint:
    gradients in ca, cb, dca, dcb and both sources, and the adjoint state."""
    from oracle_harness import Oracle3D, _oracle3d_born_bggrad
    from test_born_oracle import _case3d, _perturbation3d

    from tide_b200 import em3d

    dev = cuda_device
    pb = _case3d(dtype, ("ez", "ey"), stencil=stencil)
    pb.grad_interval = k
    dca, dcb, df = _perturbation3d(pb, 23)
    q, r, _, st, shot_bytes = _born3d_store_cuda(pb, dca, dcb, df, dev, k, 0)
    S, shape = q.n_shots, (q.n_shots, q.nz, q.ny, q.nx)
    grad_r = torch.randn((pb.nt, S, pb.n_rec), generator=torch.Generator().manual_seed(7),
                         dtype=dtype)
    z = lambda: torch.zeros(shape, device=dev, dtype=dtype)  # noqa: E731
    lam, lmem, eta, emem = [z() for _ in range(6)], [z() for _ in range(12)], \
        [z() for _ in range(6)], [z() for _ in range(12)]
    scratch = torch.empty((24, *shape), device=dev, dtype=dtype)
    work = [z() for _ in range(3)]
    mshape = (q.nz, q.ny, q.nx)
    g = [torch.zeros(mshape, device=dev, dtype=dtype) for _ in range(4)]
    gs = [torch.empty(shape, device=dev, dtype=dtype) for _ in range(4)]
    gf0 = torch.zeros(pb.nt * S * q.n_src, device=dev, dtype=dtype)
    gdf = torch.zeros_like(gf0)
    fn = nat.get_backend_function("maxwell_3d", "born_backward_bggrad", q.stencil, dtype, dev)
    p = nat.ptr
    s18 = []
    for c in range(6):
        s18 += [p(st[c]), 0, 0]
    stream = torch.cuda.current_stream(dev).cuda_stream
    d = [t.to(dev) for t in (dca, dcb, df)]
    fn(p(q.ca), p(q.cb), p(q.cq), p(d[0]), p(d[1]), p(q.f), p(d[2]), p(grad_r.to(dev)),
       *[p(t) for t in lam], *[p(t) for t in lmem], *[p(t) for t in eta], *[p(t) for t in emem],
       p(scratch), *s18, *[p(st[6 + c]) for c in range(6)], p(gf0), p(gdf), *[p(t) for t in g],
       *[p(t) for t in gs], *[p(t) for t in work], *em3d._profile_ptrs(q), p(q.sources_i),
       p(q.receivers_i), q.rdz, q.rdy, q.rdx, q.dt, q.nt, S, q.nz, q.ny, q.nx, q.n_src, q.n_rec,
       k, 0, 0, shot_bytes, True, True, True, True, q.batched, q.batched, q.batched, q.nt,
       *q.pml, q.src_comp, q.rec_comp, 0, dev.index or 0, 0, stream, stream)
    nat.check("born_backward_bggrad 3-D")
    torch.cuda.synchronize()
    # oracle: Born forward with the 12 histories, then the joint adjoint
    F, M = Oracle3D.full_state(pb)
    DF, DM = [torch.zeros_like(t) for t in F], [torch.zeros_like(t) for t in M]
    r_o = torch.zeros((pb.nt, S, pb.n_rec), dtype=dtype)
    bg_o = torch.zeros_like(r_o)
    st_o = [torch.zeros(t.shape, dtype=t.dtype) for t in st]
    o = Oracle3D()
    o.born_forward(pb, dca, dcb, pb.f, df, F, M, DF, DM, r_o, bg_o, store=st_o, k=k)
    for c in range(12):
        assert torch.equal(st[c].cpu(), st_o[c]), f"history {c}"
    gca, gcb, gdca, gdcb, of0, odf = _oracle3d_born_bggrad(o, pb, dca, dcb, grad_r, st_o[:6],
                                                           st_o[6:], k=k)
    n = pb.nt * S * pb.n_src
    for name, a, b in (("ca", g[0], gca), ("cb", g[1], gcb), ("dca", g[2], gdca),
                       ("dcb", g[3], gdcb), ("f0", gf0, of0.reshape(-1)[:n]),
                       ("df", gdf, odf.reshape(-1)[:n])):
        assert float(b.abs().max()) > 0, name
        _same(a.reshape(b.shape), b, f"grad {name}")
    assert nat.device_status(dev) == 0


def test_born3d_second_order_gradient_vs_reference_golden(cuda_device):
    """born3d with the background and the direction all requiring gradients
    (FP64, stencil 2): the gradients of <w, scattered receivers> in epsilon,
    sigma, depsilon and dsigma against the reference Python path's autograd
    (born3d_bggrad.npz) to 1e-9."""
    from tide_b200 import em3d

    z = np.load(GOLDEN / "em3d_case.npz")
    g = np.load(GOLDEN / "born3d_grad.npz")
    h = np.load(GOLDEN / "born3d_bggrad.npz")
    dev = cuda_device
    eps = torch.from_numpy(z["eps"]).to(dev).requires_grad_(True)
    sig = torch.from_numpy(z["sig"]).to(dev).requires_grad_(True)
    deps = torch.from_numpy(g["deps"]).to(dev).requires_grad_(True)
    dsig = torch.from_numpy(g["dsig"]).to(dev).requires_grad_(True)
    out = em3d.born3d(eps, sig, torch.from_numpy(z["mu"]).to(dev), float(z["dx"]), float(z["dt"]),
                      torch.from_numpy(z["amp"]).to(dev), torch.from_numpy(z["src"]).to(dev),
                      torch.from_numpy(z["rec"]).to(dev), depsilon=deps, dsigma=dsig,
                      stencil=2, pml_width=int(z["pml"]))
    r = out[-1]
    assert rel_l2(r.detach().cpu(), torch.from_numpy(h["r_s2"])) < 1e-13
    (r * torch.from_numpy(h["w_s2"]).to(dev)).sum().backward()
    for name, t in (("geps", eps), ("gsig", sig), ("gdeps", deps), ("gdsig", dsig)):
        err = rel_l2(t.grad.cpu(), torch.from_numpy(h[f"{name}_s2"]))
        assert err < 1e-9, (name, err)
    assert nat.device_status(dev) == 0


def test_maxwell3d_second_vjp_matches_central_difference_of_jvp(cuda_device):
    """3-D: <second_vjp(v, w), u> = d/ds <w, J(m + s u) v> at s = 0 (FP64)."""
    op, model, v = _operator3d(cuda_device)
    lin = op.linearize(model)
    w = torch.randn(lin.primal.receiver_data.shape, generator=torch.Generator().manual_seed(8),
                    dtype=torch.float64).to(cuda_device)
    g = lin.second_vjp(v, w)
    gu = torch.Generator().manual_seed(10)
    u_eps = (0.2 * torch.randn(model.epsilon.shape, generator=gu, dtype=torch.float64)).to(cuda_device)
    u_sig = (1e-3 * torch.randn(model.sigma.shape, generator=gu, dtype=torch.float64)).to(cuda_device)
    analytic = float((g.epsilon * u_eps).sum() + (g.sigma * u_sig).sum())
    h = 1e-4

    def jw(s):
        m = tide.EMModel(model.epsilon + s * u_eps, model.sigma + s * u_sig, model.mu)
        return float((op.linearize(m).jvp(v).receiver_data * w).sum())

    fd = (jw(h) - jw(-h)) / (2 * h)
    assert abs(fd) > 0
    assert abs(analytic - fd) <= 1e-6 * abs(fd), (analytic, fd)
