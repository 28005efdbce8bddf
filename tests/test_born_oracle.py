"""Pinning of the Born (tangent) oracle.

Three pins of the C restatement's Born forward (oracle/tm2d_oracle_impl.h,
tide_oracle_tm_born_forward_*):
* the reference's Python Born path (golden fixture born_case.npz, FP64,
  stencils 2 and 4, with and without source linearization): bit for bit,
  background and scattered receivers and the final scattered Ey;
* the reference's CPU backend (maxwell_tm_{S}_{dtype}_born_forward_cpu,
  compiled from the reference sources into oracle/_ref): background receivers
  bit for bit; the scattered field to rounding (relative L2 <= 1e-5 FP32,
  <= 1e-14 FP64), because that build's -Ofast reassociates the four-term
  scattered update ca dE + cb dcurl + dca E + dcb curl;
* a central finite difference of the oracle forward in (ca, cb, f): O(h^2);
* the adjoint dot product against the oracle's exact adjoint over the stored
  background history (the Born adjoint in the perturbation).
The 3-D Born forward is pinned to the reference CPU backend (stencils 2, 4,
8), and its adjoint in the perturbation (Born forward with background
histories, then the exact background adjoint) to the reference Python path's
autograd gradient in depsilon / dsigma (golden born3d_grad.npz, FP64).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from cases import clone_problem, random_problem
from conftest import GOLDEN
from oracle_harness import REF_SO, Oracle, RefCPU, rel_l2


def _perturbation(pb, seed):
    g = torch.Generator().manual_seed(seed)
    shape = (1, pb.ny, pb.nx)
    dca = (1e-3 * torch.randn(shape, generator=g, dtype=torch.float64)).to(pb.dtype)
    dcb = (1e-3 * torch.randn(shape, generator=g, dtype=torch.float64)).to(pb.dtype) * pb.cb
    df = (torch.randn(pb.f.shape, generator=g, dtype=torch.float64).to(pb.dtype) * 0.1
          * pb.f.abs().max())
    return dca.contiguous(), dcb.contiguous(), df.contiguous()


def _zeros_r(pb):
    return torch.zeros((pb.nt, pb.n_shots, pb.n_rec), dtype=pb.dtype)


def _tangent_state(pb):
    return [torch.zeros_like(t) for t in pb.fields]


def _run(driver, pb, dca, dcb, df):
    q = clone_problem(pb)
    tan = _tangent_state(q)
    r, bg = _zeros_r(q), _zeros_r(q)
    driver.born_forward(q, dca, dcb, q.f, df, tan, r, bg)
    return r, bg, q.fields, tan


@pytest.mark.skipif(not REF_SO.exists(), reason="reference CPU backend not built here")
@pytest.mark.parametrize("stencil", [2, 4])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_born_oracle_equals_reference_cpu(stencil, dtype):
    pb = random_problem(610 + stencil, 33, 41, 2, 70, stencil=stencil, dtype=dtype, pml=6)
    dca, dcb, df = _perturbation(pb, 3)
    got = _run(Oracle(), pb, dca, dcb, df)
    ref = _run(RefCPU(), pb, dca, dcb, df)
    assert torch.equal(got[1], ref[1]), "background receivers"
    for a, b in zip(got[2], ref[2]):
        assert torch.equal(a, b), "background state"
    tol = 1e-5 if dtype == torch.float32 else 1e-14
    assert rel_l2(got[0], ref[0]) <= tol
    for a, b in zip(got[3], ref[3]):
        assert rel_l2(a, b) <= tol
    assert float(got[0].abs().max()) > 0


@pytest.mark.parametrize("stencil", [2, 4])
@pytest.mark.parametrize("lin", [True, False])
def test_born_oracle_equals_reference_python_golden(stencil, lin):
    import numpy as np
    from conftest import GOLDEN
    from cases import hetero_inputs
    from tide_b200.born import prepare_born
    from tide_b200.tm2d import prepare_tm2d

    z = np.load(GOLDEN / "born_case.npz")
    c = hetero_inputs(torch.float64)
    pb = prepare_tm2d(c["eps"], c["sig"], c["mu"], c["dx"], c["dt"], c["amp"], c["src"], c["rec"],
                      stencil=stencil, pml_width=c["pml"])
    dca, dcb, df = prepare_born(pb, 1, c["dx"], c["amp"], depsilon=torch.from_numpy(z["deps"]),
                                dsigma=torch.from_numpy(z["dsig"]), linearize_source=lin)
    r, bg, _, tan = _run(Oracle(), pb, dca, dcb, df)
    tag = f"s{stencil}_{'lin' if lin else 'nolin'}"
    assert torch.equal(bg, torch.from_numpy(z[f"bg_r_{tag}"]))
    assert torch.equal(r, torch.from_numpy(z[f"r_{tag}"])), rel_l2(r, torch.from_numpy(z[f"r_{tag}"]))
    assert torch.equal(pb.crop(tan[0]), torch.from_numpy(z[f"dey_{tag}"]))


def test_born_oracle_matches_central_difference():
    pb = random_problem(77, 30, 38, 2, 80, dtype=torch.float64, pml=5)
    dca, dcb, df = _perturbation(pb, 5)
    r_born, bg, _, _ = _run(Oracle(), pb, dca, dcb, df)
    o = Oracle()

    def receivers(h):
        q = clone_problem(pb)
        r = _zeros_r(q)
        o.forward(q, q.ca + h * dca, q.cb + h * dcb, q.f + h * df, r)
        return r

    h = 1e-4
    fd = (receivers(h) - receivers(-h)) / (2 * h)
    assert rel_l2(r_born, fd) < 1e-6
    assert torch.equal(bg, receivers(0.0))


def test_born_adjoint_is_the_adjoint_over_the_background_history():
    """<J v, w> = <v, J^T w> with J v the oracle Born forward in (dca, dcb, df)
    and J^T w the oracle's exact adjoint over the stored background history
    (Ey^n, curl H^n): the scattered update is linear in (dca, dcb, df) with
    the background factors of (ca, cb, f), so the Born adjoint in the
    perturbation (born_backward) is that adjoint (FP64)."""
    pb = random_problem(91, 28, 36, 2, 50, dtype=torch.float64, pml=5)
    dca, dcb, df = _perturbation(pb, 13)
    r, _, _, _ = _run(Oracle(), pb, dca, dcb, df)
    o = Oracle()
    q = clone_problem(pb)
    shape = (q.nt, q.n_shots, q.ny, q.nx)
    store = (torch.zeros(shape, dtype=q.dtype), torch.zeros(shape, dtype=q.dtype))
    o.forward(q, q.ca, q.cb, q.f, _zeros_r(q), store=store, need_ca=True, need_cb=True)
    w = torch.randn(r.shape, generator=torch.Generator().manual_seed(8), dtype=torch.float64)
    gca, gcb, gf, _ = o.backward(q, q.ca, q.cb, w, store)
    lhs = float((r * w).sum())
    rhs = float((dca[0] * gca).sum() + (dcb[0] * gcb).sum() + (df.reshape(gf.shape) * gf).sum())
    assert abs(lhs) > 0
    assert abs(lhs - rhs) <= 1e-11 * abs(lhs)


# ---------------------------------------------------------------------- 3-D
def _case3d(dtype, comps=("ey", "ey"), seed=5, stencil=2):
    from tide_b200.em3d import prepare_em3d

    g = torch.Generator().manual_seed(seed)
    nz, ny, nx, S, nt = 9, 10, 11, 2, 40
    eps = (1.5 + 6.0 * torch.rand((nz, ny, nx), generator=g, dtype=torch.float64)).to(dtype)
    sig = (0.006 * torch.rand((nz, ny, nx), generator=g, dtype=torch.float64)).to(dtype)
    mu = torch.ones((nz, ny, nx), dtype=dtype)
    dx = 0.02
    dt = 0.9 * dx / (299792458.0 / float(eps.min().double().sqrt()) * 3 ** 0.5)
    dt = dt if stencil == 2 else 0.5 * dt
    t = torch.arange(nt, dtype=torch.float64) * dt
    amp = (torch.sin(2 * 3.14159265 * 6e8 * t) * torch.exp(-((t - 3e-9) / 1e-9) ** 2))
    amp = amp.view(1, 1, nt).repeat(S, 1, 1).to(dtype)
    src = torch.stack([torch.randint(2, n - 2, (S, 1), generator=g) for n in (nz, ny, nx)], -1)
    rec = torch.stack([torch.randint(0, n, (S, 4), generator=g) for n in (nz, ny, nx)], -1)
    return prepare_em3d(eps, sig, mu, dx, dt, amp, src, rec, pml_width=3, stencil=stencil,
                        source_component=comps[0], receiver_component=comps[1])


def _perturbation3d(pb, seed):
    g = torch.Generator().manual_seed(seed)
    shape = (1, pb.nz, pb.ny, pb.nx)
    dca = (1e-3 * torch.randn(shape, generator=g, dtype=torch.float64)).to(pb.dtype)
    dcb = (1e-3 * torch.randn(shape, generator=g, dtype=torch.float64)).to(pb.dtype) * pb.cb
    df = (torch.randn(pb.f.shape, generator=g, dtype=torch.float64).to(pb.dtype) * 0.1
          * pb.f.abs().max())
    return dca.contiguous(), dcb.contiguous(), df.contiguous()


def _run3d(driver, pb, dca, dcb, df):
    from oracle_harness import Oracle3D

    F, M = Oracle3D.full_state(pb)
    DF, DM = [torch.zeros_like(t) for t in F], [torch.zeros_like(t) for t in M]
    r = torch.zeros((pb.nt, pb.n_shots, pb.n_rec), dtype=pb.dtype)
    bg = torch.zeros_like(r)
    driver.born_forward(pb, dca, dcb, pb.f, df, F, M, DF, DM, r, bg)
    return r, bg, F + M, DF + DM


@pytest.mark.skipif(not REF_SO.exists(), reason="reference CPU backend not built here")
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("comps", [("ey", "ey"), ("ex", "ez")])
@pytest.mark.parametrize("stencil", [2, 4, 8])
def test_born3d_oracle_equals_reference_cpu(dtype, comps, stencil):
    """Background bit-identical at order 2; at orders 4 to 8 the reference
    CPU build (-Ofast) may reassociate the multi-term differences, so every
    output is held to rounding there."""
    from oracle_harness import Oracle3D, RefCPU3D

    pb = _case3d(dtype, comps, stencil=stencil)
    dca, dcb, df = _perturbation3d(pb, 7)
    got = _run3d(Oracle3D(), pb, dca, dcb, df)
    ref = _run3d(RefCPU3D(), pb, dca, dcb, df)
    tol = 1e-5 if dtype == torch.float32 else (1e-14 if stencil == 2 else 1e-12)
    if stencil == 2:
        assert torch.equal(got[1], ref[1]), "background receivers"
        for a, b in zip(got[2], ref[2]):
            assert torch.equal(a, b), "background state"
    else:
        assert rel_l2(got[1], ref[1]) <= tol
        for a, b in zip(got[2], ref[2]):
            assert rel_l2(a, b) <= tol
    assert rel_l2(got[0], ref[0]) <= tol
    for a, b in zip(got[3], ref[3]):
        assert rel_l2(a, b) <= tol
    assert float(got[0].abs().max()) > 0


def test_born3d_oracle_matches_central_difference():
    from oracle_harness import Oracle3D

    pb = _case3d(torch.float64)
    dca, dcb, df = _perturbation3d(pb, 9)
    r_born, bg, _, _ = _run3d(Oracle3D(), pb, dca, dcb, df)
    o = Oracle3D()

    def receivers(h):
        F, M = Oracle3D.full_state(pb)
        r = torch.zeros((pb.nt, pb.n_shots, pb.n_rec), dtype=pb.dtype)
        o.forward(pb, pb.ca + h * dca, pb.cb + h * dcb, pb.f + h * df, r, F, M)
        return r

    h = 1e-4
    fd = (receivers(h) - receivers(-h)) / (2 * h)
    assert rel_l2(r_born, fd) < 1e-6
    assert torch.equal(bg, receivers(0.0))


# ------------------------------------------- 3-D Born adjoint (perturbation)
class _OracleBorn3D(torch.autograd.Function):
    """(dca, dcb, df) -> scattered receivers on the oracle: Born forward with
    background E / curl H histories, backward = the exact background adjoint
    imaging against them (the restatement of maxwell_3d_*_born_backward)."""

    @staticmethod
    def forward(ctx, dca, dcb, df, pb):
        from oracle_harness import Oracle3D

        F, M = Oracle3D.full_state(pb)
        DF, DM = [torch.zeros_like(t) for t in F], [torch.zeros_like(t) for t in M]
        r = torch.zeros((pb.nt, pb.n_shots, pb.n_rec), dtype=pb.dtype)
        bg = torch.zeros_like(r)
        st = [torch.zeros((pb.nt, pb.n_shots, pb.nz, pb.ny, pb.nx), dtype=pb.dtype)
              for _ in range(6)] + [None] * 6
        Oracle3D().born_forward(pb, dca.detach(), dcb.detach(), pb.f, df.detach(), F, M, DF,
                                DM, r, bg, store=st)
        ctx.pb, ctx.st = pb, st[:6]
        return r

    @staticmethod
    def backward(ctx, grad_r):
        from oracle_harness import Oracle3D

        pb = ctx.pb
        gca, gcb, gf, _, _ = Oracle3D().backward(pb, pb.ca, pb.cb, grad_r.contiguous(), ctx.st)
        return gca.unsqueeze(0), gcb.unsqueeze(0), gf.reshape(-1), None


def born3d_oracle(eps, sig, mu, dx, dt, amp, src, rec, pml, stencil, deps, dsig):
    """The Born receivers of born3d(depsilon, dsigma) on the oracle, CPU,
    differentiable in deps / dsig (the born3d preparation restated)."""
    from tide_b200.born import linearize_material_coefficients
    from tide_b200 import physics as ph
    from tide_b200.em3d import prepare_em3d

    pb = prepare_em3d(eps, sig, mu, dx, dt, amp, src, rec, pml_width=pml, stencil=stencil)
    pad = [a + b for a, b in zip(pb.fd_pad, pb.pml_width)]
    shape = (pb.nz, pb.ny, pb.nx)
    zp = lambda t: torch.nn.functional.pad(t, ph._torch_pad_order(pad))  # noqa: E731
    dca, dcb = linearize_material_coefficients(pb.ca[0], pb.cb[0], pb.dt, zp(deps), zp(dsig))
    dca, dcb = dca.reshape(1, *shape), dcb.reshape(1, *shape)
    S, N = pb.n_shots, pb.nz * pb.ny * pb.nx
    dcb_at = dcb.reshape(1, N).expand(S, -1).gather(1, pb.sources_i)
    df = (amp.permute(2, 0, 1) * dcb_at[None] * (-1.0 / (dx * dx * dx))).reshape(-1)
    return _OracleBorn3D.apply(dca, dcb, df, pb)


@pytest.mark.parametrize("stencil", [2, 4])
def test_born3d_oracle_adjoint_matches_reference_autograd(stencil):
    """The perturbation gradient of the Born receivers through the oracle's
    Born forward + background adjoint equals the reference Python path's
    autograd gradient (tests/golden/born3d_grad.npz, make_golden_born3d.py),
    FP64, relative L2 < 1e-9; the receivers to 1e-13."""
    z = np.load(GOLDEN / "em3d_case.npz")
    g = np.load(GOLDEN / "born3d_grad.npz")
    eps, sig, mu = (torch.from_numpy(z[n]) for n in ("eps", "sig", "mu"))
    amp = torch.from_numpy(z["amp"] if stencil == 2 else np.load(GOLDEN / "em3d_hi_case.npz")["amp"])
    deps = torch.from_numpy(g["deps"]).requires_grad_(True)
    dsig = torch.from_numpy(g["dsig"]).requires_grad_(True)
    r = born3d_oracle(eps, sig, mu, float(z["dx"]), float(g[f"dt_s{stencil}"]), amp,
                      torch.from_numpy(z["src"]), torch.from_numpy(z["rec"]), int(z["pml"]),
                      stencil, deps, dsig)
    assert rel_l2(r.detach(), torch.from_numpy(g[f"r_s{stencil}"])) < 1e-13
    (r * torch.from_numpy(g[f"w_s{stencil}"])).sum().backward()
    assert rel_l2(deps.grad, torch.from_numpy(g[f"geps_s{stencil}"])) < 1e-9
    assert rel_l2(dsig.grad, torch.from_numpy(g[f"gsig_s{stencil}"])) < 1e-9


# ------------------------------------ second-order Born (background gradient)
class _OracleBornFull(torch.autograd.Function):
    """(dca, dcb, df, ca, cb, f0) -> (background receivers, scattered
    receivers) on the oracle; backward = the joint adjoint of the background
    and scattered recurrences (the restatement of born_backward_bggrad)."""

    @staticmethod
    def forward(ctx, dca, dcb, df, ca, cb, f0, pb):
        q = clone_problem(pb)
        q.ca, q.cb = ca.detach(), cb.detach()
        tan = _tangent_state(q)
        r, bg = _zeros_r(q), _zeros_r(q)
        shape = (q.nt, q.n_shots, q.ny, q.nx)
        st = [torch.zeros(shape, dtype=q.dtype) for _ in range(4)]
        Oracle().born_forward(q, dca.detach(), dcb.detach(), f0.detach(), df.detach(), tan, r, bg,
                              store=st)
        ctx.q, ctx.st = q, st
        ctx.save_for_backward(dca, dcb)
        return bg, r

    @staticmethod
    def backward(ctx, g_bg, g_r):
        dca, dcb = ctx.saved_tensors
        q = ctx.q
        gca, gcb, gdca, gdcb, gf0, gdf, _, _ = Oracle().born_bggrad(
            q, dca.detach(), dcb.detach(), g_r.contiguous(), g_bg.contiguous(), ctx.st)
        n = q.nt * q.n_shots * q.n_src
        return (gdca.unsqueeze(0), gdcb.unsqueeze(0), gdf.reshape(-1)[:n], gca.unsqueeze(0),
                gcb.unsqueeze(0), gf0.reshape(-1)[:n], None)


@pytest.mark.parametrize("stencil", [2, 4])
def test_born_second_order_oracle_matches_reference_autograd(stencil):
    """Gradient of <w, scattered> + <wb, background> receivers in the
    background epsilon / sigma and the direction depsilon / dsigma, through
    the oracle's joint adjoint chained by torch autograd, equals the
    reference Python Born path's autograd (born_bggrad.npz, FP64) to 1e-9."""
    from cases import hetero_inputs
    from tide_b200.born import prepare_born
    from tide_b200.tm2d import prepare_tm2d

    z = np.load(GOLDEN / "born_bggrad.npz")
    c = hetero_inputs(torch.float64)
    eps = c["eps"].clone().requires_grad_(True)
    sig = c["sig"].clone().requires_grad_(True)
    deps = torch.from_numpy(z["deps"]).requires_grad_(True)
    dsig = torch.from_numpy(z["dsig"]).requires_grad_(True)
    pb = prepare_tm2d(eps, sig, c["mu"], c["dx"], c["dt"], c["amp"], c["src"], c["rec"],
                      stencil=stencil, pml_width=c["pml"])
    dca, dcb, df = prepare_born(pb, 1, c["dx"], c["amp"], depsilon=deps, dsigma=dsig)
    bg, r = _OracleBornFull.apply(dca, dcb, df, pb.ca, pb.cb, pb.f, pb)
    tag = f"s{stencil}"
    assert rel_l2(r.detach(), torch.from_numpy(z[f"r_{tag}"])) < 1e-13
    assert rel_l2(bg.detach(), torch.from_numpy(z[f"bg_r_{tag}"])) < 1e-13
    ((r * torch.from_numpy(z[f"w_{tag}"])).sum() + (bg * torch.from_numpy(z[f"wb_{tag}"])).sum()
     ).backward()
    for name, t in (("geps", eps), ("gsig", sig), ("gdeps", deps), ("gdsig", dsig)):
        err = rel_l2(t.grad, torch.from_numpy(z[f"{name}_{tag}"]))
        assert err < 1e-9, (name, err)


class _OracleBorn3DFull(torch.autograd.Function):
    """(dca, dcb, df, ca, cb, f0) -> scattered receivers on the 3-D oracle;
    backward = the 3-D joint adjoint (born_backward_bggrad's algorithm)."""

    @staticmethod
    def forward(ctx, dca, dcb, df, ca, cb, f0, pb):
        import copy

        from oracle_harness import Oracle3D

        q = copy.copy(pb)
        q.ca, q.cb, q.f = ca.detach(), cb.detach(), f0.detach()
        F, M = Oracle3D.full_state(q)
        DF, DM = [torch.zeros_like(t) for t in F], [torch.zeros_like(t) for t in M]
        r = torch.zeros((q.nt, q.n_shots, q.n_rec), dtype=q.dtype)
        bg = torch.zeros_like(r)
        st = [torch.zeros((q.nt, q.n_shots, q.nz, q.ny, q.nx), dtype=q.dtype) for _ in range(12)]
        Oracle3D().born_forward(q, dca.detach(), dcb.detach(), q.f, df.detach(), F, M, DF, DM, r,
                                bg, store=st)
        ctx.q, ctx.st = q, st
        ctx.save_for_backward(dca, dcb)
        return r

    @staticmethod
    def backward(ctx, grad_r):
        from oracle_harness import Oracle3D, _oracle3d_born_bggrad

        dca, dcb = ctx.saved_tensors
        q = ctx.q
        gca, gcb, gdca, gdcb, gf0, gdf = _oracle3d_born_bggrad(
            Oracle3D(), q, dca.detach(), dcb.detach(), grad_r.contiguous(), ctx.st[:6],
            ctx.st[6:])
        n = q.nt * q.n_shots * q.n_src
        return (gdca.unsqueeze(0), gdcb.unsqueeze(0), gdf.reshape(-1)[:n], gca.unsqueeze(0),
                gcb.unsqueeze(0), gf0.reshape(-1)[:n], None)


def test_born3d_second_order_oracle_matches_reference_autograd():
    """The 3-D joint adjoint chained by torch autograd: gradients of
    <w, scattered receivers> in epsilon, sigma, depsilon and dsigma equal
    the reference Python path's autograd (born3d_bggrad.npz, FP64) to 1e-9."""
    from tide_b200 import physics as ph
    from tide_b200.born import linearize_material_coefficients
    from tide_b200.em3d import prepare_em3d

    z = np.load(GOLDEN / "em3d_case.npz")
    g = np.load(GOLDEN / "born3d_grad.npz")
    h = np.load(GOLDEN / "born3d_bggrad.npz")
    eps = torch.from_numpy(z["eps"]).requires_grad_(True)
    sig = torch.from_numpy(z["sig"]).requires_grad_(True)
    deps = torch.from_numpy(g["deps"]).requires_grad_(True)
    dsig = torch.from_numpy(g["dsig"]).requires_grad_(True)
    dx, amp = float(z["dx"]), torch.from_numpy(z["amp"])
    pb = prepare_em3d(eps, sig, torch.from_numpy(z["mu"]), dx, float(z["dt"]), amp,
                      torch.from_numpy(z["src"]), torch.from_numpy(z["rec"]),
                      pml_width=int(z["pml"]))
    pad = [a + b for a, b in zip(pb.fd_pad, pb.pml_width)]
    shape = (pb.nz, pb.ny, pb.nx)
    zp = lambda t: torch.nn.functional.pad(t, ph._torch_pad_order(pad))  # noqa: E731
    dca, dcb = linearize_material_coefficients(pb.ca[0], pb.cb[0], pb.dt, zp(deps), zp(dsig))
    dca, dcb = dca.reshape(1, *shape), dcb.reshape(1, *shape)
    S, N = pb.n_shots, pb.nz * pb.ny * pb.nx
    dcb_at = dcb.reshape(1, N).expand(S, -1).gather(1, pb.sources_i)
    df = (amp.permute(2, 0, 1) * dcb_at[None] * (-1.0 / (dx * dx * dx))).reshape(-1)
    r = _OracleBorn3DFull.apply(dca, dcb, df, pb.ca, pb.cb, pb.f, pb)
    assert rel_l2(r.detach(), torch.from_numpy(h["r_s2"])) < 1e-13
    (r * torch.from_numpy(h["w_s2"])).sum().backward()
    for name, t in (("geps", eps), ("gsig", sig), ("gdeps", deps), ("gdsig", dsig)):
        err = rel_l2(t.grad, torch.from_numpy(h[f"{name}_s2"]))
        assert err < 1e-9, (name, err)
