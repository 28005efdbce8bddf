"""The 3-D CPU oracle, pinned against the reference (no GPU needed).

* Forward: bit-identical receivers, fields and CPML memories to the
  reference's own 3-D CPU backend compiled from its sources (oracle/_ref),
  FP32 and FP64, unbatched and batched models (skipped where that build is
  absent).
* Forward through the public-API preparation: receivers equal the golden
  fixture from the reference's functional API (tests/golden/em3d_case.npz,
  made by make_golden_em3d.py), FP64, relative L2 < 1e-13.
* Gradient: the oracle's exact adjoint chained to epsilon / sigma equals the
  reference Python path's autograd gradient (FP64, relative L2 < 1e-9) and a
  central finite difference of the receiver functional.
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from oracle_harness import REF_SO, Oracle3D, OracleEM3D, RefCPU3D, rel_l2
from tide_b200.em3d import prepare_em3d


def _golden():
    return np.load(GOLDEN / "em3d_case.npz")


def _case(dtype=torch.float64, batched=False, seed=3):
    z = _golden()
    eps = torch.from_numpy(z["eps"]).to(dtype)
    sig = torch.from_numpy(z["sig"]).to(dtype)
    mu = torch.from_numpy(z["mu"]).to(dtype)
    if batched:
        g = torch.Generator().manual_seed(seed)
        eps = torch.stack([eps, eps * (1 + 0.1 * torch.rand(eps.shape, generator=g, dtype=dtype))])
        sig = torch.stack([sig, sig * 0.5])
        mu = torch.stack([mu, mu])
    amp = torch.from_numpy(z["amp"]).to(dtype)
    return dict(eps=eps, sig=sig, mu=mu, dx=float(z["dx"]), dt=float(z["dt"]), amp=amp,
                src=torch.from_numpy(z["src"]), rec=torch.from_numpy(z["rec"]), pml=int(z["pml"]))


def _prep(c, **kw):
    return prepare_em3d(c["eps"], c["sig"], c["mu"], c["dx"], c["dt"], c["amp"], c["src"], c["rec"],
                        pml_width=c["pml"], **kw)


def test_oracle_forward_matches_public_api_golden():
    z = _golden()
    pb = _prep(_case())
    r = torch.zeros((pb.nt, pb.n_shots, pb.n_rec), dtype=pb.dtype)
    fields, mem = Oracle3D.full_state(pb)
    Oracle3D().forward(pb, pb.ca, pb.cb, pb.f, r, fields, mem)
    assert rel_l2(r, torch.from_numpy(z["r_native_f64"])) < 1e-13
    assert rel_l2(r, torch.from_numpy(z["r_python_f64"])) < 1e-13


@pytest.mark.skipif(not REF_SO.exists(), reason="reference CPU backend not built here")
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("batched", [False, True])
@pytest.mark.parametrize("comp", [("ey", "ey"), ("ex", "ez"), ("ez", "ex")])
def test_oracle_forward_bitwise_vs_reference_cpu(dtype, batched, comp):
    c = _case(dtype, batched)
    pb = _prep(c, source_component=comp[0], receiver_component=comp[1])
    r_o = torch.zeros((pb.nt, pb.n_shots, pb.n_rec), dtype=dtype)
    f_o, m_o = Oracle3D.full_state(pb)
    Oracle3D().forward(pb, pb.ca, pb.cb, pb.f, r_o, f_o, m_o)
    r_r = torch.zeros_like(r_o)
    f_r, m_r = Oracle3D.full_state(pb)
    RefCPU3D().forward(pb, pb.ca, pb.cb, pb.f, r_r, f_r, m_r, n_threads=1)
    assert torch.equal(r_o, r_r)
    for a, b in zip(f_o + m_o, f_r + m_r):
        assert torch.equal(a, b)


def _functional(eps, sig, c, w):
    pb = prepare_em3d(eps, sig, c["mu"], c["dx"], c["dt"], c["amp"], c["src"], c["rec"],
                      pml_width=c["pml"])
    r = OracleEM3D.apply(pb.ca, pb.cb, pb.f, pb, Oracle3D())
    return (r * w).sum()


def test_oracle_gradient_matches_reference_autograd():
    z = _golden()
    c = _case()
    eps = c["eps"].clone().requires_grad_(True)
    sig = c["sig"].clone().requires_grad_(True)
    w = torch.randn((int(z["nt"]), 2, 3), generator=torch.Generator().manual_seed(5),
                    dtype=torch.float64)
    _functional(eps, sig, c, w).backward()
    assert rel_l2(eps.grad, torch.from_numpy(z["geps_python_f64"])) < 1e-9
    assert rel_l2(sig.grad, torch.from_numpy(z["gsig_python_f64"])) < 1e-9


def test_oracle_gradient_matches_finite_difference():
    c = _case()
    w = torch.randn((int(_golden()["nt"]), 2, 3), generator=torch.Generator().manual_seed(5),
                    dtype=torch.float64)
    g = torch.Generator().manual_seed(9)
    d_eps = torch.randn(c["eps"].shape, generator=g, dtype=torch.float64)
    eps = c["eps"].clone().requires_grad_(True)
    sig = c["sig"].clone()
    _functional(eps, sig, c, w).backward()
    analytic = float((eps.grad * d_eps).sum())
    h = 1e-4
    with torch.no_grad():
        fp = float(_functional(c["eps"] + h * d_eps, sig, c, w))
        fm = float(_functional(c["eps"] - h * d_eps, sig, c, w))
    fd = (fp - fm) / (2 * h)
    assert abs(analytic - fd) <= 1e-6 * abs(fd), (analytic, fd)


# ------------------------------------------------------- stencil orders 4, 6, 8
def _hi_case(dtype=torch.float64, batched=False):
    c = _case(dtype, batched)
    hi = np.load(GOLDEN / "em3d_hi_case.npz")
    c["dt"], c["amp"] = float(hi["dt"]), torch.from_numpy(hi["amp"]).to(dtype)
    return c, hi


@pytest.mark.parametrize("stencil", [4, 6, 8])
def test_oracle_high_order_forward_matches_public_api_golden(stencil):
    c, hi = _hi_case()
    pb = _prep(c, stencil=stencil)
    r = torch.zeros((pb.nt, pb.n_shots, pb.n_rec), dtype=pb.dtype)
    fields, mem = Oracle3D.full_state(pb)
    Oracle3D().forward(pb, pb.ca, pb.cb, pb.f, r, fields, mem)
    assert rel_l2(r, torch.from_numpy(hi[f"r_python_s{stencil}"])) < 1e-13
    assert rel_l2(r, torch.from_numpy(hi[f"r_native_s{stencil}"])) < 1e-13


@pytest.mark.skipif(not REF_SO.exists(), reason="reference CPU backend not built here")
@pytest.mark.parametrize("stencil", [4, 6, 8])
@pytest.mark.parametrize("dtype,tol", [(torch.float32, 1e-5), (torch.float64, 1e-13)])
@pytest.mark.parametrize("batched", [False, True])
def test_oracle_high_order_forward_vs_reference_cpu(stencil, dtype, tol, batched):
    """The reference CPU backend is built with -Ofast (its CMake flags), which
    lets the compiler reassociate the multi-term differences; the strict
    restatement agrees to rounding, state arrays included."""
    c, _ = _hi_case(dtype, batched)
    pb = _prep(c, stencil=stencil, source_component="ex", receiver_component="ez")
    r_o = torch.zeros((pb.nt, pb.n_shots, pb.n_rec), dtype=dtype)
    f_o, m_o = Oracle3D.full_state(pb)
    Oracle3D().forward(pb, pb.ca, pb.cb, pb.f, r_o, f_o, m_o)
    r_r = torch.zeros_like(r_o)
    f_r, m_r = Oracle3D.full_state(pb)
    RefCPU3D().forward(pb, pb.ca, pb.cb, pb.f, r_r, f_r, m_r, n_threads=1)
    assert rel_l2(r_o, r_r) < tol
    for a, b in zip(f_o, f_r):
        assert rel_l2(a, b) < tol


@pytest.mark.parametrize("stencil", [4, 6, 8])
def test_oracle_high_order_gradient_matches_reference_autograd(stencil):
    c, hi = _hi_case()
    eps = c["eps"].clone().requires_grad_(True)
    sig = c["sig"].clone().requires_grad_(True)
    w = torch.randn((int(_golden()["nt"]), 2, 3), generator=torch.Generator().manual_seed(5),
                    dtype=torch.float64)
    pb = prepare_em3d(eps, sig, c["mu"], c["dx"], c["dt"], c["amp"], c["src"], c["rec"],
                      pml_width=c["pml"], stencil=stencil)
    r = OracleEM3D.apply(pb.ca, pb.cb, pb.f, pb, Oracle3D())
    (r * w).sum().backward()
    assert rel_l2(eps.grad, torch.from_numpy(hi[f"geps_s{stencil}"])) < 1e-9
    assert rel_l2(sig.grad, torch.from_numpy(hi[f"gsig_s{stencil}"])) < 1e-9
