"""The Debye-medium CPU oracle against the reference (CPU only).

Fixture tests/golden/debye_case.npz (tests/golden/make_golden_debye.py): a
heterogeneous 1-pole Debye medium run through the reference's functional
API.  The oracle's forward must give the reference CPU backend's receivers
bit for bit (FP32 and FP64); its exact adjoint, chained to epsilon, sigma,
delta_epsilon and tau by torch autograd through the same coefficient
formulas, must give the reference's autograd gradients (FP64, relative L2
<= 1e-12: the reference differentiates its Python time loop, the oracle
transposes the step, so only rounding differs).
"""

from __future__ import annotations

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from oracle_harness import OracleDebye, rel_l2
from tide_b200 import debye as dby
from tide_b200 import physics as ph
from tide_b200 import tm2d


def _load(dtype):
    z = np.load(GOLDEN / "debye_case.npz")
    tag = "f32" if dtype == torch.float32 else "f64"
    c = {k: torch.from_numpy(z[f"in_{k}_{tag}"]) for k in ("eps", "sig", "deps", "tau", "mu",
                                                         "amp", "w")}
    c.update(src=torch.from_numpy(z["in_src"]), rec=torch.from_numpy(z["in_rec"]),
             dx=float(z["in_dx"]), dt=float(z["in_dt"]), pml=int(z["in_pml"]))
    return z, c, tag


def _problem(c, grads=False, stencil=2, k=1):
    leaves = {n: (c[n].clone().requires_grad_(True) if grads else c[n])
              for n in ("eps", "sig", "deps", "tau")}
    with torch.set_grad_enabled(grads):
        pb = tm2d.prepare_tm2d(leaves["eps"], leaves["sig"], c["mu"], c["dx"], c["dt"], c["amp"],
                               c["src"], c["rec"], stencil=stencil, pml_width=c["pml"],
                               model_gradient_sampling_interval=k,
                               dispersion=ph.DebyeDispersion(leaves["deps"], leaves["tau"]))
    return pb, leaves


def run_oracle(pb, k=1, fmt=0, need=None, grad_r=None):
    """Oracle forward with storage then the full adjoint; returns r, the
    adjoint state and the snapshots."""
    o = OracleDebye()
    d = pb.debye
    ca, cb, f = pb.ca.detach(), pb.cb.detach(), pb.f.detach()
    a, b, cp = d["a"].detach(), d["b"].detach(), d["cp"].detach()
    need = need or {n: True for n in ("ca", "cb", "cp", "a", "b")}
    sdt = torch.bfloat16 if fmt else pb.dtype
    snaps = dby.Snapshots(-(-pb.nt // k), pb, sdt, True, True, True, True)
    r = torch.zeros((pb.nt, pb.n_shots, pb.n_rec), dtype=pb.dtype)
    o.forward(pb, ca, cb, f, r, a, b, cp, snaps, k=k, fmt=fmt)
    st = dby.AdjointState(pb, need)
    gr = r.clone() if grad_r is None else grad_r
    o.backward(pb, ca, cb, a, b, cp, gr, st, snaps, pb.nt, pb.nt, k=k, fmt=fmt)
    return r, st, snaps


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_forward_receivers_equal_reference_cpu(dtype):
    z, c, tag = _load(dtype)
    pb, _ = _problem(c)
    o = OracleDebye()
    d = pb.debye
    snaps = dby.Snapshots(0, pb, dtype, False, False, False, False)
    r = torch.zeros((pb.nt, pb.n_shots, pb.n_rec), dtype=dtype)
    o.forward(pb, pb.ca, pb.cb, pb.f, r, d["a"], d["b"], d["cp"], snaps)
    ref = torch.from_numpy(z[f"r_native_{tag}"])
    assert rel_l2(r, ref) <= 1e-6
    assert torch.equal(r, ref)


def test_adjoint_gradients_equal_reference_autograd():
    z, c, _ = _load(torch.float64)
    pb, leaves = _problem(c, grads=True)
    d = pb.debye
    w = c["w"]
    _, st, _ = run_oracle(pb, grad_r=w.contiguous())
    g = st.g
    outs = [pb.ca, pb.cb, pb.f, d["a"], d["b"], d["cp"]]
    gouts = [g["ca"].unsqueeze(0), g["cb"].unsqueeze(0), st.grad_f.reshape(-1), g["a"], g["b"],
             g["cp"]]
    ge, gs, gd, gt = torch.autograd.grad(outs, [leaves[n] for n in ("eps", "sig", "deps", "tau")],
                                         gouts)
    for name, mine, key in (("eps", ge, "geps_f64"), ("sigma", gs, "gsig_f64"),
                            ("delta_eps", gd, "gdeps_f64"), ("tau", gt, "gtau_f64")):
        err = rel_l2(mine, torch.from_numpy(z[key]))
        assert err <= 1e-12, f"{name}: rel l2 {err}"


def test_adjoint_sampling_interval_and_bf16_close():
    """k = 2 and BF16 snapshots give the FP32 k = 1 gradient within their
    approximation (relative L2 below 0.2 and 2e-2)."""
    _, c, _ = _load(torch.float32)
    base = run_oracle(_problem(c)[0])[1].g["ca"]
    k2 = run_oracle(_problem(c, k=2)[0], k=2)[1].g["ca"]
    bf = run_oracle(_problem(c)[0], fmt=1)[1].g["ca"]
    assert rel_l2(k2, base) < 0.2
    assert rel_l2(bf, base) < 2e-2
