"""Gradient parity on the benchmarked geometry (config 2).

The seeded config-2 model and acquisition (model 512 x 1024, padded 553 x
1065 with CPML 20, sources and receivers on row 10, Ricker 400 MHz), the
first 2 shots, 250 steps, loss 0.5 |r|^2:

* native level (C-ABI forward_with_storage + backward): receivers and the
  ca / cb gradients bit-identical to the C oracle run in the kernels'
  step-major shot order, and within the FP32 bar (relative L2 <= 1e-5) of
  the oracle in the reference's order;
* public API (coefficients prepared on the GPU, eps / sigma through torch
  autograd): receivers and gradients within 1e-5 of the FP32
  oracle and within 1e-3 of the FP64 oracle (the FP32 error statement);
  BF16 snapshots within 1e-2 of FP32 snapshots, the reference's bound for
  compressed storage (tests/backends/test_storage.py:278-293).
"""

from __future__ import annotations

import pathlib
import sys

import pytest
import torch

from cases import clone_problem
from oracle_harness import rel_l2, set_grad_order
from tide_b200 import storage as stg
from tide_b200 import tm2d

sys.path.insert(0, str(pathlib.Path(__file__).resolve().parent.parent))
import bench  # noqa: E402
import parity_config2 as pc2  # noqa: E402

pytestmark = pytest.mark.gpu
TOL = 1e-5  # FP32 parity bar: relative L2
SHOTS, NT = 2, 250


@pytest.fixture(scope="module")
def cfg():
    return bench.config2(shots=SHOTS, nt=NT)


def test_config2_native_gradients_vs_oracle(oracle, cuda_device, cfg):
    pb = tm2d.prepare_tm2d(cfg["eps"], cfg["sig"], cfg["mu"], cfg["dx"], cfg["dt"], cfg["amp"],
                           cfg["src"], cfg["rec"], stencil=2, pml_width=cfg["pml"])
    assert (pb.ny, pb.nx) == (553, 1065) and pb.n_rec == 256
    S, ny, nx, nt = pb.n_shots, pb.ny, pb.nx, pb.nt
    qb = clone_problem(pb)
    store = (torch.zeros((nt, S, ny, nx)), torch.zeros((nt, S, ny, nx)))
    r_o = torch.zeros((nt, S, pb.n_rec))
    oracle.forward(qb, qb.ca, qb.cb, qb.f, r_o, store=store, need_ca=True, need_cb=True)
    grad_r = r_o.clone()  # d(0.5 |r|^2) / dr

    g = clone_problem(pb, cuda_device)
    snaps = stg.allocate(stg.STORAGE_DEVICE, torch.float32, 0, nt, S, ny, nx, cuda_device, True,
                         True)
    r = torch.zeros((nt, S, pb.n_rec), device=cuda_device)
    tm2d._run_forward_storage(g, g.ca, g.cb, g.f, r, snaps, True, True, None, 0)
    gca, gcb, _ = tm2d._run_backward(g, g.ca, g.cb, grad_r.to(cuda_device), snaps, True, True,
                                     True, {})
    torch.cuda.synchronize()
    assert torch.equal(r.cpu(), r_o)
    assert float(r_o.abs().max()) > 0
    set_grad_order(oracle, 1)
    try:
        oca, ocb, _, _ = oracle.backward(qb, qb.ca, qb.cb, grad_r, store)
    finally:
        set_grad_order(oracle, 0)
    for got, want, name in ((gca[0], oca, "grad_ca"), (gcb[0], ocb, "grad_cb")):
        assert rel_l2(got, want) <= TOL, name
        assert torch.equal(got.cpu(), want), f"{name} not bit-identical"
    rca, rcb, _, _ = oracle.backward(qb, qb.ca, qb.cb, grad_r, store)
    assert rel_l2(gca[0], rca) <= TOL and rel_l2(gcb[0], rcb) <= TOL


def test_config2_public_api_gradients(cuda_device, cfg):
    e = pc2.config2_sample_errors(cfg, cuda_device)
    print("config-2 sample errors:", e)
    assert e["receivers_rel_l2_vs_oracle_fp32"] <= TOL
    assert e["grad_eps_rel_l2_vs_oracle_fp32"] <= TOL
    assert e["grad_sigma_rel_l2_vs_oracle_fp32"] <= TOL
    assert e["receivers_rel_l2_vs_oracle_fp64"] <= 1e-3
    assert e["grad_eps_rel_l2_vs_oracle_fp64"] <= 1e-3
    assert e["grad_sigma_rel_l2_vs_oracle_fp64"] <= 1e-3
    assert e["bf16_snapshots_grad_eps_rel_l2_vs_fp32_snapshots"] <= 1e-2
    assert e["bf16_snapshots_grad_sigma_rel_l2_vs_fp32_snapshots"] <= 1e-2


def test_config1_errors(cuda_device):
    e = pc2.config1_errors(cuda_device)
    assert e["rel_l2_vs_reference_cpu_fp32"] <= TOL
    assert e["rel_l2_vs_reference_cpu_fp64"] < 1e-5
