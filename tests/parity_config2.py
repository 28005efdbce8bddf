"""Accuracy of the benchmarked configuration against the CPU checkers.

Test infrastructure (the checker, never the product): used by
tests/test_gpu_config2.py and by bench.py's CPU-baseline leg, which reports
the numbers in its JSON line.

* Config 1 (96 x 96, 300 steps): receivers of the B200 library through the
  public API against the reference CPU backend's FP32 and FP64 runs
  (tests/golden/config1.npz, made by running the reference).
* Config-2 sample: the seeded config-2 model and acquisition on the full
  553 x 1065 padded grid (CPML 20), the first `shots` shots, `nt` steps,
  loss 0.5 |r|^2.  The eps / sigma gradients of the public API (FP32,
  snapshots on the device) against the C oracle's exact adjoint chained to
  eps / sigma by torch autograd, in FP32 (the reference's summation order)
  and in FP64 (the error statement), and the BF16-snapshot gradient against
  the FP32-snapshot one.
"""

from __future__ import annotations

import pathlib

import numpy as np
import torch

GOLDEN = pathlib.Path(__file__).resolve().parent / "golden"


def rel_l2(a: torch.Tensor, b: torch.Tensor) -> float:
    a = a.detach().double().cpu()
    b = b.detach().double().cpu()
    den = torch.linalg.vector_norm(b)
    return float(torch.linalg.vector_norm(a - b) / (den if den > 0 else 1.0))


def config1_errors(dev) -> dict:
    """Config-1 receivers (public API, FP32, GPU) against the reference CPU
    backend in FP32 (expected 0: bit-identical) and in FP64."""
    import tide_b200 as tide

    z = np.load(GOLDEN / "config1.npz")
    nt, dt = 300, 4e-11
    eps = torch.full((96, 96), 4.0, device=dev)
    amp = tide.ricker(800e6, nt, dt, device=dev).view(1, 1, nt)
    out = tide.maxwelltm(eps, torch.zeros_like(eps), torch.ones_like(eps), 0.02, dt, amp,
                         torch.tensor([[[20, 48]]], device=dev),
                         torch.tensor([[[20, 60]]], device=dev), stencil=2, pml_width=10)
    r = out[-1].detach().cpu()
    return {
        "rel_l2_vs_reference_cpu_fp32": rel_l2(r, torch.from_numpy(z["r_native_f32"])),
        "rel_l2_vs_reference_cpu_fp64": rel_l2(r, torch.from_numpy(z["r_native_f64"])),
    }


def gpu_gradient(cfg: dict, dev, compression: bool = False):
    """Receivers and eps / sigma gradients of loss 0.5 |r|^2 through the
    public API on `dev` (FP32, snapshots on the device)."""
    import tide_b200 as tide

    d = {k: (v.to(dev) if torch.is_tensor(v) else v) for k, v in cfg.items()}
    eps = d["eps"].detach().requires_grad_(True)
    sig = d["sig"].detach().requires_grad_(True)
    out = tide.maxwelltm(eps, sig, d["mu"], d["dx"], d["dt"], d["amp"], d["src"], d["rec"],
                         stencil=2, pml_width=d["pml"], storage_mode="device",
                         storage_compression=compression)
    r = out[-1]
    (0.5 * (r * r).sum()).backward()
    return r.detach().cpu(), eps.grad.detach().cpu(), sig.grad.detach().cpu()


def oracle_gradient(cfg: dict, dtype, oracle=None):
    """The same with the C oracle's exact adjoint (CPU), in `dtype`, summing
    the per-shot image terms in the reference's order."""
    from oracle_harness import Oracle, OracleTM, set_grad_order
    from tide_b200.tm2d import prepare_tm2d

    oracle = oracle or Oracle()
    set_grad_order(oracle, 0)
    eps = cfg["eps"].cpu().to(dtype).requires_grad_(True)
    sig = cfg["sig"].cpu().to(dtype).requires_grad_(True)
    pb = prepare_tm2d(eps, sig, cfg["mu"].cpu().to(dtype), cfg["dx"], cfg["dt"],
                      cfg["amp"].cpu().to(dtype), cfg["src"].cpu(), cfg["rec"].cpu(),
                      stencil=2, pml_width=cfg["pml"])
    r = OracleTM.apply(pb.ca, pb.cb, pb.f, pb, oracle, 1, 0)
    ge, gs = torch.autograd.grad(0.5 * (r * r).sum(), [eps, sig])
    return r.detach(), ge, gs


def config2_sample_errors(cfg: dict, dev) -> dict:
    """The config-2 sample's gradient errors (see the module docstring)."""
    r, ge, gs = gpu_gradient(cfg, dev)
    _, ge16, gs16 = gpu_gradient(cfg, dev, compression=True)
    r32, oe32, os32 = oracle_gradient(cfg, torch.float32)
    r64, oe64, os64 = oracle_gradient(cfg, torch.float64)
    return {
        "receivers_rel_l2_vs_oracle_fp32": rel_l2(r, r32),
        "grad_eps_rel_l2_vs_oracle_fp32": rel_l2(ge, oe32),
        "grad_sigma_rel_l2_vs_oracle_fp32": rel_l2(gs, os32),
        "receivers_rel_l2_vs_oracle_fp64": rel_l2(r, r64),
        "grad_eps_rel_l2_vs_oracle_fp64": rel_l2(ge, oe64),
        "grad_sigma_rel_l2_vs_oracle_fp64": rel_l2(gs, os64),
        "bf16_snapshots_grad_eps_rel_l2_vs_fp32_snapshots": rel_l2(ge16, ge),
        "bf16_snapshots_grad_sigma_rel_l2_vs_fp32_snapshots": rel_l2(gs16, gs),
        "bf16_snapshots_grad_eps_rel_l2_vs_oracle_fp64": rel_l2(ge16, oe64),
    }
