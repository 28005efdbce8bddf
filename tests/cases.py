"""Seeded problem builders shared by the CPU and GPU tests."""

from __future__ import annotations

import numpy as np
import torch

from conftest import GOLDEN
from tide_b200 import physics as ph
from tide_b200.tm2d import prepare_tm2d


def config1_problem(dtype=torch.float32, device="cpu"):
    """96x96, eps_r=4, dx=0.02, dt=4e-11, nt=300, CPML 10."""
    nt, dt = 300, 4e-11
    eps = torch.full((96, 96), 4.0, dtype=dtype, device=device)
    amp = ph.ricker(800e6, nt, dt, dtype=dtype, device=device).view(1, 1, nt)
    return prepare_tm2d(
        eps, torch.zeros_like(eps), torch.ones_like(eps), 0.02, dt, amp,
        torch.tensor([[[20, 48]]], device=device), torch.tensor([[[20, 60]]], device=device),
        stencil=2, pml_width=10,
    )


def hetero_inputs(dtype=torch.float64):
    z = np.load(GOLDEN / "prep_tm2d.npz")
    d = {k[3:]: torch.from_numpy(z[k]) for k in z.files if k.startswith("in_")}
    out = {
        "eps": d["eps"].to(dtype), "sig": d["sig"].to(dtype), "mu": d["mu"].to(dtype),
        "dx": [float(v) for v in d["dx"]], "dt": float(d["dt"]), "amp": d["amp"].to(dtype),
        "src": d["src"], "rec": d["rec"], "w": d["w"].to(dtype), "nt": int(d["nt"]),
        "pml": int(d["pml"]),
    }
    return out


def hetero_problem(stencil=2, dtype=torch.float32, device="cpu", eps=None, sig=None, k=1):
    c = hetero_inputs(dtype)
    e = c["eps"] if eps is None else eps
    s = c["sig"] if sig is None else sig
    return prepare_tm2d(
        e.to(device), s.to(device), c["mu"].to(device), c["dx"], c["dt"], c["amp"].to(device),
        c["src"].to(device), c["rec"].to(device), stencil=stencil, pml_width=c["pml"],
        model_gradient_sampling_interval=k,
    ), c


def random_problem(seed, ny, nx, shots, nt, *, stencil=2, pml=8, dtype=torch.float32,
                   n_rec=7, batched=False, device="cpu", k=1):
    """Smooth random heterogeneous eps/sigma with sources and receivers per shot."""
    g = torch.Generator().manual_seed(seed)
    shape = (shots, ny, nx) if batched else (ny, nx)
    base = 1.5 + 8.0 * torch.rand(shape, generator=g, dtype=torch.float64)
    kern = torch.ones((1, 1, 5, 5), dtype=torch.float64) / 25
    b4 = base.reshape(-1, 1, ny, nx)
    eps = torch.nn.functional.conv2d(torch.nn.functional.pad(b4, (2, 2, 2, 2), mode="replicate"), kern)
    eps = eps.reshape(shape)
    sig = 0.008 * torch.rand(shape, generator=g, dtype=torch.float64)
    mu = torch.ones(shape, dtype=torch.float64)
    dx = 0.02
    vmax = ph.C0 / float(eps.min().sqrt())
    # 0.9 x the 2-D CFL limit, shrunk by the stencil's coefficient sum so the
    # higher orders stay stable too.
    csum = {2: 1.0, 4: 9 / 8 + 1 / 24, 6: 75 / 64 + 25 / 384 + 3 / 640,
            8: 1225 / 1024 + 245 / 3072 + 49 / 5120 + 5 / 7168}[stencil]
    dt = 0.9 * (dx / (vmax * 2**0.5)) / csum
    amp = ph.ricker(500e6, nt, dt, dtype=torch.float64).view(1, 1, nt).repeat(shots, 1, 1)
    amp = amp * (1 + 0.1 * torch.arange(shots, dtype=torch.float64)).view(shots, 1, 1)
    sy = torch.randint(1, ny - 1, (shots, 1, 1), generator=g)
    sx = torch.randint(1, nx - 1, (shots, 1, 1), generator=g)
    src = torch.cat([sy, sx], dim=-1)
    ry = torch.randint(0, ny, (shots, n_rec, 1), generator=g)
    rx = torch.randint(0, nx, (shots, n_rec, 1), generator=g)
    rec = torch.cat([ry, rx], dim=-1)
    pb = prepare_tm2d(
        eps.to(dtype).to(device), sig.to(dtype).to(device), mu.to(dtype).to(device), dx, dt,
        amp.to(dtype).to(device), src.to(device), rec.to(device), stencil=stencil, pml_width=pml,
        model_gradient_sampling_interval=k,
    )
    return pb


def clone_problem(pb, device=None):
    """Deep copy of a prepared problem (optionally moved to another device)."""
    import copy

    q = copy.copy(pb)
    mv = (lambda t: t.detach().clone()) if device is None else (lambda t: t.detach().to(device).clone())
    q.ca, q.cb, q.cq, q.f = mv(pb.ca), mv(pb.cb), mv(pb.cq), mv(pb.f)
    q.profiles = {k: mv(v) for k, v in pb.profiles.items()}
    q.sources_i, q.receivers_i = mv(pb.sources_i), mv(pb.receivers_i)
    q.fields = [mv(t) for t in pb.fields]
    q.models = {}
    if pb.debye is not None:
        q.debye = {k: (mv(v) if torch.is_tensor(v) else v) for k, v in pb.debye.items()}
    return q
