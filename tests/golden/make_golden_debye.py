"""Generate the Debye golden fixture (debye_case.npz) from the reference.

Run where the reference tree is mounted at $TIDE_REFERENCE (default: a directory
`reference` beside the repository) and after `make -C oracle ref` built oracle/_ref/:

    python tests/golden/make_golden_debye.py

A small heterogeneous 1-pole Debye medium (2 shots, nt = 120, stencil 2, CPML
6; delta_epsilon and tau vary in space; sources and receivers away from the
padded border).  The reference runs its public functional API:

  r_native_{f32,f64}   receivers of the native CPU backend (Debye forward);
  r_python_{f32,f64}   receivers of the Python reference;
  g{eps,sig,deps,tau}_f64  exact gradients (Python reference, torch autograd,
                       FP64) of sum(w * receivers) with respect to epsilon,
                       sigma, delta_epsilon and tau;
  a, b, cp (f64)       the padded Debye update coefficients the reference
                       compiles (utils.compile_material_coefficients).
"""

from __future__ import annotations

import ctypes
import os
import pathlib
import sys

import numpy as np
import torch

HERE = pathlib.Path(__file__).resolve().parent
REPO = HERE.parent.parent
REF = pathlib.Path(os.environ.get("TIDE_REFERENCE", pathlib.Path(__file__).resolve().parents[3] / "reference"))
sys.path.insert(0, str(REF / "src"))

import tide  # noqa: E402
from tide import backend_utils as bu  # noqa: E402
from tide import utils as rutils  # noqa: E402
from tide.maxwell import _kernel_api as kapi  # noqa: E402

bu._runtime.dll = ctypes.CDLL(str(REPO / "oracle" / "_ref" / "libtide_ref_cpu.so"))
bu._runtime.probed = True
assert bu.is_backend_available()


def case(dtype, seed=13, shots=2, ny=26, nx=34, nt=120):
    g = torch.Generator().manual_seed(seed)
    eps = 3.0 + 6.0 * torch.rand((ny, nx), generator=g, dtype=torch.float64)
    sig = 0.008 * torch.rand((ny, nx), generator=g, dtype=torch.float64)
    deps = 1.0 + 4.0 * torch.rand((ny, nx), generator=g, dtype=torch.float64)
    tau = 2e-10 + 6e-10 * torch.rand((ny, nx), generator=g, dtype=torch.float64)
    mu = torch.ones((ny, nx), dtype=torch.float64)
    dx = 0.02
    dt = 2.5e-11
    amp = tide.ricker(700e6, nt, dt, dtype=torch.float64).view(1, 1, nt).repeat(shots, 1, 1)
    amp = amp * torch.tensor([1.0, 0.7]).view(shots, 1, 1)
    src = torch.tensor([[[5, 9]], [[18, 25]]])
    rec = torch.stack([torch.stack([torch.randint(2, ny - 2, (4,), generator=g),
                                    torch.randint(2, nx - 2, (4,), generator=g)], -1)
                       for _ in range(shots)])
    w = torch.randn((nt, shots, 4), generator=g, dtype=torch.float64)
    return dict(eps=eps.to(dtype), sig=sig.to(dtype), deps=deps.to(dtype), tau=tau.to(dtype),
                mu=mu.to(dtype), dx=dx, dt=dt, amp=amp.to(dtype), src=src, rec=rec,
                w=w.to(dtype), pml=6, nt=nt)


def run(c, python_backend, grads=False):
    leaves = {}
    if grads:
        for k in ("eps", "sig", "deps", "tau"):
            leaves[k] = c[k].clone().requires_grad_(True)
    get = lambda k: leaves.get(k, c[k])  # noqa: E731
    out = kapi.maxwelltm(
        get("eps"), get("sig"), c["mu"], grid_spacing=c["dx"], dt=c["dt"],
        source_amplitude=c["amp"], source_location=c["src"], receiver_location=c["rec"],
        stencil=2, pml_width=c["pml"], python_backend=python_backend, fallback="error",
        dispersion=tide.DebyeDispersion(get("deps"), get("tau")),
    )
    r = out[-1]
    if not grads:
        return r.detach()
    loss = (r * c["w"]).sum()
    gs = torch.autograd.grad(loss, [leaves[k] for k in ("eps", "sig", "deps", "tau")])
    return r.detach(), gs


def main() -> None:
    out = {}
    for dtype, tag in ((torch.float32, "f32"), (torch.float64, "f64")):
        c = case(dtype)
        out[f"r_native_{tag}"] = run(c, False).numpy()
        out[f"r_python_{tag}"] = run(c, True).numpy()
    c = case(torch.float64)
    _, gs = run(c, True, grads=True)
    for k, gv in zip(("eps", "sig", "deps", "tau"), gs):
        out[f"g{k}_f64"] = gv.numpy()
    # the reference's padded Debye coefficients for this case
    pad = c["pml"]
    total = [pad + 1, pad, pad + 1, pad]

    def padm(t):
        order = [total[2], total[3], total[0], total[1]]
        return torch.nn.functional.pad(t[None, None], order, mode="replicate")[0, 0]

    mat = rutils.compile_material_coefficients(
        padm(c["eps"]), padm(c["sig"]), padm(c["mu"]), c["dt"],
        dispersion=tide.DebyeDispersion(padm(c["deps"]), padm(c["tau"])),
    )
    d = mat["debye"]
    for k in ("a", "b", "cp"):
        out[k] = d[k].detach().numpy()
    out["ca"] = mat["ca"].detach().numpy()
    out["cb"] = mat["cb"].detach().numpy()
    c32 = case(torch.float32)
    for k in ("eps", "sig", "deps", "tau", "mu", "amp", "w"):
        out[f"in_{k}_f64"] = c[k].numpy()
        out[f"in_{k}_f32"] = c32[k].numpy()
    out["in_src"] = c["src"].numpy()
    out["in_rec"] = c["rec"].numpy()
    out["in_dx"] = np.array(c["dx"])
    out["in_dt"] = np.array(c["dt"])
    out["in_pml"] = np.array(c["pml"])
    np.savez_compressed(HERE / "debye_case.npz", **out)
    print("wrote", HERE / "debye_case.npz", {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
