"""Generate tests/golden/born3d_grad.npz from the reference's 3-D Born path.

Run where the reference tree is mounted (read-only) at $TIDE_REFERENCE
(default: a directory `reference` beside the repository):

    python tests/golden/make_golden_born3d.py

Imports the reference package and runs its public ``born3d`` on the Python
(torch) path in FP64 (python_backend=True) for the two-shot case of
em3d_case.npz and a seeded smooth (depsilon, dsigma) direction, stencils 2
and 4; then back-propagates a seeded linear functional of the scattered
receivers to depsilon and dsigma with torch autograd.  Stored: the
direction, the functional's weights, the scattered receivers and the two
gradients per stencil (born3d_grad.npz); and, with the background epsilon /
sigma requiring gradients as well, the four gradients of a second seeded
functional at stencil 2 (born3d_bggrad.npz, the second-order Born pin).
"""

from __future__ import annotations

import os
import pathlib
import sys

import numpy as np
import torch

HERE = pathlib.Path(__file__).resolve().parent
REF = pathlib.Path(os.environ.get("TIDE_REFERENCE", pathlib.Path(__file__).resolve().parents[3] / "reference"))
sys.path.insert(0, str(REF / "src"))

from tide.maxwell.maxwell3d_born import born3d  # noqa: E402


def direction(shape, seed=13):
    g = torch.Generator().manual_seed(seed)
    k = torch.ones((1, 1, 3, 3, 3), dtype=torch.float64) / 27

    def smooth(scale):
        u = torch.randn((1, 1) + shape, generator=g, dtype=torch.float64)
        u = torch.nn.functional.conv3d(torch.nn.functional.pad(u, (1,) * 6, mode="replicate"), k)
        return scale * u[0, 0]

    return smooth(0.5), smooth(2e-3)


def main():
    z = np.load(HERE / "em3d_case.npz")
    eps, sig, mu = (torch.from_numpy(z[n]) for n in ("eps", "sig", "mu"))
    amp, src, rec = (torch.from_numpy(z[n]) for n in ("amp", "src", "rec"))
    deps, dsig = direction(tuple(eps.shape))
    out = {"deps": deps.numpy(), "dsig": dsig.numpy()}
    for stencil in (2, 4):
        dt = float(z["dt"]) * (1.0 if stencil == 2 else 0.5)
        a = amp if stencil == 2 else torch.from_numpy(np.load(HERE / "em3d_hi_case.npz")["amp"])
        de = deps.clone().requires_grad_(True)
        ds = dsig.clone().requires_grad_(True)
        res = born3d(eps, sig, mu, float(z["dx"]), dt, a, src, rec, depsilon=de, dsigma=ds,
                     stencil=stencil, pml_width=int(z["pml"]), python_backend=True,
                     fallback="error")
        r = res[-1]
        w = torch.randn(r.shape, generator=torch.Generator().manual_seed(17), dtype=r.dtype)
        (r * w).sum().backward()
        out[f"w_s{stencil}"] = w.numpy()
        out[f"r_s{stencil}"] = r.detach().numpy()
        out[f"geps_s{stencil}"] = de.grad.numpy()
        out[f"gsig_s{stencil}"] = ds.grad.numpy()
        out[f"dt_s{stencil}"] = dt
        print(stencil, float(r.abs().max()), float(de.grad.abs().max()), float(ds.grad.abs().max()))
    np.savez_compressed(HERE / "born3d_grad.npz", **out)

    # second order: the background epsilon / sigma require gradients too
    sec = {}
    for stencil in (2,):
        dt = float(z["dt"])
        e_ = eps.clone().requires_grad_(True)
        s_ = sig.clone().requires_grad_(True)
        de = deps.clone().requires_grad_(True)
        ds = dsig.clone().requires_grad_(True)
        res = born3d(e_, s_, mu, float(z["dx"]), dt, amp, src, rec, depsilon=de, dsigma=ds,
                     stencil=stencil, pml_width=int(z["pml"]), python_backend=True,
                     fallback="error")
        r = res[-1]
        w = torch.randn(r.shape, generator=torch.Generator().manual_seed(31), dtype=r.dtype)
        (r * w).sum().backward()
        tag = f"s{stencil}"
        sec.update({f"w_{tag}": w.numpy(), f"r_{tag}": r.detach().numpy(),
                    f"geps_{tag}": e_.grad.numpy(), f"gsig_{tag}": s_.grad.numpy(),
                    f"gdeps_{tag}": de.grad.numpy(), f"gdsig_{tag}": ds.grad.numpy()})
        print("second order", stencil, {k: float(np.abs(v).max()) for k, v in sec.items()})
    np.savez_compressed(HERE / "born3d_bggrad.npz", **sec)


if __name__ == "__main__":
    main()
