"""Generate tests/golden/born_bggrad.npz: the second-order Born gradient from
the reference's own Python path.

Run where the reference tree is mounted (read-only) at $TIDE_REFERENCE
(default: a directory `reference` beside the repository):

    python tests/golden/make_golden_born_bggrad.py

Imports the reference package and runs its public ``borntm`` on the Python
(torch) path in FP64 (python_backend=True) for the heterogeneous 2-shot case
of prep_tm2d.npz and the seeded direction of make_golden_born.py, with the
background epsilon / sigma and the direction depsilon / dsigma all requiring
gradients; back-propagates <w, scattered receivers> + <wb, background
receivers> (seeded weights) with torch autograd.  Stored per stencil (2, 4):
the weights, both receiver sets and the four gradients.
"""

from __future__ import annotations

import os
import pathlib
import sys

import numpy as np
import torch

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
REF = pathlib.Path(os.environ.get("TIDE_REFERENCE", pathlib.Path(__file__).resolve().parents[3] / "reference"))
sys.path.insert(0, str(REF / "src"))

from make_golden_born import direction, inputs  # noqa: E402
from tide.maxwell.tm2d_born import borntm  # noqa: E402


def main():
    c = inputs()
    deps0, dsig0 = direction(tuple(c["eps"].shape))
    out = {"deps": deps0.numpy(), "dsig": dsig0.numpy()}
    for stencil in (2, 4):
        eps = c["eps"].clone().requires_grad_(True)
        sig = c["sig"].clone().requires_grad_(True)
        deps = deps0.clone().requires_grad_(True)
        dsig = dsig0.clone().requires_grad_(True)
        res = borntm(eps, sig, c["mu"], c["dx"], c["dt"], c["amp"], c["src"], c["rec"], c["rec"],
                     depsilon=deps, dsigma=dsig, stencil=stencil, pml_width=c["pml"],
                     python_backend=True, fallback="error")
        bg_r, r = res[-2], res[-1]
        g = torch.Generator().manual_seed(23)
        w = torch.randn(r.shape, generator=g, dtype=r.dtype)
        wb = torch.randn(bg_r.shape, generator=g, dtype=r.dtype)
        ((r * w).sum() + (bg_r * wb).sum()).backward()
        tag = f"s{stencil}"
        out.update({f"w_{tag}": w.numpy(), f"wb_{tag}": wb.numpy(),
                    f"r_{tag}": r.detach().numpy(), f"bg_r_{tag}": bg_r.detach().numpy(),
                    f"geps_{tag}": eps.grad.numpy(), f"gsig_{tag}": sig.grad.numpy(),
                    f"gdeps_{tag}": deps.grad.numpy(), f"gdsig_{tag}": dsig.grad.numpy()})
        print(stencil, {k: float(np.abs(v).max()) for k, v in out.items() if k.endswith(tag)})
    np.savez_compressed(HERE / "born_bggrad.npz", **out)


if __name__ == "__main__":
    main()
