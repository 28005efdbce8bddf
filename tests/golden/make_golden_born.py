"""Generate tests/golden/born_case.npz from the reference's Born propagator.

Run where the reference tree is mounted (read-only) at $TIDE_REFERENCE
(default: a directory `reference` beside the repository):

    python tests/golden/make_golden_born.py

It imports the reference Python package and runs its public ``borntm`` on
its Python (torch) path in FP64 (``python_backend=True``), for the
heterogeneous 2-shot case of prep_tm2d.npz (inputs stored there) and a
seeded smooth (depsilon, dsigma) direction, stencils 2 and 4, with and
without source linearization.  Stored: the direction, the background and
scattered receiver data, and the final scattered Ey.
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

from tide.maxwell.tm2d_born import borntm  # noqa: E402


def inputs():
    z = np.load(HERE / "prep_tm2d.npz")
    d = {k[3:]: torch.from_numpy(z[k]) for k in z.files if k.startswith("in_")}
    return dict(eps=d["eps"].double(), sig=d["sig"].double(), mu=d["mu"].double(),
                dx=[float(v) for v in d["dx"]], dt=float(d["dt"]), amp=d["amp"].double(),
                src=d["src"], rec=d["rec"], nt=int(d["nt"]), pml=int(d["pml"]))


def direction(shape, seed=11):
    g = torch.Generator().manual_seed(seed)
    k = torch.ones((1, 1, 5, 5), dtype=torch.float64) / 25
    def smooth(scale):
        u = torch.randn((1, 1) + shape, generator=g, dtype=torch.float64)
        u = torch.nn.functional.conv2d(torch.nn.functional.pad(u, (2, 2, 2, 2), mode="reflect"), k)
        return scale * u[0, 0]
    return smooth(0.5), smooth(2e-3)


def main():
    c = inputs()
    deps, dsig = direction(tuple(c["eps"].shape))
    out = {"deps": deps.numpy(), "dsig": dsig.numpy()}
    for stencil in (2, 4):
        for lin in (True, False):
            res = borntm(
                c["eps"], c["sig"], c["mu"], c["dx"], c["dt"], c["amp"], c["src"], c["rec"],
                c["rec"], depsilon=deps, dsigma=dsig, stencil=stencil, pml_width=c["pml"],
                linearize_source=lin, python_backend=True, fallback="error",
            )
            tag = f"s{stencil}_{'lin' if lin else 'nolin'}"
            out[f"bg_r_{tag}"] = res[-2].detach().numpy()
            out[f"r_{tag}"] = res[-1].detach().numpy()
            out[f"dey_{tag}"] = res[7].detach().numpy()
    np.savez_compressed(HERE / "born_case.npz", **out)
    print("wrote", HERE / "born_case.npz", {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
