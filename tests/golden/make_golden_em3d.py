"""Generate the 3-D golden fixture from the reference itself.

Run where the reference tree is mounted (read-only) at $TIDE_REFERENCE
(default: a directory `reference` beside the repository), after `make -C oracle ref`:

    python tests/golden/make_golden_em3d.py

Runs the reference's public 3-D functional API (tide.maxwell3d) on a small
seeded heterogeneous case with two shots, in FP64:
  - receivers from the reference CPU backend compiled from its own sources
    (oracle/_ref) and from the reference Python path;
  - exact gradients of a seeded linear functional of the receivers with
    respect to epsilon and sigma, from the Python path (torch autograd);
  - the inputs, so the tests rebuild the identical problem.
Output: em3d_case.npz.

The same runs at stencil orders 4, 6 and 8 (the time step halved, inside the
stability limit of every order) give em3d_hi_case.npz: receivers from the
reference CPU backend and the Python path, and Python-path gradients, keyed
by order (r_native_s4, r_python_s4, geps_s4, gsig_s4, ...).
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
from tide.maxwell import _kernel_api as kapi  # noqa: E402

bu._runtime.dll = ctypes.CDLL(str(REPO / "oracle" / "_ref" / "libtide_ref_cpu.so"))
bu._runtime.probed = True


def case(seed: int = 11):
    g = torch.Generator().manual_seed(seed)
    nz, ny, nx, S, nt = 10, 12, 14, 2, 60
    eps = 1.5 + 6.0 * torch.rand((nz, ny, nx), generator=g, dtype=torch.float64)
    eps = torch.nn.functional.avg_pool3d(eps[None, None], 3, 1, 1, count_include_pad=False)[0, 0]
    sig = 0.006 * torch.rand((nz, ny, nx), generator=g, dtype=torch.float64)
    mu = torch.ones((nz, ny, nx), dtype=torch.float64)
    dx = 0.02
    vmax = 299792458.0 / float(eps.min().sqrt())
    dt = 0.9 * dx / (vmax * 3 ** 0.5)
    amp = tide.ricker(700e6, nt, dt, dtype=torch.float64).view(1, 1, nt).repeat(S, 1, 1)
    amp = amp * torch.tensor([1.0, 0.7], dtype=torch.float64).view(S, 1, 1)
    src = torch.tensor([[[4, 5, 6]], [[6, 7, 5]]])
    rec = torch.tensor([[[2, 3, 4], [3, 8, 9], [7, 2, 11]], [[2, 9, 3], [5, 5, 5], [8, 10, 12]]])
    return dict(eps=eps, sig=sig, mu=mu, dx=dx, dt=dt, amp=amp, src=src, rec=rec, nt=nt, pml=3)


def run(c, python_backend, grads, stencil=2):
    eps = c["eps"].clone().requires_grad_(grads)
    sig = c["sig"].clone().requires_grad_(grads)
    out = kapi.maxwell3d(eps, sig, c["mu"], c["dx"], c["dt"], c["amp"], c["src"], c["rec"],
                         stencil=stencil, pml_width=c["pml"], python_backend=python_backend,
                         source_component="ey", receiver_component="ey")
    r = out[-1]
    if not grads:
        return r.detach().numpy(), None, None
    w = torch.randn(r.shape, generator=torch.Generator().manual_seed(5), dtype=r.dtype)
    (r * w).sum().backward()
    return r.detach().numpy(), eps.grad.numpy(), sig.grad.numpy()


def main():
    c = case()
    r_native, _, _ = run(c, False, False)
    r_py, geps, gsig = run(c, True, True)
    np.savez_compressed(
        HERE / "em3d_case.npz", eps=c["eps"].numpy(), sig=c["sig"].numpy(), mu=c["mu"].numpy(),
        dx=c["dx"], dt=c["dt"], amp=c["amp"].numpy(), src=c["src"].numpy(),
        rec=c["rec"].numpy(), nt=c["nt"], pml=c["pml"], r_native_f64=r_native,
        r_python_f64=r_py, geps_python_f64=geps, gsig_python_f64=gsig)
    print("rel(native, python) receivers:", np.linalg.norm(r_native - r_py) / np.linalg.norm(r_py))

    c = case()
    c["dt"] = 0.5 * c["dt"]
    c["amp"] = tide.ricker(700e6, c["nt"], c["dt"], dtype=torch.float64).view(1, 1, -1).repeat(2, 1, 1)
    c["amp"] = c["amp"] * torch.tensor([1.0, 0.7], dtype=torch.float64).view(2, 1, 1)
    hi = dict(dt=c["dt"], amp=c["amp"].numpy())
    for st in (4, 6, 8):
        r_native, _, _ = run(c, False, False, st)
        r_py, geps, gsig = run(c, True, True, st)
        hi.update({f"r_native_s{st}": r_native, f"r_python_s{st}": r_py, f"geps_s{st}": geps,
                   f"gsig_s{st}": gsig})
        print(f"stencil {st}: rel(native, python) receivers:",
              np.linalg.norm(r_native - r_py) / np.linalg.norm(r_py))
    np.savez_compressed(HERE / "em3d_hi_case.npz", **hi)


if __name__ == "__main__":
    main()
