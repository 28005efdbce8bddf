"""Generate the golden fixtures in this directory from the reference itself.

Run in a container where the reference tree is mounted (read-only) at
$TIDE_REFERENCE (default: a directory `reference` beside the repository) and after `make -C oracle ref`
has compiled the reference CPU backend into oracle/_ref/:

    python tests/golden/make_golden.py

It imports the reference Python package, points its ctypes loader at the
reference CPU backend compiled from the reference's own sources, and runs the
reference's public functional API.  Outputs (small .npz files):

  config1.npz      BASELINE config 1 (96x96, nt=300, CPML 10, stencil 2):
                   receivers from the native CPU backend in FP32 and FP64 and
                   from the Python reference in FP32; final Ey (FP32, native).
  prep_tm2d.npz    the exact padded inputs (ca, cb, cq, f, 12 CPML profiles,
                   source/receiver flat indices) the reference hands to its
                   native forward for a small heterogeneous 2-shot case.
  hetero_fwd.npz   receivers of that case from the native CPU backend and from
                   the Python reference, FP32 and FP64, stencils 2, 4, 6, 8.
  abi_specs.json   the reference loader's ctypes argtypes and argument names
                   for the TM forward / forward_with_storage / backward passes.
  hetero_grad.npz  exact gradients (Python reference, torch autograd, FP64 and
                   FP32) of a seeded linear functional of the receivers with
                   respect to epsilon and sigma, stencils 2 and 4.
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
assert bu.is_backend_available()


def config1(dtype, python_backend):
    ny = nx = 96
    nt = 300
    dx = 0.02
    dt = 4e-11
    eps = torch.full((ny, nx), 4.0, dtype=dtype)
    sig = torch.zeros_like(eps)
    mu = torch.ones_like(eps)
    amp = tide.ricker(800e6, nt, dt, dtype=dtype).view(1, 1, nt)
    src = torch.tensor([[[20, 48]]])
    rec = torch.tensor([[[20, 60]]])
    out = kapi.maxwelltm(
        eps, sig, mu, grid_spacing=dx, dt=dt, source_amplitude=amp, source_location=src,
        receiver_location=rec, stencil=2, pml_width=10, python_backend=python_backend,
        fallback="error",
    )
    return out


def hetero_case(dtype, seed=7, shots=2, ny=24, nx=30, nt=150):
    g = torch.Generator().manual_seed(seed)
    base = 2.0 + 7.0 * torch.rand((ny, nx), generator=g, dtype=torch.float64)
    k = torch.tensor([[1.0, 2.0, 1.0], [2.0, 4.0, 2.0], [1.0, 2.0, 1.0]], dtype=torch.float64) / 16
    eps = torch.nn.functional.conv2d(base[None, None], k[None, None], padding=1)[0, 0]
    sig = 0.01 * torch.rand((ny, nx), generator=g, dtype=torch.float64)
    mu = torch.ones((ny, nx), dtype=torch.float64)
    dx = [0.02, 0.025]
    dt = 3.0e-11
    amp = tide.ricker(600e6, nt, dt, dtype=torch.float64).view(1, 1, nt).repeat(shots, 1, 1)
    amp[1] *= 0.7
    src = torch.tensor([[[4, 6]], [[5, 22]]])[:shots]
    rec = torch.tensor(
        [[[3, 2], [10, 9], [20, 15], [12, 27], [0, 0]], [[2, 28], [9, 3], [21, 20], [13, 13], [23, 29]]]
    )[:shots]
    w = torch.randn((nt, shots, rec.shape[1]), generator=g, dtype=torch.float64)
    return dict(eps=eps.to(dtype), sig=sig.to(dtype), mu=mu.to(dtype), dx=dx, dt=dt, amp=amp.to(dtype),
                src=src, rec=rec, w=w.to(dtype), nt=nt, pml=6)


def run_case(c, stencil, python_backend, grads=False):
    eps = c["eps"].clone().requires_grad_(grads)
    sig = c["sig"].clone().requires_grad_(grads)
    out = kapi.maxwelltm(
        eps, sig, c["mu"], grid_spacing=c["dx"], dt=c["dt"], source_amplitude=c["amp"],
        source_location=c["src"], receiver_location=c["rec"], stencil=stencil,
        pml_width=c["pml"], python_backend=python_backend, fallback="error",
    )
    r = out[-1]
    if not grads:
        return r.detach(), None, None
    loss = (r * c["w"]).sum()
    ge, gs = torch.autograd.grad(loss, [eps, sig])
    return r.detach(), ge, gs


def capture_prepared(c):
    captured: list[torch.Tensor] = []
    orig = bu.tensor_to_ptr

    def rec_ptr(t):
        captured.append(t)
        return orig(t)

    bu.tensor_to_ptr = rec_ptr
    try:
        run_case(c, 2, False)
    finally:
        bu.tensor_to_ptr = orig
    names = ["ca", "cb", "cq", "f", "ey", "hx", "hz", "m_ey_x", "m_ey_z", "m_hx_z", "m_hz_x",
             "debye_a", "debye_b", "debye_cp", "polarization", "ey_prev", "r",
             "ay", "by", "ayh", "byh", "ax", "bx", "axh", "bxh", "ky", "kyh", "kx", "kxh",
             "sources_i", "receivers_i"]
    d = dict(zip(names, captured[: len(names)]))
    keep = ["ca", "cb", "cq", "f", "ay", "by", "ayh", "byh", "ax", "bx", "axh", "bxh",
            "ky", "kyh", "kx", "kxh", "sources_i", "receivers_i"]
    return {k: d[k].detach().numpy() for k in keep}


def abi_specs():
    import json

    specs = {}
    passes = {
        "maxwell_tm": ("forward", "forward_with_storage", "backward", "background_vjp_reuse",
                       "born_forward", "born_forward_with_storage",
                       "born_tangent_forward_with_storage", "born_backward",
                       "born_backward_bggrad"),
        "maxwell_3d": ("forward", "forward_with_storage", "backward", "born_forward",
                       "born_forward_with_storage", "born_backward", "born_backward_bggrad"),
    }
    for prop, names in passes.items():
        for pass_name in names:
            for dt in ("float", "double"):
                ats = bu._template_argtypes(f"{prop}_{pass_name}", dt)
                specs[f"{prop}_{pass_name}_{dt}"] = [a.__name__ for a in ats]
            specs[f"{prop}_{pass_name}_names"] = list(bu.backend_signature(prop, pass_name))
    (HERE / "abi_specs.json").write_text(json.dumps(specs, indent=1))


def main():
    if sys.argv[1:] == ["specs"]:  # only the loader's argtypes
        abi_specs()
        return
    abi_specs()
    out = {}
    n32 = config1(torch.float32, False)
    n64 = config1(torch.float64, False)
    p32 = config1(torch.float32, True)
    out["r_native_f32"] = n32[-1].numpy()
    out["r_native_f64"] = n64[-1].numpy()
    out["r_python_f32"] = p32[-1].numpy()
    out["ey_native_f32"] = n32[0].numpy()
    np.savez_compressed(HERE / "config1.npz", **out)

    c32 = hetero_case(torch.float32)
    c64 = hetero_case(torch.float64)
    inputs = {k: (v.numpy() if isinstance(v, torch.Tensor) else np.asarray(v)) for k, v in c64.items()}
    np.savez_compressed(HERE / "prep_tm2d.npz", **capture_prepared(c32),
                        **{"in_" + k: v for k, v in inputs.items()})

    fwd = {}
    for st in (2, 4, 6, 8):
        fwd[f"r_native_f32_s{st}"] = run_case(c32, st, False)[0].numpy()
        fwd[f"r_native_f64_s{st}"] = run_case(c64, st, False)[0].numpy()
        fwd[f"r_python_f32_s{st}"] = run_case(c32, st, True)[0].numpy()
        fwd[f"r_python_f64_s{st}"] = run_case(c64, st, True)[0].numpy()
    np.savez_compressed(HERE / "hetero_fwd.npz", **fwd)

    grad = {}
    for st in (2, 4):
        r, ge, gs = run_case(c64, st, True, grads=True)
        grad[f"r_f64_s{st}"] = r.numpy()
        grad[f"geps_f64_s{st}"] = ge.numpy()
        grad[f"gsig_f64_s{st}"] = gs.numpy()
        r, ge, gs = run_case(c32, st, True, grads=True)
        grad[f"geps_f32_s{st}"] = ge.numpy()
        grad[f"gsig_f32_s{st}"] = gs.numpy()
    np.savez_compressed(HERE / "hetero_grad.npz", **grad)
    for f in sorted(HERE.glob("*.npz")):
        print(f.name, f.stat().st_size)


if __name__ == "__main__":
    main()
