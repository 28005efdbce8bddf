"""Test-side drivers for the CPU checkers (oracle/ only; never the product).

* ``Oracle``   — ctypes binding of oracle/_build/libtide_oracle.so, the plain-C
                 restatement of the reference TM2D path (forward, storage,
                 exact adjoint), plus an autograd wrapper so gradients can be
                 chained to epsilon/sigma exactly like the product does.
* ``RefCPU``   — ctypes binding of oracle/_ref/libtide_ref_cpu.so, the
                 reference's own CPU backend compiled from its sources
                 (present only where the reference tree was available at
                 build time).

Both consume a ``TMProblem`` prepared on the CPU by
``tide_b200.tm2d.prepare_tm2d``.
"""

from __future__ import annotations

import ctypes
import pathlib
import subprocess
from ctypes import c_bool, c_double, c_float, c_int, c_int64, c_void_p

import torch

REPO = pathlib.Path(__file__).resolve().parent.parent
ORACLE_SO = REPO / "oracle" / "_build" / "libtide_oracle.so"
REF_SO = REPO / "oracle" / "_ref" / "libtide_ref_cpu.so"
PROFILES = ("ay", "by", "ayh", "byh", "ax", "bx", "axh", "bxh", "ky", "kyh", "kx", "kxh")


def _p(t):
    return 0 if t is None or t.numel() == 0 else t.data_ptr()


def build_oracle() -> pathlib.Path:
    subprocess.run(["make", "-s", "-C", str(REPO / "oracle")], check=True)
    return ORACLE_SO


class Oracle:
    def __init__(self):
        if not ORACLE_SO.exists():
            build_oracle()
        self.lib = ctypes.CDLL(str(ORACLE_SO))

    def _fn(self, name, dtype, ft):
        sfx = "float" if dtype == torch.float32 else "double"
        fn = getattr(self.lib, f"tide_oracle_tm_{name}_{sfx}")
        fn.restype = None
        return fn, (c_float if dtype == torch.float32 else c_double)

    def forward(self, pb, ca, cb, f, r, start_t=0, nt=None, *, store=None, k=1, fmt=0,
                need_ca=False, need_cb=False):
        """Advance pb.fields in place; store = (ey_store, curl_store) or None."""
        nt = pb.nt if nt is None else nt
        ey, hx, hz, mex, mez, mhx, mhz = pb.fields
        prof = [_p(pb.profiles[n]) for n in PROFILES]
        P, I, B = c_void_p, c_int64, c_bool
        if store is None:
            fn, F = self._fn("forward", pb.dtype, None)
            fn.argtypes = [c_int] + [P] * 12 + [P] * 12 + [P, P, F, F] + [I] * 6 + [B] * 3 + [I] * 5
            fn(pb.stencil, _p(ca), _p(cb), _p(pb.cq), _p(f), _p(ey), _p(hx), _p(hz), _p(mex), _p(mez),
               _p(mhx), _p(mhz), _p(r), *prof, _p(pb.sources_i), _p(pb.receivers_i), pb.rdy, pb.rdx,
               nt, pb.n_shots, pb.ny, pb.nx, pb.n_src, pb.n_rec, pb.batched, pb.batched,
               pb.batched, start_t, pb.pml_y0, pb.pml_x0, pb.pml_y1, pb.pml_x1)
            return
        fn, F = self._fn("forward_with_storage", pb.dtype, None)
        fn.argtypes = ([c_int] + [P] * 12 + [P, P] + [P] * 12 + [P, P, F, F] + [I] * 8
                       + [B] * 5 + [I] * 5)
        fn(pb.stencil, _p(ca), _p(cb), _p(pb.cq), _p(f), _p(ey), _p(hx), _p(hz), _p(mex), _p(mez),
           _p(mhx), _p(mhz), _p(r), _p(store[0]), _p(store[1]), *prof, _p(pb.sources_i),
           _p(pb.receivers_i), pb.rdy, pb.rdx, nt, pb.n_shots, pb.ny, pb.nx, pb.n_src, pb.n_rec, k,
           fmt, need_ca, need_cb, pb.batched, pb.batched, pb.batched, start_t, pb.pml_y0,
           pb.pml_x0, pb.pml_y1, pb.pml_x1)

    def backward(self, pb, ca, cb, grad_r, store, *, k=1, fmt=0, need_ca=True, need_cb=True,
                 start_t=None, nt=None, lam=None, grads=None):
        """Exact adjoint; returns (grad_ca, grad_cb, grad_f, lam_fields)."""
        S, ny, nx = pb.n_shots, pb.ny, pb.nx
        nt = pb.nt if nt is None else nt
        start_t = pb.nt if start_t is None else start_t
        dt = pb.dtype
        z = lambda *s: torch.zeros(s, dtype=dt)  # noqa: E731
        lam = lam if lam is not None else [z(S, ny, nx) for _ in range(7)]
        scratch = z(4, S, ny, nx)
        mshape = (S, ny, nx) if pb.batched else (ny, nx)
        if grads is None:
            grads = (z(*mshape), z(*mshape), z(pb.nt, S, pb.n_src) if pb.n_src else z(0))
        gca, gcb, gf = grads
        shot_ca, shot_cb = z(S, ny, nx), z(S, ny, nx)
        fn, F = self._fn("backward", dt, None)
        P, I, B = c_void_p, c_int64, c_bool
        fn.argtypes = ([c_int] + [P] * 4 + [P] * 7 + [P] + [P, P] + [P] * 5 + [P] * 12 + [P, P, F, F]
                       + [I] * 8 + [B] * 5 + [I] * 5)
        fn(pb.stencil, _p(ca), _p(cb), _p(pb.cq), _p(grad_r), *[_p(t) for t in lam], _p(scratch),
           _p(store[0]) if store else 0, _p(store[1]) if store else 0, _p(gf), _p(gca), _p(gcb),
           _p(shot_ca), _p(shot_cb), *[_p(pb.profiles[n]) for n in PROFILES], _p(pb.sources_i),
           _p(pb.receivers_i), pb.rdy, pb.rdx, nt, S, ny, nx, pb.n_src, pb.n_rec, k, fmt,
           need_ca and store is not None, need_cb and store is not None, pb.batched, pb.batched,
           pb.batched, start_t, pb.pml_y0, pb.pml_x0, pb.pml_y1, pb.pml_x1)
        return gca, gcb, gf, lam


class OracleTM(torch.autograd.Function):
    """Autograd node over (ca, cb, f) backed by the C oracle (CPU)."""

    @staticmethod
    def forward(ctx, ca, cb, f, pb, oracle, k, fmt):
        S, ny, nx, nt = pb.n_shots, pb.ny, pb.nx, pb.nt
        r = torch.zeros((nt, S, pb.n_rec), dtype=pb.dtype)
        n_store = (nt + k - 1) // k
        sdt = torch.bfloat16 if fmt == 1 else pb.dtype
        store = (torch.zeros((n_store, S, ny, nx), dtype=sdt),
                 torch.zeros((n_store, S, ny, nx), dtype=sdt))
        oracle.forward(pb, ca.detach(), cb.detach(), f.detach(), r, store=store, k=k, fmt=fmt,
                       need_ca=True, need_cb=True)
        ctx.save_for_backward(ca, cb)
        ctx.pb, ctx.oracle, ctx.store, ctx.k, ctx.fmt = pb, oracle, store, k, fmt
        return r

    @staticmethod
    def backward(ctx, grad_r):
        ca, cb = ctx.saved_tensors
        pb = ctx.pb
        gca, gcb, gf, _ = ctx.oracle.backward(pb, ca.detach(), cb.detach(), grad_r.contiguous(),
                                              ctx.store, k=ctx.k, fmt=ctx.fmt)
        if not pb.batched:
            gca, gcb = gca.unsqueeze(0), gcb.unsqueeze(0)
        return gca, gcb, (gf.reshape(-1) if pb.n_src else None), None, None, None, None


class RefCPU:
    """The reference's CPU backend (maxwell_tm_{S}_{dtype}_forward_cpu)."""

    def __init__(self, path: pathlib.Path = REF_SO):
        self.lib = ctypes.CDLL(str(path))

    def forward(self, pb, ca, cb, f, r, n_threads=0):
        import sys

        sys.path.insert(0, str(REPO / "tide-gpr_b200"))
        from tide_b200 import _native as nat

        sfx = "float" if pb.dtype == torch.float32 else "double"
        fn = getattr(self.lib, f"maxwell_tm_{pb.stencil}_{sfx}_forward_cpu")
        fn.argtypes = nat.argtypes("maxwell_tm_forward", sfx)
        fn.restype = None
        ey, hx, hz, mex, mez, mhx, mhz = pb.fields
        fn(_p(ca), _p(cb), _p(pb.cq), _p(f), _p(ey), _p(hx), _p(hz), _p(mex), _p(mez), _p(mhx),
           _p(mhz), 0, 0, 0, 0, 0, _p(r), 0, *[_p(pb.profiles[n]) for n in PROFILES],
           _p(pb.sources_i), _p(pb.receivers_i), pb.rdy, pb.rdx, pb.dt, pb.nt, pb.n_shots, pb.ny,
           pb.nx, pb.n_src, pb.n_rec, 1, False, pb.batched, pb.batched, pb.batched, 0, pb.pml_y0,
           pb.pml_x0, pb.pml_y1, pb.pml_x1, n_threads, 0, 0)


def rel_l2(a: torch.Tensor, b: torch.Tensor) -> float:
    a = a.detach().double().cpu()
    b = b.detach().double().cpu()
    den = torch.linalg.vector_norm(b)
    return float(torch.linalg.vector_norm(a - b) / (den if den > 0 else 1.0))


def set_grad_order(oracle: Oracle, order: int) -> None:
    """0: reference per-shot-then-shots order; 1: step-major (the CUDA kernels')."""
    oracle.lib.tide_oracle_set_grad_order.argtypes = [c_int]
    oracle.lib.tide_oracle_set_grad_order(order)
