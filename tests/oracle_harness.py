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


    def born_forward(self, pb, dca, dcb, f0, df, tan, r, bg_r, start_t=0, nt=None, *,
                     store=None, k=1, fmt=0):
        """Born forward: advance pb.fields (background) and tan (the 7
        scattered state tensors) in place.  store: 4 histories (background
        Ey^n, curl H^n, scattered dEy^n, dcurl; None entries skipped) or None."""
        nt = pb.nt if nt is None else nt
        prof = [_p(pb.profiles[n]) for n in PROFILES]
        P, I, B = c_void_p, c_int64, c_bool
        fn, F = self._fn("born_forward_store", pb.dtype, None)
        fn.argtypes = ([c_int] + [P] * 7 + [P] * 14 + [P] * 2 + [P] * 12 + [P, P, F, F]
                       + [I] * 6 + [B] * 3 + [I] * 5 + [P, I, I])
        st = (c_void_p * 4)(*[_p(t) if t is not None else None for t in store]) if store else None
        fn(pb.stencil, _p(pb.ca), _p(pb.cb), _p(pb.cq), _p(dca), _p(dcb), _p(f0), _p(df),
           *[_p(t) for t in pb.fields], *[_p(t) for t in tan], _p(r), _p(bg_r), *prof,
           _p(pb.sources_i), _p(pb.receivers_i), pb.rdy, pb.rdx, nt, pb.n_shots, pb.ny, pb.nx,
           pb.n_src, pb.n_rec, pb.batched, pb.batched, pb.batched, start_t, pb.pml_y0,
           pb.pml_x0, pb.pml_y1, pb.pml_x1, st, k, fmt)

    def born_bggrad(self, pb, dca, dcb, grad_r, grad_bg_r, store, *, k=1, fmt=0):
        """Second-order Born adjoint (joint background + scattered state) over
        the 4 histories of born_forward(store=...); returns grad_ca,
        grad_cb, grad_dca, grad_dcb (model-shaped), grad_f0, grad_df
        ([nt, S, n_src]), lam (7) and eta (7)."""
        S, ny, nx, dt = pb.n_shots, pb.ny, pb.nx, pb.dtype
        z = lambda *s: torch.zeros(s, dtype=dt)  # noqa: E731
        lam = [z(S, ny, nx) for _ in range(7)]
        eta = [z(S, ny, nx) for _ in range(7)]
        scratch = z(8, S, ny, nx)
        mshape = (S, ny, nx) if pb.batched else (ny, nx)
        g = [z(*mshape) for _ in range(4)]
        gf0, gdf = z(pb.nt, S, max(pb.n_src, 1)), z(pb.nt, S, max(pb.n_src, 1))
        fn, F = self._fn("born_bggrad", dt, None)
        P, I, B = c_void_p, c_int64, c_bool
        fn.argtypes = ([c_int] + [P] * 7 + [P] * 3 + [P] + [P] * 3 + [P] + [P] + [P] * 4 + [P] * 6
                       + [P] * 12 + [P, P, F, F] + [I] * 8 + [B] * 3 + [I] * 5)
        arr = lambda ts: (c_void_p * len(ts))(*[_p(t) for t in ts])  # noqa: E731
        fn(pb.stencil, _p(pb.ca), _p(pb.cb), _p(pb.cq), _p(dca), _p(dcb), _p(grad_r),
           _p(grad_bg_r), *[_p(t) for t in lam[:3]], arr(lam[3:]), *[_p(t) for t in eta[:3]],
           arr(eta[3:]), _p(scratch), *[_p(t) for t in store], _p(gdf), _p(gf0), *[_p(t) for t in g],
           *[_p(pb.profiles[n]) for n in PROFILES], _p(pb.sources_i), _p(pb.receivers_i), pb.rdy,
           pb.rdx, pb.nt, S, ny, nx, pb.n_src, pb.n_rec, k, fmt, pb.batched, pb.batched,
           pb.batched, pb.nt, pb.pml_y0, pb.pml_x0, pb.pml_y1, pb.pml_x1)
        return (*g, gf0, gdf, lam, eta)

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

    def born_forward(self, pb, dca, dcb, f0, df, tan, r, bg_r, n_threads=0):
        """The reference's maxwell_tm_{S}_{dtype}_born_forward_cpu."""
        import sys

        sys.path.insert(0, str(REPO / "tide-gpr_b200"))
        from tide_b200 import _native as nat

        sfx = "float" if pb.dtype == torch.float32 else "double"
        fn = getattr(self.lib, f"maxwell_tm_{pb.stencil}_{sfx}_born_forward_cpu")
        fn.argtypes = nat.argtypes("maxwell_tm_born_forward", sfx)
        fn.restype = None
        fn(_p(pb.ca), _p(pb.cb), _p(pb.cq), _p(dca), _p(dcb), _p(f0), _p(df),
           *[_p(t) for t in pb.fields], *[_p(t) for t in tan], _p(r), _p(bg_r),
           *[_p(pb.profiles[n]) for n in PROFILES], _p(pb.sources_i), _p(pb.receivers_i),
           pb.rdy, pb.rdx, pb.dt, pb.nt, pb.n_shots, pb.ny, pb.nx, pb.n_src, pb.n_rec, 1,
           pb.batched, pb.batched, pb.batched, 0, pb.pml_y0, pb.pml_x0, pb.pml_y1, pb.pml_x1,
           n_threads, 0, 0)


def rel_l2(a: torch.Tensor, b: torch.Tensor) -> float:
    a = a.detach().double().cpu()
    b = b.detach().double().cpu()
    den = torch.linalg.vector_norm(b)
    return float(torch.linalg.vector_norm(a - b) / (den if den > 0 else 1.0))


def set_grad_order(oracle: Oracle, order: int) -> None:
    """0: reference per-shot-then-shots order; 1: step-major (the CUDA kernels')."""
    oracle.lib.tide_oracle_set_grad_order.argtypes = [c_int]
    oracle.lib.tide_oracle_set_grad_order(order)


# --------------------------------------------------------------------- 3-D
PROFILES_3D = ("az", "bz", "azh", "bzh", "ay", "by", "ayh", "byh", "ax", "bx", "axh", "bxh",
               "kz", "kzh", "ky", "kyh", "kx", "kxh")


def _ptr_array(ts):
    return (c_void_p * len(ts))(*[_p(t) for t in ts])


class Oracle3D:
    """ctypes binding of the C restatement of the reference 3-D path
    (tide_oracle_em3d_*).  Memories are full [S, nz, ny, nx] arrays here."""

    def __init__(self):
        if not ORACLE_SO.exists():
            build_oracle()
        self.lib = ctypes.CDLL(str(ORACLE_SO))

    def _fn(self, name, dtype, stencil=2):
        self.lib.tide_oracle_em3d_set_stencil(c_int(stencil))
        sfx = "float" if dtype == torch.float32 else "double"
        fn = getattr(self.lib, f"tide_oracle_em3d_{name}_{sfx}")
        fn.restype = None
        return fn, (c_float if dtype == torch.float32 else c_double)

    @staticmethod
    def full_state(pb):
        """Full-layout copies of pb's fields and CPML memories (CPU)."""
        from tide_b200.em3d import MEM_AXES

        fields = [t.detach().cpu().clone() for t in pb.fields]
        mem = [pb.layout.unpack(m.detach().cpu(), a).contiguous()
               for m, a in zip(pb.memories, MEM_AXES)]
        return fields, mem

    def forward(self, pb, ca, cb, f, r, fields, mem, *, store=None, k=1, fmt=0, start_t=0,
                nt=None):
        nt = pb.nt if nt is None else nt
        fn, F = self._fn("forward", pb.dtype, pb.stencil)
        P, I = c_void_p, c_int64
        pml = (c_int64 * 6)(*pb.pml)
        fn.argtypes = [P, P, P, P, P, P, P, P, P, P, F, F, F, I, I, I, I, I, I, I, I, P, c_int,
                       c_int, c_int, c_int, c_int, P, I, c_int]
        prof = _ptr_array([pb.profiles[n].cpu() for n in PROFILES_3D])
        st = _ptr_array(list(store)) if store is not None else None
        fn(_p(ca), _p(cb), _p(pb.cq.cpu()), _p(f), _ptr_array(fields), _ptr_array(mem), _p(r),
           prof, _p(pb.sources_i.cpu()), _p(pb.receivers_i.cpu()), pb.rdz, pb.rdy, pb.rdx, nt,
           pb.n_shots, pb.nz, pb.ny, pb.nx, pb.n_src, pb.n_rec, start_t, pml, int(pb.batched),
           int(pb.batched), int(pb.batched), pb.src_comp, pb.rec_comp,
           st if st is not None else None, k, fmt)

    def born_forward(self, pb, dca, dcb, f0, df, fields, mem, dfields, dmem, r, bg_r, *,
                     store=None, k=1, fmt=0):
        """3-D Born forward on full-layout state lists (see full_state).
        store: 12 snapshot histories (background E x3, curl H x3, scattered
        E x3, scattered curl x3; None entries are not stored) or None."""
        fn, F = self._fn("born_forward_store", pb.dtype, pb.stencil)
        P, I = c_void_p, c_int64
        pml = (c_int64 * 6)(*pb.pml)
        fn.argtypes = ([P] * 7 + [P] * 4 + [P, P, P, P, P] + [F, F, F] + [I] * 8 + [P] +
                       [c_int] * 5 + [P, I, c_int])
        prof = _ptr_array([pb.profiles[n].cpu() for n in PROFILES_3D])
        st = (c_void_p * 12)(*[_p(t) if t is not None else None for t in store]) if store else None
        fn(_p(pb.ca), _p(pb.cb), _p(pb.cq.cpu()), _p(dca), _p(dcb), _p(f0), _p(df),
           _ptr_array(fields), _ptr_array(mem), _ptr_array(dfields), _ptr_array(dmem), _p(r),
           _p(bg_r), prof, _p(pb.sources_i.cpu()), _p(pb.receivers_i.cpu()), pb.rdz, pb.rdy,
           pb.rdx, pb.nt, pb.n_shots, pb.nz, pb.ny, pb.nx, pb.n_src, pb.n_rec, 0, pml,
           int(pb.batched), int(pb.batched), int(pb.batched), pb.src_comp, pb.rec_comp, st, k,
           fmt)

    def backward(self, pb, ca, cb, grad_r, store, *, k=1, fmt=0, need_ca=True, need_cb=True,
                 need_f=True, start_t=None, nt=None, lam=None, grads=None, eps_sigma=False):
        """Returns (grad_ca, grad_cb, grad_f, lam_fields, lam_mem[, grad_eps, grad_sigma])."""
        S, nz, ny, nx = pb.n_shots, pb.nz, pb.ny, pb.nx
        nt_all = pb.nt
        nt = nt_all if nt is None else nt
        start_t = nt_all if start_t is None else start_t
        dt = pb.dtype
        if lam is None:
            lam = ([torch.zeros((S, nz, ny, nx), dtype=dt) for _ in range(6)],
                   [torch.zeros((S, nz, ny, nx), dtype=dt) for _ in range(12)])
        mshape = (S, nz, ny, nx) if pb.batched else (nz, ny, nx)
        if grads is None:
            grads = (torch.zeros(mshape, dtype=dt), torch.zeros(mshape, dtype=dt),
                     torch.zeros((nt_all, S, max(pb.n_src, 1)), dtype=dt))
        gca, gcb, gf = grads
        geps = torch.zeros(mshape, dtype=dt) if eps_sigma else None
        gsig = torch.zeros(mshape, dtype=dt) if eps_sigma else None
        fn, F = self._fn("backward", dt, pb.stencil)
        P, I = c_void_p, c_int64
        fn.argtypes = [P, P, P, P, P, P, P, P, P, P, P, P, F, P, P, P, F, F, F, I, I, I, I, I,
                       I, I, I, c_int, I, P, c_int, c_int, c_int, c_int, c_int, c_int, c_int]
        prof = _ptr_array([pb.profiles[n].cpu() for n in PROFILES_3D])
        pml = (c_int64 * 6)(*pb.pml)
        fn(_p(ca), _p(cb), _p(pb.cq.cpu()), _p(grad_r), _ptr_array(lam[0]), _ptr_array(lam[1]),
           _ptr_array(list(store)), _p(gf) if need_f and pb.n_src else None,
           _p(gca) if need_ca else None, _p(gcb) if need_cb else None, _p(geps), _p(gsig),
           pb.dt, prof, _p(pb.sources_i.cpu()), _p(pb.receivers_i.cpu()), pb.rdz, pb.rdy,
           pb.rdx, nt, S, nz, ny, nx, pb.n_src, pb.n_rec, k, fmt, start_t, pml,
           int(pb.batched), int(pb.batched), int(pb.batched), pb.src_comp, pb.rec_comp,
           int(need_ca), int(need_cb))
        out = (gca, gcb, gf, lam[0], lam[1])
        return out + ((geps, gsig) if eps_sigma else ())


def _oracle3d_born_bggrad(o, pb, dca, dcb, grad_r, store, dstore, k=1, fmt=0):
    """3-D second-order Born adjoint on the oracle (full-layout state);
    returns grad_ca, grad_cb, grad_dca, grad_dcb (model-shaped), grad_f0 and
    grad_df ([nt, S, n_src])."""
    S, nz, ny, nx, dt = pb.n_shots, pb.nz, pb.ny, pb.nx, pb.dtype
    z = lambda *s: torch.zeros(s, dtype=dt)  # noqa: E731
    L = [z(S, nz, ny, nx) for _ in range(6)]
    lm = [z(S, nz, ny, nx) for _ in range(12)]
    E = [z(S, nz, ny, nx) for _ in range(6)]
    em = [z(S, nz, ny, nx) for _ in range(12)]
    mshape = (S, nz, ny, nx) if pb.batched else (nz, ny, nx)
    g = [z(*mshape) for _ in range(4)]
    gf0, gdf = z(pb.nt, S, max(pb.n_src, 1)), z(pb.nt, S, max(pb.n_src, 1))
    fn, F = o._fn("born_bggrad", dt, pb.stencil)
    P, I = c_void_p, c_int64
    fn.argtypes = ([P] * 6 + [P] * 4 + [P, P] + [P] * 6 + [P, P, P] + [F, F, F] + [I] * 8
                   + [c_int, I, P] + [c_int] * 5)
    prof = _ptr_array([pb.profiles[n].cpu() for n in PROFILES_3D])
    pml = (c_int64 * 6)(*pb.pml)
    fn(_p(pb.ca), _p(pb.cb), _p(pb.cq.cpu()), _p(dca), _p(dcb), _p(grad_r), _ptr_array(L),
       _ptr_array(lm), _ptr_array(E), _ptr_array(em), _ptr_array(list(store)),
       _ptr_array(list(dstore)), _p(gf0), _p(gdf), *[_p(t) for t in g], prof,
       _p(pb.sources_i.cpu()), _p(pb.receivers_i.cpu()), pb.rdz, pb.rdy, pb.rdx, pb.nt, S, nz,
       ny, nx, pb.n_src, pb.n_rec, k, fmt, pb.nt, pml, int(pb.batched), int(pb.batched),
       int(pb.batched), pb.src_comp, pb.rec_comp)
    return (*g, gf0, gdf)


class OracleEM3D(torch.autograd.Function):
    """Autograd node over (ca, cb, f) backed by the 3-D C oracle (CPU)."""

    @staticmethod
    def forward(ctx, ca, cb, f, pb, oracle):
        S, nz, ny, nx, nt = pb.n_shots, pb.nz, pb.ny, pb.nx, pb.nt
        r = torch.zeros((nt, S, pb.n_rec), dtype=pb.dtype)
        store = [torch.zeros((nt, S, nz, ny, nx), dtype=pb.dtype) for _ in range(6)]
        fields, mem = Oracle3D.full_state(pb)
        oracle.forward(pb, ca.detach(), cb.detach(), f.detach(), r, fields, mem, store=store)
        ctx.save_for_backward(ca, cb)
        ctx.pb, ctx.oracle, ctx.store = pb, oracle, store
        return r

    @staticmethod
    def backward(ctx, grad_r):
        ca, cb = ctx.saved_tensors
        pb = ctx.pb
        gca, gcb, gf, _, _ = ctx.oracle.backward(pb, ca.detach(), cb.detach(),
                                                 grad_r.contiguous(), ctx.store)
        if not pb.batched:
            gca, gcb = gca.unsqueeze(0), gcb.unsqueeze(0)
        return gca, gcb, (gf.reshape(-1) if pb.n_src else None), None, None


class RefCPU3D:
    """The reference's 3-D CPU backend (maxwell_3d_2_{dtype}_forward_cpu);
    memories are full arrays on this path."""

    def __init__(self, path: pathlib.Path = REF_SO):
        self.lib = ctypes.CDLL(str(path))

    def forward(self, pb, ca, cb, f, r, fields, mem, n_threads=0):
        import sys

        sys.path.insert(0, str(REPO / "tide-gpr_b200"))
        from tide_b200 import _native as nat

        sfx = "float" if pb.dtype == torch.float32 else "double"
        fn = getattr(self.lib, f"maxwell_3d_{pb.stencil}_{sfx}_forward_cpu")
        fn.argtypes = nat.argtypes("maxwell_3d_forward", sfx)
        fn.restype = None
        b = pb.batched
        fn(_p(ca), _p(cb), _p(pb.cq.cpu()), _p(f), *[_p(t) for t in fields],
           *[_p(t) for t in mem], *([0] * 9), _p(r), 0,
           *[_p(pb.profiles[n].cpu()) for n in PROFILES_3D], _p(pb.sources_i.cpu()),
           _p(pb.receivers_i.cpu()), pb.rdz, pb.rdy, pb.rdx, pb.dt, pb.nt, pb.n_shots, pb.nz,
           pb.ny, pb.nx, pb.n_src, pb.n_rec, 1, False, b, b, b, 0, *pb.pml, pb.src_comp,
           pb.rec_comp, n_threads, 0, 0, 0)

    def born_forward(self, pb, dca, dcb, f0, df, fields, mem, dfields, dmem, r, bg_r,
                     n_threads=0):
        import sys

        sys.path.insert(0, str(REPO / "tide-gpr_b200"))
        from tide_b200 import _native as nat

        sfx = "float" if pb.dtype == torch.float32 else "double"
        fn = getattr(self.lib, f"maxwell_3d_{pb.stencil}_{sfx}_born_forward_cpu")
        fn.argtypes = nat.argtypes("maxwell_3d_born_forward", sfx)
        fn.restype = None
        b = pb.batched
        fn(_p(pb.ca), _p(pb.cb), _p(pb.cq.cpu()), _p(dca), _p(dcb), _p(f0), _p(df),
           *[_p(t) for t in fields], *[_p(t) for t in mem], *[_p(t) for t in dfields],
           *[_p(t) for t in dmem], _p(r), _p(bg_r),
           *[_p(pb.profiles[n].cpu()) for n in PROFILES_3D], _p(pb.sources_i.cpu()),
           _p(pb.receivers_i.cpu()), pb.rdz, pb.rdy, pb.rdx, pb.dt, pb.nt, pb.n_shots, pb.nz,
           pb.ny, pb.nx, pb.n_src, pb.n_rec, 1, b, b, b, 0, *pb.pml, pb.src_comp, pb.rec_comp,
           n_threads, 0, 0, 0)


class OracleDebye:
    """Debye-medium forward with storage and exact adjoint of the C oracle,
    driven with the product's argument struct (tide_b200.debye.CDebye) on
    host tensors; a problem prepared on the CPU by prepare_tm2d."""

    def __init__(self):
        if not ORACLE_SO.exists():
            build_oracle()
        self.lib = ctypes.CDLL(str(ORACLE_SO))

    def _call(self, name, dtype, A):
        from tide_b200.debye import CDebye

        sfx = "float" if dtype == torch.float32 else "double"
        fn = getattr(self.lib, f"tide_oracle_tm_debye_{name}_{sfx}")
        fn.argtypes = [ctypes.POINTER(CDebye)]
        fn.restype = None
        fn(ctypes.byref(A))

    def forward(self, pb, ca, cb, f, r, a, b, cp, snaps, start_t=0, nt=None, k=1, fmt=0, q0=0):
        from tide_b200 import debye as dby

        A = dby.make_args(pb, ca, cb, a, b, cp, f=f, r=r, start_t=start_t, nt=nt, k=k, fmt=fmt,
                          q0=q0, stream=0)
        A.pol = _p(dby.polarization(pb))
        snaps.bind(A)
        self._call("forward_with_storage", pb.dtype, A)

    def backward(self, pb, ca, cb, a, b, cp, grad_r, st, snaps, start_t, nt, k=1, fmt=0, q0=0):
        from tide_b200 import debye as dby

        A = dby.make_args(pb, ca, cb, a, b, cp, start_t=start_t, nt=nt, k=k, fmt=fmt, q0=q0,
                          stream=0)
        A.grad_r = _p(grad_r)
        snaps.bind(A)
        st.bind(A)
        self._call("backward", pb.dtype, A)
