"""Gradients through Debye media (2-D TM), on the native Debye adjoint.

The reference differentiates Debye media only in Python, with torch autograd
through its time loop (src/tide/maxwell/tm2d_python.py:440-503); its native
backends run them forward only.  Here the forward records, per stored step,
Ey, curl H, the polarisation P (and E^{t+1} + E^t when the b coefficients
need a gradient), and the exact discrete adjoint of the Debye step
(include/tide_b200_debye.h) returns the gradients of ca, cb, the source
amplitudes and the pole coefficients a, b, cp; torch autograd chains them to
epsilon, sigma, delta_epsilon and tau through the coefficient formulas.

Storage: "device" keeps the whole history in HBM; "checkpoint" keeps the full
state (fields, CPML memories, polarisation) every storage_chunk_steps steps
and recomputes each segment's snapshots in the adjoint, last segment first
(the form for histories larger than HBM).
"""

from __future__ import annotations

import ctypes
from ctypes import c_double, c_int64, c_void_p

import torch

from . import _native as nat
from . import storage as stg

_P = c_void_p


class CDebye(ctypes.Structure):
    """TideTMDebye (include/tide_b200_debye.h)."""

    _fields_ = [
        *[(n, c_int64) for n in ("stencil", "n_shots", "ny", "nx", "nt", "start_t", "n_src",
                                 "n_rec", "n_poles", "step_ratio", "storage_format", "q0",
                                 "pml_y0", "pml_x0", "pml_y1", "pml_x1")],
        ("rdy", c_double), ("rdx", c_double),
        ("profiles", _P * 12),
        *[(n, _P) for n in ("ca", "cb", "cq", "a", "b", "cp")],
        ("fields", _P * 7), ("pol", _P), ("f", _P), ("r", _P),
        ("sources_i", _P), ("receivers_i", _P),
        *[(n, _P) for n in ("ey_store", "curl_store", "pol_store", "esum_store", "grad_r")],
        ("lam", _P * 7), ("lam_pol", _P), ("scratch", _P), ("grad_f", _P),
        *[(n, _P) for n in ("grad_ca", "grad_cb", "grad_cp", "grad_a", "grad_b")],
        ("device", c_int64), ("stream", _P),
    ]


PROFILE_ORDER = ("ay", "by", "ayh", "byh", "ax", "bx", "axh", "bxh", "ky", "kyh", "kx", "kxh")
_BOUND = False


def _fn(name: str, dtype: torch.dtype):
    global _BOUND
    lib = nat.load()
    if not _BOUND:
        for pas in ("forward_with_storage", "backward"):
            for d in ("float", "double"):
                f = getattr(lib, f"tide_b200_tm_debye_{pas}_{d}")
                f.argtypes = [ctypes.POINTER(CDebye)]
                f.restype = None
        _BOUND = True
    return getattr(lib, f"tide_b200_tm_debye_{name}_{nat.DTYPES[dtype]}")


def make_args(pb, ca, cb, a, b, cp, *, f=None, r=None, start_t=0, nt=None, k=1, fmt=0,
              q0=0, stream=None) -> CDebye:
    """Argument struct of one call (pointers of the given tensors; unset
    buffers are null).  Works for device tensors (the library) and host
    tensors (the CPU oracle)."""
    A = CDebye()
    A.stencil, A.n_shots, A.ny, A.nx = pb.stencil, pb.n_shots, pb.ny, pb.nx
    A.nt = pb.nt if nt is None else nt
    A.start_t, A.n_src, A.n_rec = start_t, pb.n_src, pb.n_rec
    A.n_poles, A.step_ratio, A.storage_format, A.q0 = int(pb.debye["n_poles"]), k, fmt, q0
    A.pml_y0, A.pml_x0, A.pml_y1, A.pml_x1 = pb.pml_y0, pb.pml_x0, pb.pml_y1, pb.pml_x1
    A.rdy, A.rdx = pb.rdy, pb.rdx
    for i, n in enumerate(PROFILE_ORDER):
        A.profiles[i] = nat.ptr(pb.profiles[n])
    A.ca, A.cb, A.cq = nat.ptr(ca), nat.ptr(cb), nat.ptr(pb.cq)
    A.a, A.b, A.cp = nat.ptr(a), nat.ptr(b), nat.ptr(cp)
    for i, t in enumerate(pb.fields):
        A.fields[i] = nat.ptr(t)
    A.f, A.r = nat.ptr(f), nat.ptr(r)
    A.sources_i, A.receivers_i = nat.ptr(pb.sources_i), nat.ptr(pb.receivers_i)
    dev = pb.device
    A.device = (dev.index or 0) if dev.type == "cuda" else 0
    if stream is not None:
        A.stream = int(stream)
    elif dev.type == "cuda":
        A.stream = int(torch.cuda.current_stream(dev).cuda_stream)
    return A


def polarization(pb) -> torch.Tensor:
    """The problem's polarisation state [S, n_poles, ny, nx] (zero at first use)."""
    d = pb.debye
    return d.setdefault(
        "polarization",
        torch.zeros((pb.n_shots, d["n_poles"], pb.ny, pb.nx), device=pb.device, dtype=pb.dtype),
    )


class Snapshots:
    """Stored steps of a Debye forward (slots q0, q0 + 1, ...)."""

    def __init__(self, n_slots, pb, sdtype, need_ca, need_cb, need_pol, need_esum):
        S, ny, nx, P = pb.n_shots, pb.ny, pb.nx, int(pb.debye["n_poles"])
        e = lambda *s: torch.empty(s, device=pb.device, dtype=sdtype)  # noqa: E731
        self.ey = e(n_slots, S, ny, nx) if need_ca else None
        self.curl = e(n_slots, S, ny, nx) if need_cb else None
        self.pol = e(n_slots, S, P, ny, nx) if need_pol else None
        self.esum = e(n_slots, S, ny, nx) if need_esum else None

    def bind(self, A: CDebye) -> None:
        A.ey_store, A.curl_store = nat.ptr(self.ey), nat.ptr(self.curl)
        A.pol_store, A.esum_store = nat.ptr(self.pol), nat.ptr(self.esum)


def native_forward_storage(pb, ca, cb, f, r, a, b, cp, snaps: Snapshots, start_t, nt, k, fmt,
                           q0=0) -> None:
    A = make_args(pb, ca, cb, a, b, cp, f=f, r=r, start_t=start_t, nt=nt, k=k, fmt=fmt, q0=q0)
    A.pol = nat.ptr(polarization(pb))
    snaps.bind(A)
    _fn("forward_with_storage", pb.dtype)(ctypes.byref(A))
    nat.check("maxwell_tm Debye forward_with_storage")


class AdjointState:
    """Adjoint fields, polarisation adjoint, scratch and gradient accumulators."""

    def __init__(self, pb, need):
        S, ny, nx, P = pb.n_shots, pb.ny, pb.nx, int(pb.debye["n_poles"])
        dev, dt = pb.device, pb.dtype
        z = lambda *s: torch.zeros(s, device=dev, dtype=dt)  # noqa: E731
        self.lam = [z(S, ny, nx) for _ in range(7)]
        self.lam_pol = z(S, P, ny, nx)
        self.scratch = torch.empty((5, S, ny, nx), device=dev, dtype=dt)
        self.grad_f = z(pb.nt, S, pb.n_src) if pb.n_src > 0 else None
        self.g = {n: (z(ny, nx) if n in ("ca", "cb") else z(P, ny, nx)) if need[n] else None
                  for n in ("ca", "cb", "cp", "a", "b")}

    def bind(self, A: CDebye) -> None:
        for i, t in enumerate(self.lam):
            A.lam[i] = nat.ptr(t)
        A.lam_pol, A.scratch, A.grad_f = (nat.ptr(self.lam_pol), nat.ptr(self.scratch),
                                          nat.ptr(self.grad_f))
        A.grad_ca, A.grad_cb = nat.ptr(self.g["ca"]), nat.ptr(self.g["cb"])
        A.grad_cp, A.grad_a, A.grad_b = (nat.ptr(self.g["cp"]), nat.ptr(self.g["a"]),
                                         nat.ptr(self.g["b"]))


def native_backward(pb, ca, cb, a, b, cp, grad_r, st: AdjointState, snaps: Snapshots, start_t,
                    nt, k, fmt, q0=0) -> None:
    A = make_args(pb, ca, cb, a, b, cp, start_t=start_t, nt=nt, k=k, fmt=fmt, q0=q0)
    A.grad_r = nat.ptr(grad_r)
    snaps.bind(A)
    st.bind(A)
    _fn("backward", pb.dtype)(ctypes.byref(A))
    nat.check("maxwell_tm Debye backward")


def _grad_r(pb, grad_r):
    if grad_r is None or grad_r.numel() == 0:
        return torch.zeros((pb.nt, pb.n_shots, pb.n_rec), device=pb.device, dtype=pb.dtype)
    return grad_r.contiguous()


class DebyePropagate(torch.autograd.Function):
    """Autograd node over (ca, cb, f, a, b, cp) of a Debye-medium propagation."""

    @staticmethod
    def forward(ctx, ca, cb, f, a, b, cp, pb, opts):
        from .tm2d import checkpoint_steps

        nt, S = pb.nt, pb.n_shots
        r = torch.zeros((nt, S, pb.n_rec), device=pb.device, dtype=pb.dtype)
        need = {"ca": ca.requires_grad, "cb": cb.requires_grad, "cp": cp.requires_grad,
                "a": a.requires_grad, "b": b.requires_grad}
        k = pb.grad_interval
        fmt, sdtype = stg.compression_format(opts.get("storage_compression", False), pb.dtype)
        flags = (need["ca"], need["cb"], need["cp"] or need["a"], need["b"])
        mode = str(opts.get("storage_mode", "device")).lower()
        if mode == "auto":
            mode = "device"
        if mode not in ("device", "checkpoint"):
            raise NotImplementedError(
                "Debye gradients support storage_mode='device' or 'checkpoint'")
        polarization(pb)
        if mode == "device":
            snaps = Snapshots(-(-nt // k), pb, sdtype, *flags)
            native_forward_storage(pb, ca, cb, f, r, a, b, cp, snaps, 0, nt, k, fmt)
            ctx.plan = ("device", snaps)
        else:
            seg = checkpoint_steps(nt, k, opts.get("storage_chunk_steps"))
            ckpts = []
            dummy = Snapshots(0, pb, sdtype, False, False, False, False)
            for s0 in range(0, nt, seg):
                ckpts.append([t.clone() for t in pb.fields] + [polarization(pb).clone()])
                native_forward_storage(pb, ca, cb, f, r, a, b, cp, dummy, s0,
                                       min(seg, nt - s0), k, fmt)
            ctx.plan = ("checkpoint", (seg, ckpts, sdtype, fmt))
        ctx.pb, ctx.opts, ctx.need, ctx.flags, ctx.k, ctx.fmt = pb, opts, need, flags, k, fmt
        ctx.f = f.detach()
        ctx.save_for_backward(ca, cb, a, b, cp)
        for t in pb.fields:
            ctx.mark_non_differentiable(t)
        return (*pb.fields, r)

    @staticmethod
    def backward(ctx, *grads):
        pb = ctx.pb
        ca, cb, a, b, cp = ctx.saved_tensors
        grad_r = _grad_r(pb, grads[7])
        st = AdjointState(pb, ctx.need)
        kind, data = ctx.plan
        k, fmt = ctx.k, ctx.fmt
        if kind == "device":
            native_backward(pb, ca, cb, a, b, cp, grad_r, st, data, pb.nt, pb.nt, k, fmt)
        else:
            seg, ckpts, sdtype, fmt = data
            final = [t.clone() for t in pb.fields] + [polarization(pb).clone()]
            snaps = Snapshots(-(-seg // k), pb, sdtype, *ctx.flags)
            r_seg = torch.zeros((pb.nt, pb.n_shots, pb.n_rec), device=pb.device, dtype=pb.dtype)
            state = list(pb.fields) + [polarization(pb)]
            for idx in range(len(ckpts) - 1, -1, -1):
                s0 = idx * seg
                n = min(seg, pb.nt - s0)
                for dst, src in zip(state, ckpts[idx]):
                    dst.copy_(src)
                native_forward_storage(pb, ca, cb, ctx.f, r_seg, a, b, cp, snaps, s0, n, k, fmt,
                                       q0=s0 // k)
                native_backward(pb, ca, cb, a, b, cp, grad_r, st, snaps, s0 + n, n, k, fmt,
                                q0=s0 // k)
            for dst, src in zip(state, final):
                dst.copy_(src)
        if not ctx.opts.get("retain_history"):
            ctx.plan = None  # release the history (a linearization keeps it)
        g = st.g
        gf = st.grad_f.reshape(-1) if (st.grad_f is not None and ctx.needs_input_grad[2]) else None
        return (g["ca"].unsqueeze(0) if g["ca"] is not None else None,
                g["cb"].unsqueeze(0) if g["cb"] is not None else None,
                gf, g["a"], g["b"], g["cp"], None, None)


def propagate_debye(pb, opts):
    """Run a Debye-medium problem whose coefficients need gradients."""
    d = pb.debye
    if pb.batched:
        raise NotImplementedError("Debye gradients need an unbatched model")
    out = DebyePropagate.apply(pb.ca, pb.cb, pb.f, d["a"], d["b"], d["cp"], pb, opts)
    return list(out[:7]), out[7]


__all__ = ["AdjointState", "CDebye", "DebyePropagate", "Snapshots", "make_args",
           "native_backward", "native_forward_storage", "polarization", "propagate_debye"]
