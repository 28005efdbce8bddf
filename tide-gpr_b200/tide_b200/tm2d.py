"""2-D TM Maxwell propagation on the B200 native library.

Host-side mirror of the reference's TM2D native adapter
(src/tide/maxwell/tm2d_cuda.py:29-826) and autograd function
(src/tide/maxwell/tm2d_autograd.py:26-873):

1. ``prepare_tm2d`` pads the model (replicate) by fd_pad + CPML width with the
   asymmetric staggered padding [p, p-1, p, p-1], compiles ca/cb/cq, flattens
   source/receiver positions into the padded grid, pre-scales the source as
   f = amp * cb[src] * (-1 / (dy dx)) laid out [nt, S, n_src], builds the 12
   CPML profiles and the strip bounds pml_y0/y1/x0/x1.
2. ``TMPropagate`` (a torch.autograd.Function over ca, cb, f) runs the native
   forward, storing Ey^t and curl H^t every k steps when ca/cb need
   gradients, and the native exact adjoint in backward; torch autograd then
   carries dJ/dca, dJ/dcb, dJ/df back to epsilon, sigma and the amplitudes
   through the coefficient formulas, the replicate padding and the source
   pre-scale, exactly as in the reference.

Everything runs on CUDA through libtide_b200.so; CPU tensors are rejected.
"""

from __future__ import annotations

from collections.abc import Callable, Sequence
from dataclasses import dataclass, field
from typing import Any

import torch

from . import _native as nat
from . import physics as ph
from . import storage as stg


@dataclass
class CallbackState:
    """State handed to forward/backward observers (src/tide/callbacks.py)."""

    dt: float
    step: int
    nt: int
    wavefields: dict[str, torch.Tensor]
    models: dict[str, torch.Tensor]
    gradients: dict[str, torch.Tensor] | None
    fd_pad: list[int]
    pml_width: list[int]
    is_backward: bool


Callback = Callable[[CallbackState], None]


@dataclass
class TMProblem:
    """Padded, compiled inputs of one TM2D propagation (all on one CUDA device)."""

    ca: torch.Tensor
    cb: torch.Tensor
    cq: torch.Tensor
    f: torch.Tensor  # [nt * S * n_src] (empty if no sources)
    profiles: dict[str, torch.Tensor]
    sources_i: torch.Tensor
    receivers_i: torch.Tensor
    rdy: float
    rdx: float
    dt: float
    nt: int
    n_shots: int
    ny: int
    nx: int
    n_src: int
    n_rec: int
    grad_interval: int
    stencil: int
    batched: bool
    pml_y0: int
    pml_x0: int
    pml_y1: int
    pml_x1: int
    fd_pad: list[int]
    pml_width: list[int]
    fields: list[torch.Tensor]  # Ey, Hx, Hz, m_Ey_x, m_Ey_z, m_Hx_z, m_Hz_x
    debye: dict | None = None
    models: dict[str, torch.Tensor] = field(default_factory=dict)

    @property
    def device(self) -> torch.device:
        return self.ca.device

    @property
    def dtype(self) -> torch.dtype:
        return self.ca.dtype

    def crop(self, t: torch.Tensor) -> torch.Tensor:
        """Remove the finite-difference padding (keeps the CPML layer)."""
        p = self.fd_pad
        return t[:, p[0] : self.ny - p[1] if p[1] > 0 else None, p[2] : self.nx - p[3] if p[3] > 0 else None]


def prepare_tm2d(
    epsilon: torch.Tensor,
    sigma: torch.Tensor,
    mu: torch.Tensor,
    grid_spacing: float | Sequence[float],
    dt: float,
    source_amplitude: torch.Tensor | None,
    source_location: torch.Tensor | None,
    receiver_location: torch.Tensor | None,
    *,
    stencil: int = 2,
    pml_width: int | Sequence[int] = 20,
    initial_state: Sequence[torch.Tensor | None] | None = None,
    nt: int | None = None,
    model_gradient_sampling_interval: int = 1,
    dispersion: ph.DebyeDispersion | None = None,
) -> TMProblem:
    """Build the padded native inputs (src/tide/maxwell/tm2d_cuda.py:65-360).

    Pure tensor preparation: it runs on any device (the test suite prepares on
    the CPU so the CUDA path and the oracle see bit-identical inputs); the
    propagation itself only runs on CUDA.
    """
    if epsilon.ndim not in (2, 3):
        raise RuntimeError("epsilon must be 2D or batched 3D")
    if sigma.shape != epsilon.shape or mu.shape != epsilon.shape:
        raise RuntimeError("sigma and mu must have the same shape as epsilon")
    if stencil not in (2, 4, 6, 8):
        raise ValueError("stencil must be one of 2, 4, 6, 8")
    device, dtype = epsilon.device, epsilon.dtype
    batched = epsilon.ndim == 3
    model_ny, model_nx = epsilon.shape[-2:]
    dy, dx = ph.normalize_spacing_2d(grid_spacing)
    widths = ph.normalize_pml_width_2d(pml_width)
    if nt is None:
        if source_amplitude is None:
            raise ValueError("Either nt or source_amplitude must be provided")
        nt = int(source_amplitude.shape[-1])
    nt = int(nt)
    k = max(1, int(model_gradient_sampling_interval))
    if nt > 0:
        k = min(k, nt)
    if source_amplitude is not None and source_amplitude.numel() > 0:
        n_shots = int(source_amplitude.shape[0])
    elif source_location is not None and source_location.numel() > 0:
        n_shots = int(source_location.shape[0])
    elif receiver_location is not None and receiver_location.numel() > 0:
        n_shots = int(receiver_location.shape[0])
    else:
        n_shots = 1
    if batched and int(epsilon.shape[0]) != n_shots:
        raise RuntimeError("Batched model count must match the shot count.")

    p = stencil // 2
    fd_pad = [p, p - 1, p, p - 1]
    total = [a + b for a, b in zip(fd_pad, widths)]
    ny = model_ny + total[0] + total[1]
    nx = model_nx + total[2] + total[3]

    eps_p = ph.pad_model(epsilon, total)
    sig_p = ph.pad_model(sigma, total)
    mu_p = ph.pad_model(mu, total)
    disp_p = None
    if dispersion is not None:
        def padp(v):
            t = torch.as_tensor(v, device=device, dtype=dtype)
            if t.ndim == 0:
                return t
            if t.ndim == 2:
                return ph.pad_model(t, total)
            return ph.pad_model(t, total)  # [n_poles, ny, nx]
        disp_p = ph.DebyeDispersion(padp(dispersion.delta_epsilon), padp(dispersion.tau))
    mat = ph.compile_material_coefficients(eps_p, sig_p, mu_p, dt, dispersion=disp_p)
    ca, cb, cq = mat["ca"], mat["cb"], mat["cq"]
    if not batched:
        ca, cb, cq = ca[None], cb[None], cq[None]
    ca, cb, cq = ca.contiguous(), cb.contiguous(), cq.contiguous()

    N = ny * nx
    if source_location is not None and source_location.numel() > 0:
        sy = source_location[..., 0] + total[0]
        sx = source_location[..., 1] + total[2]
        sources_i = (sy * nx + sx).long().contiguous().to(device)
        n_src = int(source_location.shape[1])
    else:
        sources_i = torch.empty(0, device=device, dtype=torch.long)
        n_src = 0
    if receiver_location is not None and receiver_location.numel() > 0:
        ry = receiver_location[..., 0] + total[0]
        rx = receiver_location[..., 1] + total[2]
        receivers_i = (ry * nx + rx).long().contiguous().to(device)
        n_rec = int(receiver_location.shape[1])
    else:
        receivers_i = torch.empty(0, device=device, dtype=torch.long)
        n_rec = 0

    # Source pre-scale (src/tide/maxwell/tm2d_helpers.py:48-82).
    coeff = -1.0 / (dx * dy)
    if n_src > 0 and source_amplitude is not None and source_amplitude.numel() > 0:
        cb_flat = cb.reshape(n_shots, N) if batched else cb.expand(n_shots, -1, -1).reshape(n_shots, N)
        cb_at_src = cb_flat.gather(1, sources_i)
        src = source_amplitude.permute(2, 0, 1).contiguous().to(dtype)
        src = src * cb_at_src.to(dtype).unsqueeze(0)
        src = src * coeff
        f = src.reshape(nt * n_shots * n_src).contiguous()
    else:
        f = torch.empty(0, device=device, dtype=dtype)

    init = list(initial_state) if initial_state is not None else [None] * 7
    size = (n_shots, ny, nx)
    fields = [ph.pad_field(init[i], fd_pad, size, device, dtype) for i in range(7)]
    for wf, dim in zip(fields[3:], (1, 0, 0, 1)):
        ph.zero_interior(wf, fd_pad, widths, dim)

    prof = ph.set_pml_profiles(widths, fd_pad, dt, [dy, dx], dtype, device, ny, nx)
    debye = None
    if mat["has_dispersion"]:
        d = mat["debye"]
        debye = {
            "a": d["a"].contiguous(),
            "b": d["b"].contiguous(),
            "cp": d["cp"].contiguous(),
            "n_poles": d["n_poles"],
        }
    return TMProblem(
        ca=ca, cb=cb, cq=cq, f=f, profiles=prof, sources_i=sources_i, receivers_i=receivers_i,
        rdy=1.0 / dy, rdx=1.0 / dx, dt=dt, nt=nt, n_shots=n_shots, ny=ny, nx=nx,
        n_src=n_src, n_rec=n_rec, grad_interval=k, stencil=stencil, batched=batched,
        pml_y0=fd_pad[0] + widths[0], pml_x0=fd_pad[2] + widths[2],
        pml_y1=ny - fd_pad[1] - widths[1], pml_x1=nx - fd_pad[3] - widths[3],
        fd_pad=fd_pad, pml_width=widths, fields=fields, debye=debye,
        models={"epsilon": eps_p, "sigma": sig_p, "mu": mu_p, "ca": ca, "cb": cb, "cq": cq},
    )


_PROFILE_ORDER = ("ay", "by", "ayh", "byh", "ax", "bx", "axh", "bxh", "ky", "kyh", "kx", "kxh")


def _profile_ptrs(pb: TMProblem) -> list[int]:
    return [nat.ptr(pb.profiles[n]) for n in _PROFILE_ORDER]


def _stream_handle(device: torch.device) -> int:
    return int(torch.cuda.current_stream(device).cuda_stream)


def native_forward(
    pb: TMProblem,
    ca: torch.Tensor,
    cb: torch.Tensor,
    f: torch.Tensor,
    r: torch.Tensor,
    start_t: int,
    nt: int,
) -> None:
    """One forward call without storage (src/tide/csrc/tm2d/maxwell_tm_cuda_inst.cu:1281)."""
    fn = nat.get_backend_function("maxwell_tm", "forward", pb.stencil, pb.dtype, pb.device)
    ey, hx, hz, mex, mez, mhx, mhz = pb.fields
    d = pb.debye
    n_poles = 0
    dba = dbb = dbc = pol = None
    if d is not None:
        n_poles = d["n_poles"]
        dba, dbb, dbc = d["a"], d["b"], d["cp"]
        pol = d.setdefault(
            "polarization",
            torch.zeros((pb.n_shots, n_poles, pb.ny, pb.nx), device=pb.device, dtype=pb.dtype),
        )
    fn(
        nat.ptr(ca), nat.ptr(cb), nat.ptr(pb.cq), nat.ptr(f),
        nat.ptr(ey), nat.ptr(hx), nat.ptr(hz), nat.ptr(mex), nat.ptr(mez), nat.ptr(mhx), nat.ptr(mhz),
        nat.ptr(dba), nat.ptr(dbb), nat.ptr(dbc), nat.ptr(pol), 0, nat.ptr(r), n_poles,
        *_profile_ptrs(pb), nat.ptr(pb.sources_i), nat.ptr(pb.receivers_i),
        pb.rdy, pb.rdx, pb.dt, nt, pb.n_shots, pb.ny, pb.nx, pb.n_src, pb.n_rec, 1,
        d is not None, pb.batched, pb.batched, pb.batched, start_t,
        pb.pml_y0, pb.pml_x0, pb.pml_y1, pb.pml_x1, 0, pb.device.index or 0,
        _stream_handle(pb.device),
    )
    nat.check("maxwell_tm forward")


class TMPropagate(torch.autograd.Function):
    """Autograd node over (ca, cb, f) driving the native forward and adjoint."""

    @staticmethod
    def forward(ctx, ca, cb, f, pb: TMProblem, opts: dict):
        device, dtype = pb.device, pb.dtype
        nt, S = pb.nt, pb.n_shots
        r = (
            torch.zeros((nt, S, pb.n_rec), device=device, dtype=dtype)
            if pb.n_rec > 0
            else torch.empty(0, device=device, dtype=dtype)
        )
        need_ca, need_cb = ca.requires_grad, cb.requires_grad
        need_f = f.requires_grad
        fwd_cb: Callback | None = opts.get("forward_callback")
        freq = int(opts.get("callback_frequency", 1)) if fwd_cb else 0
        k = pb.grad_interval
        snaps = None
        ckpt = None
        if (need_ca or need_cb) and str(opts.get("storage_mode", "device")).lower() == "checkpoint":
            if pb.debye is not None:
                raise NotImplementedError(
                    "Debye media: gradients run through tide_b200.debye (propagate routes "
                    "them there)"
                )
            seg_len = checkpoint_steps(nt, k, opts.get("storage_chunk_steps"))
            ckpt = (seg_len, _run_forward_checkpointed(pb, ca, cb, f, r, seg_len, fwd_cb,
                                                       max(1, freq)))
        elif need_ca or need_cb:
            fmt, sdtype = stg.compression_format(opts.get("storage_compression", False), dtype)
            n_store = (nt + k - 1) // k
            mode = stg.resolve_mode(
                opts.get("storage_mode", "device"), device=device, n_store=n_store, n_shots=S,
                ny=pb.ny, nx=pb.nx, itemsize=sdtype.itemsize,
                n_arrays=int(need_ca) + int(need_cb),
                bytes_limit_device=opts.get("storage_bytes_limit_device"),
                bytes_limit_host=opts.get("storage_bytes_limit_host"),
            )
            if mode == stg.STORAGE_NONE:
                raise ValueError("storage_mode='none' is incompatible with model gradients")
            snaps = stg.allocate(mode, sdtype, fmt, n_store, S, pb.ny, pb.nx, device, need_ca,
                                 need_cb, path=opts.get("storage_path") or ".")
            if pb.debye is not None:
                raise NotImplementedError(
                    "Debye media: gradients run through tide_b200.debye (propagate routes "
                    "them there)"
                )
            _run_forward_storage(pb, ca, cb, f, r, snaps, need_ca, need_cb, fwd_cb, freq)
        else:
            _run_forward_plain(pb, ca, cb, f, r, fwd_cb, freq)
        ctx.pb = pb
        ctx.snaps = snaps
        ctx.ckpt = ckpt
        ctx.f = f.detach()
        ctx.opts = opts
        ctx.need = (need_ca, need_cb, need_f)
        ctx.save_for_backward(ca, cb)
        ey, hx, hz, mex, mez, mhx, mhz = pb.fields
        for t in (ey, hx, hz, mex, mez, mhx, mhz):
            ctx.mark_non_differentiable(t)
        return ey, hx, hz, mex, mez, mhx, mhz, r

    @staticmethod
    def backward(ctx, *grads):
        pb: TMProblem = ctx.pb
        ca, cb = ctx.saved_tensors
        need_ca, need_cb, need_f = ctx.need
        grad_r = grads[7]
        if ctx.ckpt is not None:
            seg_len, ckpts = ctx.ckpt
            g_ca, g_cb, g_f = _run_backward_checkpointed(pb, ca, cb, ctx.f, grad_r, ckpts, seg_len,
                                                         need_ca, need_cb, need_f, ctx.opts)
        else:
            g_ca, g_cb, g_f = _run_backward(pb, ca, cb, grad_r, ctx.snaps, need_ca, need_cb,
                                            need_f, ctx.opts)
        if not ctx.opts.get("retain_history"):
            # release the history now (a linearization keeps it for more vjps)
            ctx.snaps = None
            ctx.ckpt = None
        return g_ca, g_cb, g_f, None, None


def _run_forward_plain(pb, ca, cb, f, r, fwd_cb, freq):
    nt = pb.nt
    chunk = nt if not fwd_cb else max(1, freq)
    for step in range(0, nt, chunk):
        n = min(chunk, nt - step)
        native_forward(pb, ca, cb, f, r, step, n)
        if fwd_cb:
            fwd_cb(_fwd_state(pb, step + n))


def _fwd_state(pb: TMProblem, step: int) -> CallbackState:
    names = ("Ey", "Hx", "Hz", "m_Ey_x", "m_Ey_z", "m_Hx_z", "m_Hz_x")
    return CallbackState(
        dt=pb.dt, step=step, nt=pb.nt, wavefields=dict(zip(names, pb.fields)), models=pb.models,
        gradients=None, fd_pad=list(pb.fd_pad), pml_width=list(pb.pml_width), is_backward=False,
    )


def _storage_call(pb, ca, cb, f, r_ptr, ptrs, mode, fmt, shot_bytes, need_ca, need_cb, start, n,
                  side=None):
    """One forward_with_storage call over steps [start, start + n); r_ptr and
    ptrs = (ey_dev, ey_host, curl_dev, curl_host) are raw addresses."""
    fn = nat.get_backend_function(
        "maxwell_tm", "forward_with_storage", pb.stencil, pb.dtype, pb.device
    )
    ey, hx, hz, mex, mez, mhx, mhz = pb.fields
    fn(
        nat.ptr(ca), nat.ptr(cb), nat.ptr(pb.cq), nat.ptr(f),
        nat.ptr(ey), nat.ptr(hx), nat.ptr(hz), nat.ptr(mex), nat.ptr(mez), nat.ptr(mhx),
        nat.ptr(mhz), r_ptr, *ptrs,
        *_profile_ptrs(pb), nat.ptr(pb.sources_i), nat.ptr(pb.receivers_i),
        pb.rdy, pb.rdx, pb.dt, n, pb.n_shots, pb.ny, pb.nx, pb.n_src, pb.n_rec,
        pb.grad_interval, mode, fmt, shot_bytes, need_ca, need_cb,
        pb.batched, pb.batched, pb.batched, start,
        pb.pml_y0, pb.pml_x0, pb.pml_y1, pb.pml_x1, 0, pb.device.index or 0,
        _stream_handle(pb.device), int(side.cuda_stream) if side is not None else 0,
    )
    nat.check("maxwell_tm forward_with_storage")


def _snap_ptrs(snaps, shift_bytes: int = 0):
    """Raw addresses of a snapshot set (ey device, ey host, ey file names,
    curl device, curl host, curl file names); device pointers shifted back by
    shift_bytes so that a segment-sized buffer receives the slots of a later
    segment (the native call adds slot * step_bytes)."""
    d = lambda t: nat.ptr(t) - shift_bytes if t is not None and t.numel() else 0  # noqa: E731
    files = snaps.files
    fp = (lambda k: files.pointer(k)) if files is not None else (lambda k: 0)  # noqa: E731
    return (d(snaps.ey_dev), nat.ptr(snaps.ey_host), fp(0), d(snaps.curl_dev),
            nat.ptr(snaps.curl_host), fp(1))


def _run_forward_storage(pb, ca, cb, f, r, snaps, need_ca, need_cb, fwd_cb, freq):
    side = (torch.cuda.Stream(pb.device)
            if snaps.mode in (stg.STORAGE_CPU, stg.STORAGE_DISK) else None)
    snaps.keep.append(side)
    nt = pb.nt
    chunk = nt if not fwd_cb else max(1, freq)
    for step in range(0, nt, chunk):
        n = min(chunk, nt - step)
        _storage_call(pb, ca, cb, f, nat.ptr(r), _snap_ptrs(snaps), snaps.mode, snaps.fmt,
                      snaps.shot_bytes, need_ca, need_cb, step, n, side)
        if fwd_cb:
            fwd_cb(_fwd_state(pb, step + n))


class _AdjointState:
    """Adjoint fields, scratch and gradient accumulators of one backward pass
    (kept across the calls of a chunked or checkpointed backward)."""

    def __init__(self, pb, need_ca, need_cb, scratch=True):
        device, dtype = pb.device, pb.dtype
        S, ny, nx, nt = pb.n_shots, pb.ny, pb.nx, pb.nt
        shape = (S, ny, nx)
        z = lambda: torch.zeros(shape, device=device, dtype=dtype)  # noqa: E731
        self.lam = [z() for _ in range(7)]
        self.scratch = (torch.empty((4, S, ny, nx), device=device, dtype=dtype) if scratch
                        else None)
        self.grad_f = (
            torch.zeros((nt, S, pb.n_src), device=device, dtype=dtype)
            if pb.n_src > 0
            else torch.empty(0, device=device, dtype=dtype)
        )
        empty = torch.empty(0, device=device, dtype=dtype)
        model_shape = shape if pb.batched else (ny, nx)
        self.grad_ca = torch.zeros(model_shape, device=device, dtype=dtype) if need_ca else empty
        self.grad_cb = torch.zeros(model_shape, device=device, dtype=dtype) if need_cb else empty
        self.shot_ca = torch.empty(shape, device=device, dtype=dtype) if need_ca and not pb.batched else empty
        self.shot_cb = torch.empty(shape, device=device, dtype=dtype) if need_cb and not pb.batched else empty

    def result(self, pb, need_ca, need_cb, need_f):
        g_ca = (self.grad_ca if pb.batched else self.grad_ca.unsqueeze(0)) if need_ca else None
        g_cb = (self.grad_cb if pb.batched else self.grad_cb.unsqueeze(0)) if need_cb else None
        g_f = self.grad_f.reshape(-1) if (need_f and pb.n_src > 0) else None
        return g_ca, g_cb, g_f


def _backward_call(pb, ca, cb, grad_r, st: _AdjointState, ptrs, mode, fmt, shot_bytes, need_ca,
                   need_cb, start_t, n, side=None, bg_shots=None):
    """One backward call over t = start_t-1 down to start_t-n.  With
    bg_shots (< n_shots) the snapshot history holds bg_shots shots and shot s
    images against snapshot shot s % bg_shots (the background_vjp_reuse
    entry point)."""
    reuse = bg_shots is not None and bg_shots != pb.n_shots
    fn = nat.get_backend_function("maxwell_tm", "background_vjp_reuse" if reuse else "backward",
                                  pb.stencil, pb.dtype, pb.device)
    storage = (mode, fmt, shot_bytes, bg_shots) if reuse else (mode, fmt, shot_bytes)
    fn(
        nat.ptr(ca), nat.ptr(cb), nat.ptr(pb.cq), nat.ptr(grad_r),
        *[nat.ptr(t) for t in st.lam], nat.ptr(st.scratch),
        *ptrs,
        nat.ptr(st.grad_f), nat.ptr(st.grad_ca), nat.ptr(st.grad_cb), nat.ptr(st.shot_ca),
        nat.ptr(st.shot_cb), *_profile_ptrs(pb), nat.ptr(pb.sources_i), nat.ptr(pb.receivers_i),
        pb.rdy, pb.rdx, pb.dt, n, pb.n_shots, pb.ny, pb.nx, pb.n_src, pb.n_rec, pb.grad_interval,
        *storage, need_ca, need_cb, pb.batched, pb.batched, pb.batched, start_t,
        pb.pml_y0, pb.pml_x0, pb.pml_y1, pb.pml_x1, 0, pb.device.index or 0,
        _stream_handle(pb.device), int(side.cuda_stream) if side is not None else 0,
    )
    nat.check("maxwell_tm backward")


def _grad_r(pb, grad_r):
    if grad_r is None or grad_r.numel() == 0:
        return torch.zeros((pb.nt, pb.n_shots, pb.n_rec), device=pb.device, dtype=pb.dtype)
    return grad_r.contiguous()


def _adjoint_callback(pb, st: _AdjointState, bwd_cb, step, need_ca, need_cb):
    names = ("lambda_Ey", "lambda_Hx", "lambda_Hz", "m_lambda_Ey_x", "m_lambda_Ey_z",
             "m_lambda_Hx_z", "m_lambda_Hz_x")
    grads = {}
    if need_ca:
        grads["ca"] = st.grad_ca
    if need_cb:
        grads["cb"] = st.grad_cb
    bwd_cb(CallbackState(
        dt=pb.dt, step=step, nt=pb.nt, wavefields=dict(zip(names, st.lam)), models=pb.models,
        gradients=grads, fd_pad=list(pb.fd_pad), pml_width=list(pb.pml_width), is_backward=True,
    ))


def _run_backward(pb, ca, cb, grad_r, snaps, need_ca, need_cb, need_f, opts, bg_shots=None):
    grad_r = _grad_r(pb, grad_r)
    nt = pb.nt
    st = _AdjointState(pb, need_ca, need_cb)
    mode = snaps.mode if snaps is not None else stg.STORAGE_NONE
    fmt = snaps.fmt if snaps is not None else 0
    shot_bytes = snaps.shot_bytes if snaps is not None else 0
    ptrs = _snap_ptrs(snaps) if snaps is not None else (0,) * 6
    side = torch.cuda.Stream(pb.device) if mode in (stg.STORAGE_CPU, stg.STORAGE_DISK) else None
    bwd_cb: Callback | None = opts.get("backward_callback")
    freq = int(opts.get("callback_frequency", 1)) if bwd_cb else 0
    chunk = nt if not bwd_cb else max(1, freq)
    for start_t in range(nt, 0, -chunk):
        n = min(chunk, start_t)
        _backward_call(pb, ca, cb, grad_r, st, ptrs, mode, fmt, shot_bytes,
                       need_ca and snaps is not None, need_cb and snaps is not None, start_t, n,
                       side, bg_shots)
        if bwd_cb:
            _adjoint_callback(pb, st, bwd_cb, start_t - n, need_ca, need_cb)
    return st.result(pb, need_ca, need_cb, need_f)


def checkpoint_steps(nt: int, k: int, requested: int | None) -> int:
    """Segment length of the checkpointed gradient: a multiple of the
    gradient sampling interval k, default about sqrt(nt) steps."""
    seg = int(requested or 0) or max(1, int(round(nt ** 0.5)))
    return max(k, (seg + k - 1) // k * k)


def _run_forward_checkpointed(pb, ca, cb, f, r, seg_len, fwd_cb=None, freq=0):
    """Plain forward that keeps the full state (fields and CPML memories) at
    the start of every segment of seg_len steps."""
    ckpts = []
    step = 0
    while step < pb.nt:
        if step % seg_len == 0:
            ckpts.append([t.clone() for t in pb.fields])
        end = min(pb.nt, (step // seg_len + 1) * seg_len)
        if fwd_cb:
            end = min(end, (step // freq + 1) * freq)
        native_forward(pb, ca, cb, f, r, step, end - step)
        step = end
        if fwd_cb and (step % freq == 0 or step == pb.nt):
            fwd_cb(_fwd_state(pb, step))
    return ckpts


def _run_backward_checkpointed(pb, ca, cb, f, grad_r, ckpts, seg_len, need_ca, need_cb, need_f,
                               opts):
    """Checkpoint-and-recompute gradient: for each segment, last first, the
    forward is recomputed from its checkpoint with the segment's snapshots in
    a segment-sized device buffer, then the adjoint runs over the segment."""
    grad_r = _grad_r(pb, grad_r)
    final = [t.clone() for t in pb.fields]
    st = _AdjointState(pb, need_ca, need_cb)
    k = pb.grad_interval
    fmt, sdtype = stg.compression_format(opts.get("storage_compression", False), pb.dtype)
    n_slots = (seg_len + k - 1) // k
    snaps = stg.allocate(stg.STORAGE_DEVICE, sdtype, fmt, n_slots, pb.n_shots, pb.ny, pb.nx,
                         pb.device, need_ca, need_cb)
    step_bytes = snaps.shot_bytes * pb.n_shots
    r_seg = torch.empty((seg_len, pb.n_shots, max(pb.n_rec, 1)), device=pb.device, dtype=pb.dtype)
    r_step_bytes = pb.n_shots * pb.n_rec * r_seg.element_size()
    bwd_cb: Callback | None = opts.get("backward_callback")
    freq = max(1, int(opts.get("callback_frequency", 1))) if bwd_cb else 0
    for idx in range(len(ckpts) - 1, -1, -1):
        seg = idx * seg_len
        n = min(seg_len, pb.nt - seg)
        for dst, src in zip(pb.fields, ckpts[idx]):
            dst.copy_(src)
        # the segment's slots and receivers land in segment-sized buffers: the
        # native call indexes them by absolute step, so their bases move back
        ptrs = _snap_ptrs(snaps, (seg // k) * step_bytes)
        r_ptr = nat.ptr(r_seg) - seg * r_step_bytes if pb.n_rec > 0 else 0
        _storage_call(pb, ca, cb, f, r_ptr, ptrs, stg.STORAGE_DEVICE, fmt, snaps.shot_bytes,
                      need_ca, need_cb, seg, n)
        end = seg + n
        while end > seg:
            # callbacks fall where the stored-history backward makes them:
            # every freq steps counted down from nt, and at step 0
            lo = max(seg, pb.nt - ((pb.nt - end) // freq + 1) * freq) if bwd_cb else seg
            _backward_call(pb, ca, cb, grad_r, st, ptrs, stg.STORAGE_DEVICE, fmt,
                           snaps.shot_bytes, need_ca, need_cb, end, end - lo)
            end = lo
            if bwd_cb and ((pb.nt - end) % freq == 0 or end == 0):
                _adjoint_callback(pb, st, bwd_cb, end, need_ca, need_cb)
    for dst, src in zip(pb.fields, final):
        dst.copy_(src)
    return st.result(pb, need_ca, need_cb, need_f)


def propagate(pb: TMProblem, opts: dict | None = None):
    """Run the TM2D propagation; returns (7 padded state tensors, receivers [nt, S, n_rec])."""
    opts = opts or {}
    needs_graph = pb.ca.requires_grad or pb.cb.requires_grad or pb.f.requires_grad
    if pb.debye is not None:
        d = pb.debye
        if needs_graph or any(torch.is_tensor(d[n]) and d[n].requires_grad
                              for n in ("a", "b", "cp")):
            from .debye import propagate_debye

            if opts.get("forward_callback") or opts.get("backward_callback"):
                raise NotImplementedError("callbacks are not supported for Debye gradients")
            return propagate_debye(pb, opts)
    if needs_graph:
        out = TMPropagate.apply(pb.ca, pb.cb, pb.f, pb, opts)
        return list(out[:7]), out[7]
    r = (
        torch.zeros((pb.nt, pb.n_shots, pb.n_rec), device=pb.device, dtype=pb.dtype)
        if pb.n_rec > 0
        else torch.empty(0, device=pb.device, dtype=pb.dtype)
    )
    _run_forward_plain(pb, pb.ca, pb.cb, pb.f, r, opts.get("forward_callback"),
                       int(opts.get("callback_frequency", 1)))
    return list(pb.fields), r


def build_problem(
    epsilon: torch.Tensor,
    sigma: torch.Tensor,
    mu: torch.Tensor,
    grid_spacing: float | Sequence[float],
    dt: float,
    source_amplitude: torch.Tensor | None,
    source_location: torch.Tensor | None,
    receiver_location: torch.Tensor | None,
    *,
    stencil: int = 2,
    pml_width: int | Sequence[int] = 20,
    max_vel: float | None = None,
    initial_state: Sequence[torch.Tensor | None] | None = None,
    nt: int | None = None,
    model_gradient_sampling_interval: int = 1,
    dispersion: ph.DebyeDispersion | None = None,
) -> tuple[TMProblem, int]:
    """Bounds checks, CFL sub-stepping and prepare_tm2d, as the functional
    API does them (src/tide/maxwell/tm2d.py:258-420): returns the prepared
    problem and the sub-step ratio (receivers are downsampled by it)."""
    ny_m, nx_m = epsilon.shape[-2:]
    for name, loc in (("Source", source_location), ("Receiver", receiver_location)):
        if loc is not None and loc.numel() > 0:
            if bool((loc[..., 0] >= ny_m).any()) or bool((loc[..., 1] >= nx_m).any()):
                raise RuntimeError(f"{name} location out of bounds")
    spacing = ph.normalize_spacing_2d(grid_spacing)
    if max_vel is None:
        max_vel = float((1.0 / torch.sqrt(epsilon * mu)).max().item()) * ph.C0
    inner_dt, ratio = ph.cfl_condition(spacing, dt, max_vel)
    amp = source_amplitude
    if ratio > 1 and amp is not None and amp.numel() > 0:
        amp = ph.upsample(amp, ratio)
    nt_int = nt * ratio if nt is not None else (amp.shape[-1] if amp is not None else None)
    pb = prepare_tm2d(
        epsilon, sigma, mu, spacing, inner_dt, amp, source_location, receiver_location,
        stencil=stencil, pml_width=pml_width, initial_state=initial_state, nt=nt_int,
        model_gradient_sampling_interval=model_gradient_sampling_interval,
        dispersion=dispersion,
    )
    return pb, ratio


def maxwelltm(
    epsilon: torch.Tensor,
    sigma: torch.Tensor,
    mu: torch.Tensor,
    grid_spacing: float | Sequence[float],
    dt: float,
    source_amplitude: torch.Tensor | None,
    source_location: torch.Tensor | None,
    receiver_location: torch.Tensor | None,
    stencil: int = 2,
    pml_width: int | Sequence[int] = 20,
    max_vel: float | None = None,
    Ey_0: torch.Tensor | None = None,
    Hx_0: torch.Tensor | None = None,
    Hz_0: torch.Tensor | None = None,
    m_Ey_x: torch.Tensor | None = None,
    m_Ey_z: torch.Tensor | None = None,
    m_Hx_z: torch.Tensor | None = None,
    m_Hz_x: torch.Tensor | None = None,
    nt: int | None = None,
    model_gradient_sampling_interval: int = 1,
    forward_callback: Callback | None = None,
    backward_callback: Callback | None = None,
    callback_frequency: int = 1,
    storage_mode: str = "device",
    storage_path: str = ".",
    storage_compression: bool | str = False,
    storage_bytes_limit_device: int | None = None,
    storage_bytes_limit_host: int | None = None,
    storage_chunk_steps: int = 0,
    dispersion: ph.DebyeDispersion | None = None,
    retain_history: bool = False,
    **_unused: Any,
):
    """2-D TM solver with the reference's functional signature (src/tide/maxwell/tm2d.py:258).

    Returns (Ey, Hx, Hz, m_Ey_x, m_Ey_z, m_Hx_z, m_Hz_x, receiver_amplitudes);
    wavefields are cropped to the model plus CPML layer, receivers are
    [nt, n_shots, n_receivers] at the user time step.  retain_history keeps
    the snapshot history (or checkpoints) after a backward pass so that the
    graph can be differentiated again (linearizations); by default it is
    released by the first backward pass.
    """
    if callback_frequency <= 0:
        raise ValueError("callback_frequency must be positive")
    pb, ratio = build_problem(
        epsilon, sigma, mu, grid_spacing, dt, source_amplitude, source_location,
        receiver_location, stencil=stencil, pml_width=pml_width, max_vel=max_vel,
        initial_state=[Ey_0, Hx_0, Hz_0, m_Ey_x, m_Ey_z, m_Hx_z, m_Hz_x], nt=nt,
        model_gradient_sampling_interval=model_gradient_sampling_interval,
        dispersion=dispersion,
    )
    opts = dict(
        forward_callback=forward_callback, backward_callback=backward_callback,
        callback_frequency=callback_frequency, storage_mode=storage_mode,
        storage_path=storage_path, storage_compression=storage_compression,
        storage_bytes_limit_device=storage_bytes_limit_device,
        storage_bytes_limit_host=storage_bytes_limit_host,
        storage_chunk_steps=storage_chunk_steps, retain_history=retain_history,
    )
    fields, r = propagate(pb, opts)
    if ratio > 1 and r.numel() > 0:
        r = ph.downsample(r.movedim(0, -1), ratio).movedim(-1, 0)
    return (*[pb.crop(t) for t in fields], r)


__all__ = ["CallbackState", "TMProblem", "build_problem", "maxwelltm", "prepare_tm2d",
           "propagate"]
