"""3-D Maxwell (Yee) propagation on libtide_b200.so (stencil orders 2, 4, 6, 8).

Mirrors the reference's 3-D operator path (src/tide/maxwell/maxwell3d.py:
200-951 and maxwell3d_cuda.py:27-921): coordinate order [z, y, x]; models
padded by fd_pad + CPML width per side ([p, p-1] per axis, replicate);
sources / receivers as flat indices on the padded grid; source amplitudes
scaled by -cb / (dz dy dx) at the source cell; CPML memories held compact
along their own axis (the layout the native ABI takes); an autograd
Function whose backward is the library's exact adjoint.  There is no CPU
path: CPU tensors raise.
"""

from __future__ import annotations

from collections.abc import Sequence
from dataclasses import dataclass, field

import torch

from . import _native as nat
from . import physics as ph
from . import storage as stg

COMPONENTS = {"ex": 0, "ey": 1, "ez": 2}
# Axis (0 z, 1 y, 2 x) of each forward CPML memory, ABI order:
# m_hz_y m_hy_z m_hx_z m_hz_x m_hy_x m_hx_y m_ey_z m_ez_y m_ez_x m_ex_z m_ex_y m_ey_x
MEM_AXES = (1, 0, 0, 2, 2, 1, 0, 1, 2, 0, 1, 2)
MEM_NAMES = ("m_hz_y", "m_hy_z", "m_hx_z", "m_hz_x", "m_hy_x", "m_hx_y",
             "m_ey_z", "m_ez_y", "m_ez_x", "m_ex_z", "m_ex_y", "m_ey_x")
# Adjoint memories, ABI order: ey_z ez_y ez_x ex_z ex_y ey_x hz_y hy_z hx_z hz_x hy_x hx_y
ADJ_MEM_AXES = (0, 1, 2, 0, 1, 2, 1, 0, 0, 2, 2, 1)
PROFILE_ORDER = ("az", "bz", "azh", "bzh", "ay", "by", "ayh", "byh", "ax", "bx", "axh", "bxh",
                 "kz", "kzh", "ky", "kyh", "kx", "kxh")


@dataclass
class CompactLayout:
    """CPML memory kept only on cells c < c0 and c >= max(c0, c1 - 1) of its
    axis (src/tide/grid_utils.py:96-150)."""

    shots: int
    shape: tuple[int, int, int]
    bounds: tuple[tuple[int, int], ...]

    def extent(self, axis: int) -> int:
        lo, hi = self.bounds[axis]
        return lo + self.shape[axis] - max(lo, hi - 1)

    def full_shape(self) -> tuple[int, ...]:
        return (self.shots, *self.shape)

    def compact_shape(self, axis: int) -> tuple[int, ...]:
        s = list(self.full_shape())
        s[axis + 1] = self.extent(axis)
        return tuple(s)

    def coords(self, axis: int, device=None) -> torch.Tensor:
        lo, hi = self.bounds[axis]
        n = self.shape[axis]
        return torch.cat([torch.arange(lo, device=device), torch.arange(max(lo, hi - 1), n, device=device)])

    def zeros(self, axis: int, device, dtype) -> torch.Tensor:
        return torch.zeros(self.compact_shape(axis), device=device, dtype=dtype)

    def pack(self, full: torch.Tensor, axis: int) -> torch.Tensor:
        return full.index_select(axis + 1, self.coords(axis, full.device)).contiguous()

    def unpack(self, compact: torch.Tensor, axis: int) -> torch.Tensor:
        out = torch.zeros(self.full_shape(), device=compact.device, dtype=compact.dtype)
        return out.index_copy(axis + 1, self.coords(axis, compact.device), compact)


@dataclass
class EM3DProblem:
    """Everything one native 3-D call needs (padded grid)."""

    ca: torch.Tensor
    cb: torch.Tensor
    cq: torch.Tensor
    f: torch.Tensor
    profiles: dict
    sources_i: torch.Tensor
    receivers_i: torch.Tensor
    fields: list
    memories: list
    layout: CompactLayout
    rdz: float
    rdy: float
    rdx: float
    dt: float
    nt: int
    n_shots: int
    nz: int
    ny: int
    nx: int
    n_src: int
    n_rec: int
    pml: tuple  # z0, y0, x0, z1, y1, x1
    batched: bool
    src_comp: int
    rec_comp: int
    grad_interval: int
    fd_pad: list
    pml_width: list
    dtype: torch.dtype
    device: torch.device
    models: dict = field(default_factory=dict)
    stencil: int = 2


def _widths(pml_width: int | Sequence[int]) -> list[int]:
    if isinstance(pml_width, int):
        return [pml_width] * 6
    w = [int(v) for v in pml_width]
    if len(w) == 3:
        return [w[0], w[0], w[1], w[1], w[2], w[2]]
    if len(w) != 6:
        raise ValueError("pml_width must be an int or 3 / 6 values [z0, z1, y0, y1, x0, x1]")
    return w


def _spacing(h: float | Sequence[float]) -> list[float]:
    if isinstance(h, (int, float)):
        return [float(h)] * 3
    v = [float(x) for x in h]
    if len(v) != 3:
        raise ValueError("grid_spacing must be a float or [dz, dy, dx]")
    return v


def initial_state_3d(initial_state, layout: CompactLayout, fd, device, dtype):
    """Padded fields and compact CPML memories from an 18-tensor state (None
    entries start at zero): zero fd padding as create_or_pad(...,
    mode="constant"), memories packed to their strips."""
    S = layout.shots
    shape = (S, *layout.shape)
    init = list(initial_state) if initial_state is not None else [None] * 18
    if len(init) != 18:
        raise ValueError("initial_state holds 6 fields and 12 CPML memories")

    def padded(t):
        if t.ndim == 3:
            t = t[None].expand(S, -1, -1, -1)
        t = t.to(device=device, dtype=dtype)
        if tuple(t.shape) == shape:
            return t.clone().contiguous()
        return torch.nn.functional.pad(t, ph._torch_pad_order(fd)).contiguous()

    fields = [padded(t) if t is not None and t.numel() else torch.zeros(shape, device=device, dtype=dtype)
              for t in init[:6]]
    memories = [layout.pack(padded(t), a) if t is not None and t.numel() else layout.zeros(a, device, dtype)
                for t, a in zip(init[6:], MEM_AXES)]
    return fields, memories


def prepare_em3d(
    epsilon: torch.Tensor, sigma: torch.Tensor, mu: torch.Tensor,
    grid_spacing: float | Sequence[float], dt: float,
    source_amplitude: torch.Tensor | None, source_location: torch.Tensor | None,
    receiver_location: torch.Tensor | None, *, stencil: int = 2,
    pml_width: int | Sequence[int] = 20, source_component: str = "ey",
    receiver_component: str = "ey", model_gradient_sampling_interval: int = 1,
    nt: int | None = None, initial_state: Sequence[torch.Tensor | None] | None = None,
) -> EM3DProblem:
    """Pad the model, build coefficients, CPML profiles, point indices and the
    initial state (maxwell3d_cuda.py:310-528).  initial_state: Ex, Ey, Ez, Hx,
    Hy, Hz and the 12 CPML memories in MEM_NAMES order, each [nz', ny', nx']
    or [S, nz', ny', nx'] on the model + CPML region (the shape this module
    returns) or on the full padded grid; None entries start at zero."""
    if stencil not in (2, 4, 6, 8):
        raise ValueError("stencil must be 2, 4, 6 or 8")
    if epsilon.ndim not in (3, 4) or sigma.shape != epsilon.shape or mu.shape != epsilon.shape:
        raise ValueError("epsilon, sigma, mu must share a [nz, ny, nx] or [S, nz, ny, nx] shape")
    if source_component not in COMPONENTS or receiver_component not in COMPONENTS:
        raise ValueError("components must be 'ex', 'ey' or 'ez'")
    device, dtype = epsilon.device, epsilon.dtype
    batched = epsilon.ndim == 4
    dz, dy, dx = _spacing(grid_spacing)
    widths = _widths(pml_width)
    hp = stencil // 2
    fd = [hp, hp - 1, hp, hp - 1, hp, hp - 1]
    pad = [a + b for a, b in zip(fd, widths)]
    mz, my, mx = epsilon.shape[-3:]
    nz, ny, nx = mz + pad[0] + pad[1], my + pad[2] + pad[3], mx + pad[4] + pad[5]
    pml = (fd[0] + widths[0], fd[2] + widths[2], fd[4] + widths[4],
           nz - fd[1] - widths[1], ny - fd[3] - widths[3], nx - fd[5] - widths[5])
    eps_p, sig_p, mu_p = (ph.replicate_pad(t, pad).contiguous() for t in (epsilon, sigma, mu))
    coef = ph.compile_material_coefficients(eps_p, sig_p, mu_p, dt)
    ca, cb, cq = coef["ca"], coef["cb"], coef["cq"]
    if source_amplitude is not None and source_amplitude.numel() > 0:
        S = source_amplitude.shape[0]
    elif source_location is not None and source_location.numel() > 0:
        S = source_location.shape[0]
    elif receiver_location is not None and receiver_location.numel() > 0:
        S = receiver_location.shape[0]
    else:
        S = epsilon.shape[0] if batched else 1
    if nt is None:
        if source_amplitude is None or source_amplitude.numel() == 0:
            raise ValueError("nt is needed when there are no source amplitudes")
        nt = int(source_amplitude.shape[-1])

    def flat(loc):
        if loc is None or loc.numel() == 0:
            return torch.empty(0, device=device, dtype=torch.long), 0
        loc = loc.to(device)
        z, y, x = loc[..., 0] + pad[0], loc[..., 1] + pad[2], loc[..., 2] + pad[4]
        return ((z * ny + y) * nx + x).long().contiguous(), loc.shape[1]

    sources_i, n_src = flat(source_location)
    receivers_i, n_rec = flat(receiver_location)
    if n_src > 0 and source_amplitude is not None and source_amplitude.numel() > 0:
        cbf = cb.reshape(S if batched else 1, -1).expand(S, -1)
        cb_at = cbf.gather(1, sources_i)
        f = (source_amplitude.permute(2, 0, 1) * cb_at[None] * (-1.0 / (dx * dy * dz)))
        f = f.reshape(-1).contiguous()
    else:
        f = torch.empty(0, device=device, dtype=dtype)
    prof = ph.set_pml_profiles_3d(widths, fd, dt, [dz, dy, dx], dtype, device, nz, ny, nx)
    layout = CompactLayout(S, (nz, ny, nx), ((pml[0], pml[3]), (pml[1], pml[4]), (pml[2], pml[5])))
    fields, memories = initial_state_3d(initial_state, layout, fd, device, dtype)
    shp = (S, nz, ny, nx) if batched else (1, nz, ny, nx)
    return EM3DProblem(
        ca=ca.reshape(shp), cb=cb.reshape(shp), cq=cq.reshape(shp), f=f, profiles=prof,
        sources_i=sources_i, receivers_i=receivers_i, fields=fields, memories=memories,
        layout=layout, rdz=1.0 / dz, rdy=1.0 / dy, rdx=1.0 / dx, dt=float(dt), nt=int(nt),
        n_shots=int(S), nz=nz, ny=ny, nx=nx, n_src=int(n_src), n_rec=int(n_rec), pml=pml,
        batched=batched, src_comp=COMPONENTS[source_component],
        rec_comp=COMPONENTS[receiver_component],
        grad_interval=int(model_gradient_sampling_interval), fd_pad=fd, pml_width=widths,
        dtype=dtype, device=device, models={"epsilon": eps_p, "sigma": sig_p, "mu": mu_p},
        stencil=int(stencil),
    )


# ----------------------------------------------------------------- native calls
def _p(t):
    return nat.ptr(t)


def _profile_ptrs(pb: EM3DProblem) -> list[int]:
    return [_p(pb.profiles[k]) for k in PROFILE_ORDER]


def _tail(pb: EM3DProblem, nt: int, step_ratio: int) -> list:
    return [pb.rdz, pb.rdy, pb.rdx, pb.dt, nt, pb.n_shots, pb.nz, pb.ny, pb.nx, pb.n_src,
            pb.n_rec, step_ratio]


def _flags(pb: EM3DProblem, start_t: int) -> list:
    b = pb.batched
    return [b, b, b, start_t, *pb.pml, pb.src_comp, pb.rec_comp, 0,
            pb.device.index or 0, 0]


def native_forward(pb: EM3DProblem, ca, cb, f, r, start_t: int, nt: int) -> None:
    fn = nat.get_backend_function("maxwell_3d", "forward", pb.stencil, pb.dtype, pb.device)
    stream = torch.cuda.current_stream(pb.device).cuda_stream
    fn(_p(ca), _p(cb), _p(pb.cq), _p(f), *[_p(t) for t in pb.fields],
       *[_p(t) for t in pb.memories], *([0] * 9), _p(r), 0, *_profile_ptrs(pb),
       _p(pb.sources_i), _p(pb.receivers_i), *_tail(pb, nt, 1), False, *_flags(pb, start_t),
       stream)
    nat.check("maxwell_3d forward")


@dataclass
class Snapshots3D:
    mode: int
    fmt: int
    n_store: int
    shot_bytes: int
    dev: list  # 6 device buffers (or empty)
    host: list  # 6 pinned host histories (cpu mode) or staging rings (disk mode)
    q0: int = 0  # first store slot held by the device buffers (checkpoint segments)
    files: object = None  # storage.DiskFiles of the disk mode
    side: object = None  # storage stream of the cpu / disk modes


def allocate_snapshots(pb: EM3DProblem, mode: int, fmt: int, need_ca: bool, need_cb: bool,
                       n_store: int | None = None, path: str = ".") -> Snapshots3D:
    """Buffers of the six snapshot kinds: device mode the whole history on
    the device; cpu mode a 3-slot device ring and the pinned host history;
    disk mode a 3-slot device ring, a 3-slot pinned staging ring and one
    temporary file per kind under path."""
    k = max(1, pb.grad_interval)
    n_store = (pb.nt + k - 1) // k if n_store is None else int(n_store)
    sdt = torch.bfloat16 if fmt == 1 else pb.dtype
    esz = torch.tensor([], dtype=sdt).element_size()
    shot_bytes = pb.nz * pb.ny * pb.nx * esz
    empty = torch.empty(0, device=pb.device, dtype=sdt)
    need = [need_ca] * 3 + [need_cb] * 3
    if mode != stg.STORAGE_NONE and any(need):
        stg.release_history_pool()  # a kept 2-D history would hold the device memory
    dev, host = [], []
    for c in range(6):
        if not need[c] or mode == stg.STORAGE_NONE:
            dev.append(empty)
            host.append(torch.empty(0, dtype=sdt))
        elif mode == stg.STORAGE_DEVICE:
            dev.append(torch.empty((n_store, pb.n_shots, pb.nz, pb.ny, pb.nx), device=pb.device, dtype=sdt))
            host.append(torch.empty(0, dtype=sdt))
        else:
            dev.append(torch.empty((3, pb.n_shots, pb.nz, pb.ny, pb.nx), device=pb.device, dtype=sdt))
            n_host = 3 if mode == stg.STORAGE_DISK else n_store
            host.append(torch.empty((n_host, pb.n_shots, pb.nz * pb.ny * pb.nx), dtype=sdt,
                                    pin_memory=True))
    sn = Snapshots3D(mode, fmt, n_store, shot_bytes, dev, host)
    if mode == stg.STORAGE_DISK and any(need):
        sn.files = stg.DiskFiles(path, *need, tags=("ex", "ey", "ez", "cx", "cy", "cz"))
    if mode in (stg.STORAGE_CPU, stg.STORAGE_DISK) and any(need):
        sn.side = torch.cuda.Stream(pb.device)
    return sn


def _store_ptrs(sn: Snapshots3D) -> list[int]:
    """Raw snapshot addresses; device bases move back by q0 slots so that a
    segment-sized buffer receives the slots of a later segment (the native
    call adds slot * step_bytes)."""
    out = []
    for c in range(6):
        d = sn.dev[c]
        step = d[0].numel() * d.element_size() if d.numel() else 0
        out += [_p(d) - sn.q0 * step if d.numel() else 0, _p(sn.host[c]),
                sn.files.pointer(c) if sn.files is not None else 0]
    return out


def native_forward_storage(pb: EM3DProblem, ca, cb, f, r, sn: Snapshots3D, need_ca: bool,
                           need_cb: bool, start_t: int = 0, nt: int | None = None) -> None:
    nt = pb.nt if nt is None else nt
    fn = nat.get_backend_function("maxwell_3d", "forward_with_storage", pb.stencil, pb.dtype, pb.device)
    stream = torch.cuda.current_stream(pb.device).cuda_stream
    fn(_p(ca), _p(cb), _p(pb.cq), _p(f), *[_p(t) for t in pb.fields],
       *[_p(t) for t in pb.memories], _p(r), *_store_ptrs(sn), *_profile_ptrs(pb),
       _p(pb.sources_i), _p(pb.receivers_i), *_tail(pb, nt, max(1, pb.grad_interval)),
       sn.mode, sn.fmt, sn.shot_bytes, need_ca, need_cb, *_flags(pb, start_t), stream,
       sn.side.cuda_stream if sn.side is not None else stream)
    nat.check("maxwell_3d forward_with_storage")


def native_backward(pb: EM3DProblem, ca, cb, grad_r, sn: Snapshots3D, need_ca: bool,
                    need_cb: bool, need_f: bool, *, grad_eps=None, grad_sigma=None,
                    lam=None, start_t: int | None = None, nt: int | None = None, grads=None):
    """Exact adjoint; returns (grad_ca, grad_cb, grad_f) with grad_ca/cb
    shaped like ca/cb, grad_f [nt * S * n_src].  grads: the same triple from
    an earlier call over later steps, accumulated into (chunked adjoint)."""
    dev, dt_ = pb.device, pb.dtype
    S, nz, ny, nx = pb.n_shots, pb.nz, pb.ny, pb.nx
    nt_all = pb.nt
    nt = nt_all if nt is None else nt
    start_t = nt_all if start_t is None else start_t
    shape = (S, nz, ny, nx)
    if lam is None:
        lam = {"fields": [torch.zeros(shape, device=dev, dtype=dt_) for _ in range(6)],
               "mem": [pb.layout.zeros(a, dev, dt_) for a in ADJ_MEM_AXES]}
    scratch = torch.empty(sum(m.numel() for m in lam["mem"]), device=dev, dtype=dt_)
    empty = torch.empty(0, device=dev, dtype=dt_)
    mshape = ca.shape
    if grads is not None:
        grad_ca, grad_cb, grad_f = grads
    else:
        grad_ca = torch.zeros(mshape, device=dev, dtype=dt_) if need_ca else empty
        grad_cb = torch.zeros(mshape, device=dev, dtype=dt_) if need_cb else empty
        grad_f = (torch.zeros(nt_all * S * pb.n_src, device=dev, dtype=dt_)
                  if need_f and pb.n_src > 0 else empty)
    shot_ca = torch.empty(shape, device=dev, dtype=dt_) if need_ca and not pb.batched and S > 1 else empty
    shot_cb = torch.empty(shape, device=dev, dtype=dt_) if need_cb and not pb.batched and S > 1 else empty
    fn = nat.get_backend_function("maxwell_3d", "backward", pb.stencil, dt_, dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    fn(_p(ca), _p(cb), _p(pb.cq), _p(grad_r), *[_p(t) for t in lam["fields"]],
       *[_p(t) for t in lam["mem"]], _p(scratch), *_store_ptrs(sn), _p(grad_f), _p(grad_ca),
       _p(grad_cb), _p(grad_eps), _p(grad_sigma), _p(shot_ca), _p(shot_cb), False,
       *_profile_ptrs(pb), _p(pb.sources_i), _p(pb.receivers_i),
       *_tail(pb, nt, max(1, pb.grad_interval)), sn.mode, sn.fmt, sn.shot_bytes, need_ca,
       need_cb, *_flags(pb, start_t), stream,
       sn.side.cuda_stream if sn.side is not None else stream)
    nat.check("maxwell_3d backward")
    return grad_ca, grad_cb, grad_f


CHECKPOINT = -1  # storage code of the checkpoint-and-recompute gradient (Python-side)


def checkpoint_steps(nt: int, k: int, requested: int | None) -> int:
    """Segment length of the checkpointed gradient: a multiple of the gradient
    sampling interval k, default about sqrt(nt) steps."""
    seg = int(requested or 0) or max(1, int(round(nt ** 0.5)))
    return max(k, (seg + k - 1) // k * k)


def _state(pb: EM3DProblem) -> list:
    return list(pb.fields) + list(pb.memories)


def forward_checkpointed(pb: EM3DProblem, ca, cb, f, r, seg: int) -> list:
    """Plain forward keeping the full state (6 fields, 12 compact memories) at
    the start of every segment of seg steps."""
    ckpts = []
    for t0 in range(0, pb.nt, seg):
        ckpts.append([t.clone() for t in _state(pb)])
        native_forward(pb, ca, cb, f, r, t0, min(seg, pb.nt - t0))
    return ckpts


def backward_checkpointed(pb: EM3DProblem, ca, cb, f, grad_r, ckpts: list, seg: int, fmt: int,
                          need_ca: bool, need_cb: bool, need_f: bool):
    """Checkpoint-and-recompute gradient: for each segment, last first, the
    forward is recomputed from its checkpoint with the segment's snapshots in
    a segment-sized device buffer, then the adjoint runs over the segment and
    accumulates into the same gradients.  The final forward state is put back
    at the end."""
    k = max(1, pb.grad_interval)
    final = [t.clone() for t in _state(pb)]
    sn = allocate_snapshots(pb, stg.STORAGE_DEVICE, fmt, need_ca, need_cb, n_store=seg // k)
    r_scratch = torch.empty((pb.nt, pb.n_shots, max(pb.n_rec, 1)), device=pb.device, dtype=pb.dtype)
    shape = (pb.n_shots, pb.nz, pb.ny, pb.nx)
    dev, dt_ = pb.device, pb.dtype
    lam = {"fields": [torch.zeros(shape, device=dev, dtype=dt_) for _ in range(6)],
           "mem": [pb.layout.zeros(a, dev, dt_) for a in ADJ_MEM_AXES]}
    grads = None
    for idx in range(len(ckpts) - 1, -1, -1):
        t0 = idx * seg
        n = min(seg, pb.nt - t0)
        for dst, src in zip(_state(pb), ckpts[idx]):
            dst.copy_(src)
        sn.q0 = t0 // k
        native_forward_storage(pb, ca, cb, f, r_scratch if pb.n_rec > 0 else r_scratch[:0], sn,
                               need_ca, need_cb, start_t=t0, nt=n)
        grads = native_backward(pb, ca, cb, grad_r, sn, need_ca, need_cb, need_f, lam=lam,
                                start_t=t0 + n, nt=n, grads=grads)
    for dst, src in zip(_state(pb), final):
        dst.copy_(src)
    return grads


class EM3DPropagate(torch.autograd.Function):
    """Receivers from (ca, cb, f); backward through the exact adjoint, from a
    stored snapshot history (device or pinned host) or by checkpoint segments
    with recomputation (mode CHECKPOINT)."""

    @staticmethod
    def forward(ctx, ca, cb, f, pb: EM3DProblem, mode: int, fmt: int, seg: int, retain: bool,
                path: str = "."):
        need_ca, need_cb = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        r = torch.zeros((pb.nt, pb.n_shots, pb.n_rec), device=pb.device, dtype=pb.dtype)
        ctx.pb, ctx.mode, ctx.fmt, ctx.seg, ctx.retain = pb, mode, fmt, seg, retain
        ctx.flags = (need_ca, need_cb, ctx.needs_input_grad[2])
        if mode == CHECKPOINT and (need_ca or need_cb or ctx.needs_input_grad[2]):
            ctx.ckpts = forward_checkpointed(pb, ca, cb, f, r, seg)
            ctx.save_for_backward(ca, cb, f)
        elif need_ca or need_cb or ctx.needs_input_grad[2]:
            sn = allocate_snapshots(pb, mode, fmt, need_ca, need_cb, path=path)
            native_forward_storage(pb, ca, cb, f, r, sn, need_ca, need_cb)
            ctx.sn = sn
            ctx.save_for_backward(ca, cb, f)
        else:
            native_forward(pb, ca, cb, f, r, 0, pb.nt)
        return r

    @staticmethod
    def backward(ctx, grad_r):
        ca, cb, f = ctx.saved_tensors
        need_ca, need_cb, need_f = ctx.flags
        if ctx.mode == CHECKPOINT:
            gca, gcb, gf = backward_checkpointed(ctx.pb, ca, cb, f, grad_r.contiguous(), ctx.ckpts,
                                                 ctx.seg, ctx.fmt, need_ca, need_cb, need_f)
        else:
            gca, gcb, gf = native_backward(ctx.pb, ca, cb, grad_r.contiguous(), ctx.sn, need_ca,
                                           need_cb, need_f)
        if not ctx.retain:  # release the history (a linearization keeps it)
            ctx.ckpts = ctx.sn = None
        return (gca if need_ca else None, gcb if need_cb else None,
                gf if need_f else None, None, None, None, None, None, None)


STATE_NAMES = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz") + MEM_NAMES


def _crop(pb: EM3DProblem) -> tuple:
    """Index of the model + CPML region of a padded [S, nz, ny, nx] array:
    fd_pad[before] cells off the start and fd_pad[after] off the end of each
    axis (maxwell3d_cuda.py:864-876)."""
    fd, n = pb.fd_pad, (pb.nz, pb.ny, pb.nx)
    return (slice(None),) + tuple(
        slice(fd[2 * a], n[a] - fd[2 * a + 1] if fd[2 * a + 1] > 0 else None) for a in range(3))


def maxwell3d(
    epsilon: torch.Tensor, sigma: torch.Tensor, mu: torch.Tensor,
    grid_spacing: float | Sequence[float], dt: float,
    source_amplitude: torch.Tensor | None, source_location: torch.Tensor | None,
    receiver_location: torch.Tensor | None, stencil: int = 2,
    pml_width: int | Sequence[int] = 20, max_vel: float | None = None,
    Ex_0: torch.Tensor | None = None, Ey_0: torch.Tensor | None = None,
    Ez_0: torch.Tensor | None = None, Hx_0: torch.Tensor | None = None,
    Hy_0: torch.Tensor | None = None, Hz_0: torch.Tensor | None = None,
    m_hz_y: torch.Tensor | None = None, m_hy_z: torch.Tensor | None = None,
    m_hx_z: torch.Tensor | None = None, m_hz_x: torch.Tensor | None = None,
    m_hy_x: torch.Tensor | None = None, m_hx_y: torch.Tensor | None = None,
    m_ey_z: torch.Tensor | None = None, m_ez_y: torch.Tensor | None = None,
    m_ez_x: torch.Tensor | None = None, m_ex_z: torch.Tensor | None = None,
    m_ex_y: torch.Tensor | None = None, m_ey_x: torch.Tensor | None = None,
    nt: int | None = None,
    model_gradient_sampling_interval: int = 1, source_component: str = "ey",
    receiver_component: str = "ey", storage_mode: str = "device", storage_path: str = ".",
    storage_compression: bool | str = False, storage_bytes_limit_device: int | None = None,
    storage_bytes_limit_host: int | None = None, storage_chunk_steps: int | None = None,
    forward_callback=None, backward_callback=None, callback_frequency: int = 1,
    dispersion=None, retain_history: bool = False, **_unused,
):
    """3-D Maxwell solve (src/tide/maxwell/maxwell3d.py:200-951): returns the
    final Ex, Ey, Ez, Hx, Hy, Hz and the 12 CPML memories on the model + CPML
    region (outer fd_pad cells removed), then the receiver data [nt, S, n_rec].
    Differentiable in epsilon, sigma and source_amplitude.  The initial state
    (Ex_0 .. m_ey_x) takes the same shapes.  storage_mode: 'device', 'cpu'
    (pinned host history), 'disk' (one temporary file per snapshot kind under
    storage_path), 'none', 'auto', or 'checkpoint' (segments of
    storage_chunk_steps steps, default about sqrt(nt), recomputed in the
    backward pass).  As in the reference (maxwell3d.py:418-440), a dt above
    the CFL bound for max_vel (default: the model's largest wave speed) runs
    ceil(dt / dt_max) internal steps per user step, with the source
    amplitudes upsampled and the receivers downsampled by that ratio.
    retain_history keeps the history (or checkpoints) after a backward pass
    for further vjps.  Callbacks and dispersive media are not built for the
    3-D path and raise."""
    if epsilon.device.type != "cuda":
        raise nat.NativeError("libtide_b200 runs on CUDA devices only; there is no CPU path.")
    if forward_callback is not None or backward_callback is not None:
        raise NotImplementedError("callbacks are not built for the 3-D path")
    if dispersion is not None:
        raise NotImplementedError("dispersive media are not built for the 3-D path")
    if max_vel is None:
        max_vel = float((1.0 / torch.sqrt(epsilon * mu)).max().item()) * ph.C0
    inner_dt, ratio = ph.cfl_condition(_spacing(grid_spacing), dt, max_vel)
    amp = source_amplitude
    if ratio > 1 and amp is not None and amp.numel() > 0:
        amp = ph.upsample(amp, ratio)
    nt_int = nt * ratio if nt is not None else None
    init = [Ex_0, Ey_0, Ez_0, Hx_0, Hy_0, Hz_0, m_hz_y, m_hy_z, m_hx_z, m_hz_x, m_hy_x, m_hx_y,
            m_ey_z, m_ez_y, m_ez_x, m_ex_z, m_ex_y, m_ey_x]
    pb = prepare_em3d(epsilon, sigma, mu, grid_spacing, inner_dt, amp, source_location,
                      receiver_location, stencil=stencil, pml_width=pml_width,
                      source_component=source_component, receiver_component=receiver_component,
                      model_gradient_sampling_interval=model_gradient_sampling_interval, nt=nt_int,
                      initial_state=init)
    sm = str(storage_mode).lower()
    fmt, sdtype = stg.compression_format(storage_compression, pb.dtype)
    k = max(1, pb.grad_interval)
    if sm == "checkpoint":
        mode, seg = CHECKPOINT, checkpoint_steps(pb.nt, k, storage_chunk_steps)
    else:
        # 'auto': device history if it fits the device budget, else pinned host
        mode = stg.resolve_mode(
            sm, device=pb.device, n_store=(pb.nt + k - 1) // k, n_shots=pb.n_shots,
            ny=pb.nz * pb.ny, nx=pb.nx, itemsize=torch.tensor([], dtype=sdtype).element_size(),
            n_arrays=6, bytes_limit_device=storage_bytes_limit_device,
            bytes_limit_host=storage_bytes_limit_host)
        seg = 0
    r = EM3DPropagate.apply(pb.ca, pb.cb, pb.f, pb, mode, fmt, seg, bool(retain_history),
                            storage_path or ".")
    s = _crop(pb)
    outs = [t[s] for t in pb.fields]
    outs += [pb.layout.unpack(m, a)[s] for m, a in zip(pb.memories, MEM_AXES)]
    if ratio > 1 and r.numel() > 0:
        r = ph.downsample(r.movedim(0, -1), ratio).movedim(-1, 0)
    return (*outs, r)


class Born3DPropagate(torch.autograd.Function):
    """The Born map (dca, dcb, df; ca, cb, f0) -> scattered receivers on the
    native 3-D Born entry points, as the reference's Born3DForwardFunc
    (src/tide/maxwell/maxwell3d_born_autograd.py:17-1276).  Forward:
    maxwell_3d_*_born_forward_with_storage (device history of the background
    E^n / curl H^n and, when the background needs a gradient, of the
    scattered E^n / curl; full CPML memories).  Backward:
    maxwell_3d_*_born_backward (the background adjoint imaging against the
    background history) for the perturbation alone, or
    maxwell_3d_*_born_backward_bggrad (the joint background + scattered
    adjoint) when the background (ca, cb, f0) needs a gradient.  The
    background and scattered states advance in place in the call's tensors
    (call = the arguments of the native born_forward)."""

    @staticmethod
    def forward(ctx, dca_p, dcb_p, df, ca, cb, f0, call):
        pb, k = call["pb"], max(1, call["pb"].grad_interval)
        need = ctx.needs_input_grad
        second = need[3] or need[4] or need[5]
        need_ca, need_cb = need[0] or second, need[1] or second
        n_store = (pb.nt + k - 1) // k
        shape = (n_store, pb.n_shots, pb.nz, pb.ny, pb.nx)
        empty = torch.empty(0, device=pb.device, dtype=pb.dtype)
        st = [torch.empty(shape, device=pb.device, dtype=pb.dtype)
              if (need_ca if c < 3 else need_cb) else empty for c in range(6)]
        sc = [torch.empty(shape, device=pb.device, dtype=pb.dtype) for _ in range(6)] if second \
            else [empty] * 6
        s18 = []
        for t in st:
            s18 += [_p(t), 0, 0]
        shot_bytes = pb.nz * pb.ny * pb.nx * pb.ca.element_size()
        fn = nat.get_backend_function("maxwell_3d", "born_forward_with_storage", pb.stencil,
                                      pb.dtype, pb.device)
        stream = torch.cuda.current_stream(pb.device).cuda_stream
        r = torch.zeros((pb.nt, pb.n_shots, pb.n_rec), device=pb.device, dtype=pb.dtype)
        fn(*call["head"](dca_p, dcb_p, df, r), *s18, *[_p(t) for t in sc], *_profile_ptrs(pb),
           _p(pb.sources_i), _p(pb.receivers_i), pb.rdz, pb.rdy, pb.rdx, pb.dt, pb.nt,
           pb.n_shots, pb.nz, pb.ny, pb.nx, call["n_src"], pb.n_rec, k, 0, 0, shot_bytes,
           need_ca, need_cb, pb.batched, pb.batched, pb.batched, 0, *pb.pml, pb.src_comp,
           pb.rec_comp, 0, pb.device.index or 0, 0, stream, stream)
        nat.check("maxwell_3d born_forward_with_storage")
        ctx.pb, ctx.st, ctx.sc, ctx.k, ctx.shot_bytes = pb, st, sc, k, shot_bytes
        ctx.n_src, ctx.second = call["n_src"], second
        ctx.pert = (dca_p.detach(), dcb_p.detach(), df.detach())
        return r

    @staticmethod
    def backward(ctx, grad_r):
        pb, dev, dt = ctx.pb, ctx.pb.device, ctx.pb.dtype
        S = pb.n_shots
        full = (S, pb.nz, pb.ny, pb.nx)
        empty = torch.empty(0, device=dev, dtype=dt)
        need = ctx.needs_input_grad
        z = lambda: torch.zeros(full, device=dev, dtype=dt)  # noqa: E731
        mshape = (1, pb.nz, pb.ny, pb.nx)
        s18 = []
        for t in ctx.st:
            s18 += [_p(t), 0, 0]
        stream = torch.cuda.current_stream(dev).cuda_stream
        nf = pb.nt * S * ctx.n_src
        tail = [*_profile_ptrs(pb), _p(pb.sources_i), _p(pb.receivers_i), pb.rdz, pb.rdy,
                pb.rdx, pb.dt, pb.nt, S, pb.nz, pb.ny, pb.nx, ctx.n_src, pb.n_rec, ctx.k, 0, 0,
                ctx.shot_bytes]
        flags = [pb.batched, pb.batched, pb.batched, pb.nt, *pb.pml, pb.src_comp, pb.rec_comp, 0,
                 dev.index or 0, 0, stream, stream]
        if ctx.second:
            g = [torch.zeros(mshape, device=dev, dtype=dt) for _ in range(4)]
            gs = [torch.empty(full, device=dev, dtype=dt) if S > 1 else empty for _ in range(4)]
            gf0 = torch.zeros(nf, device=dev, dtype=dt) if ctx.n_src > 0 else empty
            gdf = torch.zeros(nf, device=dev, dtype=dt) if ctx.n_src > 0 else empty
            dca, dcb, df = ctx.pert
            # every work array stays referenced until the call is enqueued: a
            # tensor dropped after taking its pointer would hand its block to
            # the next allocation, and the arrays would alias
            lam_eta = [z() for _ in range(36)]  # adjoint fields + memories, twice
            scratch = torch.empty((24, *full), device=dev, dtype=dt)
            work = [z() for _ in range(3)]
            grad_r = grad_r.contiguous()
            fn = nat.get_backend_function("maxwell_3d", "born_backward_bggrad", pb.stencil, dt,
                                          dev)
            fn(_p(pb.ca), _p(pb.cb), _p(pb.cq), _p(dca), _p(dcb), _p(pb.f), _p(df), _p(grad_r),
               *[_p(t) for t in lam_eta], _p(scratch), *s18, *[_p(t) for t in ctx.sc], _p(gf0),
               _p(gdf), _p(g[2]), _p(g[3]), _p(g[0]), _p(g[1]), *[_p(t) for t in gs],
               *[_p(t) for t in work], *tail, True, True, True, True, *flags)
            nat.check("maxwell_3d born_backward_bggrad")
            ctx.st = ctx.sc = None
            return (g[0], g[1], gdf if ctx.n_src > 0 else None, g[2], g[3],
                    gf0 if ctx.n_src > 0 else None, None)
        need_ca, need_cb = need[0], need[1]
        lam = [z() for _ in range(6)]
        lmem = [z() for _ in range(12)]
        scratch = torch.empty((12, *full), device=dev, dtype=dt)
        gca = torch.empty(mshape, device=dev, dtype=dt) if need_ca else empty
        gcb = torch.empty(mshape, device=dev, dtype=dt) if need_cb else empty
        gca_s = torch.empty(full, device=dev, dtype=dt) if need_ca and S > 1 else empty
        gcb_s = torch.empty(full, device=dev, dtype=dt) if need_cb and S > 1 else empty
        gf = torch.empty(nf, device=dev, dtype=dt) if need[2] and ctx.n_src > 0 else empty
        grad_r = grad_r.contiguous()
        fn = nat.get_backend_function("maxwell_3d", "born_backward", pb.stencil, dt, dev)
        fn(_p(pb.ca), _p(pb.cb), _p(pb.cq), _p(grad_r), *[_p(t) for t in lam],
           *[_p(t) for t in lmem], _p(scratch), *s18, _p(gf), _p(gca), _p(gcb), _p(gca_s),
           _p(gcb_s), *tail, need_ca, need_cb, *flags)
        nat.check("maxwell_3d born_backward")
        ctx.st = None
        return (gca if need_ca else None, gcb if need_cb else None,
                gf if need[2] and ctx.n_src > 0 else None, None, None, None, None)


def _born3d_prep(epsilon, sigma, mu, grid_spacing, dt, source_amplitude, source_location,
                 receiver_location, stencil, pml_width, max_vel, nt, grad_interval,
                 source_component, receiver_component, bg_init):
    """Background problem of a Born run at the CFL-resampled internal step:
    (problem, internal source amplitudes, step ratio, spacing)."""
    if max_vel is None:
        max_vel = float((1.0 / torch.sqrt(epsilon * mu)).max().item()) * ph.C0
    spacing = _spacing(grid_spacing)
    inner_dt, ratio = ph.cfl_condition(spacing, dt, max_vel)
    amp = source_amplitude
    if ratio > 1 and amp is not None and amp.numel() > 0:
        amp = ph.upsample(amp, ratio)
    nt_int = nt * ratio if nt is not None else None
    pb = prepare_em3d(epsilon, sigma, mu, grid_spacing, inner_dt, amp, source_location,
                      receiver_location, stencil=stencil, pml_width=pml_width,
                      source_component=source_component, receiver_component=receiver_component,
                      model_gradient_sampling_interval=grad_interval, nt=nt_int,
                      initial_state=bg_init)
    return pb, amp, ratio, spacing


def born3d(
    epsilon: torch.Tensor, sigma: torch.Tensor, mu: torch.Tensor,
    grid_spacing: float | Sequence[float], dt: float,
    source_amplitude: torch.Tensor | None, source_location: torch.Tensor | None,
    receiver_location: torch.Tensor | None, bg_receiver_location: torch.Tensor | None = None,
    *, depsilon: torch.Tensor | None = None, dsigma: torch.Tensor | None = None,
    dca: torch.Tensor | None = None, dcb: torch.Tensor | None = None, stencil: int = 2,
    pml_width: int | Sequence[int] = 20, max_vel: float | None = None, nt: int | None = None,
    model_gradient_sampling_interval: int = 1, parameterization: str = "epsilon_sigma",
    linearize_source: bool = True, source_component: str = "ey",
    receiver_component: str = "ey", **state_and_unused,
):
    """3-D Born propagator (src/tide/maxwell/maxwell3d_born.py:27): the
    background and the scattered (J(m) v) states advance together in
    maxwell_3d_2_{dtype}_born_forward_cuda.  The perturbation is zero-padded;
    (dca, dcb) from the closed-form coefficient derivative; with
    linearize_source the scattered source is the source pre-scale taken with
    dcb.  Initial states: Ex_0 .. m_ey_x_0 (background) and dEx_0 ..
    dm_ey_x_0 (scattered).  Returns the background final state (18 tensors),
    the scattered final state (18), the background receivers (recorded when
    bg_receiver_location equals receiver_location, else empty) and the
    scattered receivers.  The scattered receivers are differentiable in the
    perturbation (depsilon / dsigma or dca / dcb, and the linearised source),
    through the native Born backward against a device history of the
    background; the background model enters as a constant (its second-order
    terms are not built).  storage_mode is 'device' when a gradient is
    needed."""
    from .born import linearize_material_coefficients

    if epsilon.ndim != 3:
        raise NotImplementedError("born3d supports a single 3-D model only.")
    if parameterization not in ("epsilon_sigma", "ca_cb"):
        raise ValueError("parameterization must be 'epsilon_sigma' or 'ca_cb'")
    if epsilon.device.type != "cuda":
        raise nat.NativeError("libtide_b200 runs on CUDA devices only; there is no CPU path.")
    names = ("Ex", "Ey", "Ez", "Hx", "Hy", "Hz") + MEM_NAMES
    bg_init = [state_and_unused.get(f"{n}_0") for n in names]
    sc_init = [state_and_unused.get(f"d{n}_0") for n in names]
    mu = mu.detach()
    pert = (depsilon, dsigma) if parameterization == "epsilon_sigma" else (dca, dcb)
    # the background model is differentiated (second order, through the joint
    # adjoint) when it requires a gradient; otherwise it enters as values
    bg_grad = torch.is_grad_enabled() and (epsilon.requires_grad or sigma.requires_grad)
    if not bg_grad:
        epsilon, sigma = epsilon.detach(), sigma.detach()
    grad_on = bg_grad or (torch.is_grad_enabled() and any(
        t is not None and t.requires_grad for t in pert))
    with torch.set_grad_enabled(bg_grad):
        prep = _born3d_prep(epsilon, sigma, mu, grid_spacing, dt, source_amplitude,
                            source_location, receiver_location, stencil, pml_width, max_vel,
                            nt, model_gradient_sampling_interval, source_component,
                            receiver_component, bg_init)
    pb, amp, ratio, spacing = prep
    dev, dtype = pb.device, pb.dtype
    pad = [a + b for a, b in zip(pb.fd_pad, pb.pml_width)]
    shape = (pb.nz, pb.ny, pb.nx)

    def zpad(t):
        if t is None or t.numel() == 0:
            return torch.zeros(shape, device=dev, dtype=dtype)
        return torch.nn.functional.pad(t.to(device=dev, dtype=dtype),
                                       ph._torch_pad_order(pad)).contiguous()

    if parameterization == "epsilon_sigma":
        dca_p, dcb_p = linearize_material_coefficients(pb.ca[0], pb.cb[0], pb.dt, zpad(depsilon),
                                                       zpad(dsigma))
    else:
        dca_p, dcb_p = zpad(dca), zpad(dcb)
    dca_p = dca_p.reshape(1, *shape).contiguous()
    dcb_p = dcb_p.reshape(1, *shape).contiguous()
    S, N = pb.n_shots, pb.nz * pb.ny * pb.nx
    n_src = pb.n_src if pb.f.numel() else 0
    if n_src > 0:
        if linearize_source:
            dz, dy, dx = spacing
            dcb_at = dcb_p.reshape(1, N).expand(S, -1).gather(1, pb.sources_i)
            df = (amp.to(dev).permute(2, 0, 1) * dcb_at[None] * (-1.0 / (dx * dy * dz)))
            df = df.reshape(-1).contiguous()
        else:
            df = torch.zeros_like(pb.f)
    else:
        df = torch.empty(0, device=dev, dtype=dtype)
    sc_fields, sc_mem = initial_state_3d(sc_init, pb.layout, pb.fd_pad, dev, dtype)
    same_rec = bg_receiver_location is not None and receiver_location is not None and (
        bg_receiver_location.shape == receiver_location.shape
        and bool(torch.equal(bg_receiver_location.to(dev), receiver_location.to(dev))))
    r = torch.zeros((pb.nt, S, pb.n_rec), device=dev, dtype=dtype)
    bg_r = torch.zeros_like(r) if same_rec else torch.empty(0, device=dev, dtype=dtype)
    # the Born entry points keep full [S, nz, ny, nx] CPML memories
    bg_mem = [pb.layout.unpack(m, a).contiguous() for m, a in zip(pb.memories, MEM_AXES)]
    sc_mem = [pb.layout.unpack(m, a).contiguous() for m, a in zip(sc_mem, MEM_AXES)]

    def head(a, b, f, rr):
        return (_p(pb.ca), _p(pb.cb), _p(pb.cq), _p(a), _p(b), _p(pb.f), _p(f),
                *[_p(t) for t in pb.fields], *[_p(t) for t in bg_mem],
                *[_p(t) for t in sc_fields], *[_p(t) for t in sc_mem], _p(rr), _p(bg_r))

    if grad_on:
        f0 = pb.f if n_src > 0 else torch.empty(0, device=dev, dtype=dtype)
        r = Born3DPropagate.apply(dca_p, dcb_p, df, pb.ca, pb.cb, f0,
                                  {"pb": pb, "head": head, "n_src": n_src})
    else:
        fn = nat.get_backend_function("maxwell_3d", "born_forward", pb.stencil, dtype, dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        fn(*head(dca_p.detach(), dcb_p.detach(), df.detach(), r),
           *_profile_ptrs(pb), _p(pb.sources_i), _p(pb.receivers_i),
           pb.rdz, pb.rdy, pb.rdx, pb.dt, pb.nt, S, pb.nz, pb.ny, pb.nx, n_src, pb.n_rec, 1,
           pb.batched, pb.batched, pb.batched, 0, *pb.pml, pb.src_comp, pb.rec_comp, 0,
           dev.index or 0, 0, stream)
        nat.check("maxwell_3d born_forward")
    if not same_rec and bg_receiver_location is not None and bg_receiver_location.numel() > 0:
        with torch.no_grad():
            bg_r = maxwell3d(epsilon, sigma, mu, grid_spacing, dt, source_amplitude,
                             source_location, bg_receiver_location, stencil=stencil,
                             pml_width=pml_width, max_vel=max_vel, nt=nt,
                             source_component=source_component,
                             receiver_component=receiver_component, storage_mode="none",
                             **{f"{n}_0" if n[0] in "EH" else n: t
                                for n, t in zip(names, bg_init)})[-1]
    elif same_rec and ratio > 1:
        bg_r = ph.downsample(bg_r.movedim(0, -1), ratio).movedim(-1, 0)
    if ratio > 1 and r.numel() > 0:
        r = ph.downsample(r.movedim(0, -1), ratio).movedim(-1, 0)
    s = _crop(pb)

    def outs(fields, mems):
        return [t[s] for t in fields] + [m[s] for m in mems]

    return (*outs(pb.fields, bg_mem), *outs(sc_fields, sc_mem), bg_r, r)
