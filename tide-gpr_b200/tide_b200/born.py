"""Born (tangent) propagation of the TM2D path: ``borntm`` and the jvp of
MaxwellTM linearizations.

Mirrors src/tide/maxwell/tm2d_born.py:26-329 and the host glue of
tm2d_born_cuda.py: the background model is padded and compiled as for
``maxwelltm``; the perturbation (depsilon, dsigma, or dca, dcb directly) is
zero-padded; (dca, dcb) follow from the closed-form derivative of the update
coefficients (src/tide/utils.py:185-217); with ``linearize_source`` the
scattered source is the source pre-scale taken with dcb instead of cb.  The
background and scattered states then advance together in
``maxwell_tm_{S}_{dtype}_born_forward_cuda``.

The scattered field is J(m) v, linear in the perturbation.  When an input
requires a gradient the pass runs as the autograd node ``BornPropagate``
(tm2d_born_autograd.py:38-1210): the forward is
``maxwell_tm_{S}_{dtype}_born_forward_with_storage_cuda`` keeping the
background history; the scattered receivers differentiate in (dca, dcb, df)
through ``born_backward`` (the adjoint over that history) and the background
receivers in the background (ca, cb, f0) through ``backward``.  The
derivative of the scattered receivers in the background model (the
reference's born_backward_bggrad, a second-order term) is not built and
raises.
"""

from __future__ import annotations

from collections.abc import Sequence

import torch

from . import _native as nat
from . import physics as ph
from . import storage as stg
from . import tm2d as _tm
from .tm2d import _PROFILE_ORDER, _stream_handle, build_problem


def linearize_material_coefficients(ca, cb, dt, depsilon_r, dsigma):
    """dca = d ca / d eps_r * depsilon_r + d ca / d sigma * dsigma and the same
    for cb (src/tide/utils.py:185-217), in the reference's operation order."""
    dt_t = torch.as_tensor(dt, device=cb.device, dtype=cb.dtype)
    cb_sq = cb * cb
    dca_de_abs = (1.0 - ca) * cb / dt_t
    dcb_de_abs = -cb_sq / dt_t
    dca_dsigma = -0.5 * (1.0 + ca) * cb
    dcb_dsigma = -0.5 * cb_sq
    dca = dca_de_abs * ph.EP0 * depsilon_r + dca_dsigma * dsigma
    dcb = dcb_de_abs * ph.EP0 * depsilon_r + dcb_dsigma * dsigma
    return dca, dcb


def _zero_pad(t, total, shape, device, dtype):
    if t is None or t.numel() == 0:
        return torch.zeros(shape, device=device, dtype=dtype)
    t = t.to(device=device, dtype=dtype)
    return torch.nn.functional.pad(t, ph._torch_pad_order(total)).contiguous()


def _source_values(amp, coef_at_src, coeff, nt, n_shots, n_src, dtype):
    """Source pre-scale amp * coef(source cell) * coeff, [nt * S * n_src]
    (the same expression as the background's)."""
    src = amp.permute(2, 0, 1).contiguous().to(dtype)
    src = src * coef_at_src.to(dtype).unsqueeze(0)
    src = src * coeff
    return src.reshape(nt * n_shots * n_src).contiguous()


def prepare_born(pb, ratio, grid_spacing, source_amplitude, *, depsilon=None, dsigma=None,
                 dca=None, dcb=None, parameterization="epsilon_sigma", linearize_source=True):
    """Padded coefficient perturbation (dca, dcb) [1, ny, nx] and scattered
    source values df [nt * S * n_src] of a prepared background problem
    (tm2d_born_cuda.py host glue).  Pure tensor preparation on pb's device."""
    dev, dtype = pb.device, pb.dtype
    total = [a + b for a, b in zip(pb.fd_pad, pb.pml_width)]
    shape = (pb.ny, pb.nx)
    if parameterization == "epsilon_sigma":
        deps_p = _zero_pad(depsilon, total, shape, dev, dtype)
        dsig_p = _zero_pad(dsigma, total, shape, dev, dtype)
        dca_p, dcb_p = linearize_material_coefficients(pb.ca[0], pb.cb[0], pb.dt, deps_p, dsig_p)
    else:
        dca_p = _zero_pad(dca, total, shape, dev, dtype)
        dcb_p = _zero_pad(dcb, total, shape, dev, dtype)
    dca_p = dca_p.reshape(1, pb.ny, pb.nx).contiguous()
    dcb_p = dcb_p.reshape(1, pb.ny, pb.nx).contiguous()
    S, N = pb.n_shots, pb.ny * pb.nx
    if pb.n_src > 0 and pb.f.numel() > 0:
        if linearize_source:
            amp = source_amplitude
            if ratio > 1:
                amp = ph.upsample(amp, ratio)
            dcb_at_src = dcb_p.reshape(1, N).expand(S, -1).gather(1, pb.sources_i)
            dy, dx = ph.normalize_spacing_2d(grid_spacing)
            coeff = -1.0 / (dx * dy)  # as the background's pre-scale
            df = _source_values(amp.to(dev), dcb_at_src, coeff, pb.nt, S, pb.n_src, dtype)
        else:
            df = torch.zeros(pb.nt * S * pb.n_src, device=dev, dtype=dtype)
    else:
        df = torch.empty(0, device=dev, dtype=dtype)
    return dca_p, dcb_p, df


def _born_forward_call(pb, dca, dcb, df, f0, tan, r, bg_r, snaps=None, need=(False, False),
                       side=None, direct=(0, 0)):
    """One Born forward over all nt steps: born_forward, or
    born_forward_with_storage when snaps holds a background history (direct:
    addresses of device histories for the scattered dEy^n and dcurl H^n, or
    0)."""
    dev, dtype = pb.device, pb.dtype
    ey, hx, hz, mex, mez, mhx, mhz = pb.fields
    head = [nat.ptr(pb.ca), nat.ptr(pb.cb), nat.ptr(pb.cq), nat.ptr(dca), nat.ptr(dcb),
            nat.ptr(f0), nat.ptr(df), nat.ptr(ey), nat.ptr(hx), nat.ptr(hz), nat.ptr(mex),
            nat.ptr(mez), nat.ptr(mhx), nat.ptr(mhz), *[nat.ptr(t) for t in tan], nat.ptr(r),
            nat.ptr(bg_r)]
    geo = [*[nat.ptr(pb.profiles[n]) for n in _PROFILE_ORDER], nat.ptr(pb.sources_i),
           nat.ptr(pb.receivers_i), pb.rdy, pb.rdx, pb.dt, pb.nt, pb.n_shots, pb.ny, pb.nx,
           pb.n_src if f0.numel() else 0, pb.n_rec, pb.grad_interval]
    tail = [pb.batched, pb.batched, pb.batched, 0, pb.pml_y0, pb.pml_x0, pb.pml_y1, pb.pml_x1, 0,
            dev.index or 0, _stream_handle(dev)]
    if snaps is None:
        fn = nat.get_backend_function("maxwell_tm", "born_forward", pb.stencil, dtype, dev)
        fn(*head, *geo, *tail)
        nat.check("maxwell_tm born_forward")
        return
    fn = nat.get_backend_function("maxwell_tm", "born_forward_with_storage", pb.stencil, dtype,
                                  dev)
    fn(*head, *_tm._snap_ptrs(snaps), *direct, *geo, snaps.mode, snaps.fmt, snaps.shot_bytes,
       need[0], need[1], *tail, int(side.cuda_stream) if side is not None else 0)
    nat.check("maxwell_tm born_forward_with_storage")


def _born_backward_call(pb, grad_r, st, snaps, need_dca, need_dcb, side=None):
    """born_backward over all nt steps: the adjoint of the scattered receivers
    in (dca, dcb, df), accumulated into st (an _AdjointState)."""
    fn = nat.get_backend_function("maxwell_tm", "born_backward", pb.stencil, pb.dtype, pb.device)
    fn(
        nat.ptr(pb.ca), nat.ptr(pb.cb), nat.ptr(pb.cq), nat.ptr(grad_r),
        *[nat.ptr(t) for t in st.lam], *_tm._snap_ptrs(snaps),
        nat.ptr(st.grad_f), nat.ptr(st.grad_ca), nat.ptr(st.grad_cb), nat.ptr(st.shot_ca),
        nat.ptr(st.shot_cb), 0, 0, *_tm._profile_ptrs(pb), nat.ptr(pb.sources_i),
        nat.ptr(pb.receivers_i), pb.rdy, pb.rdx, pb.dt, pb.nt, pb.n_shots, pb.ny, pb.nx,
        pb.n_src, pb.n_rec, pb.grad_interval, snaps.mode, snaps.fmt, snaps.shot_bytes, need_dca,
        need_dcb, pb.batched, pb.batched, pb.batched, pb.nt, pb.pml_y0, pb.pml_x0, pb.pml_y1,
        pb.pml_x1, 0, pb.device.index or 0, _stream_handle(pb.device),
        int(side.cuda_stream) if side is not None else 0,
    )
    nat.check("maxwell_tm born_backward")


def _born_bggrad_call(pb, pert, grad_r, grad_bg_r, snaps, scattered):
    """born_backward_bggrad over all nt steps: the gradients of
    grad_r . scattered + grad_bg_r . background receivers in (dca, dcb, df,
    ca, cb, f0), shaped like those inputs."""
    dev, dt = pb.device, pb.dtype
    S, ny, nx = pb.n_shots, pb.ny, pb.nx
    dca, dcb, df = pert
    full = lambda: torch.zeros((S, ny, nx), device=dev, dtype=dt)  # noqa: E731
    lam, eta = [full() for _ in range(3)], [full() for _ in range(3)]
    mem = [full() for _ in range(8)]
    work = torch.empty((S, ny, nx), device=dev, dtype=dt)
    scratch = torch.empty((8, S, ny, nx), device=dev, dtype=dt)
    mshape = pb.ca.shape
    g_ca, g_cb, g_dca, g_dcb = (torch.zeros(mshape, device=dev, dtype=dt) for _ in range(4))
    n_src = pb.n_src if pb.f.numel() else 0
    g_f0 = torch.zeros(pb.nt * S * n_src, device=dev, dtype=dt)
    g_df = torch.zeros_like(g_f0)
    empty_r = torch.zeros((pb.nt, S, pb.n_rec), device=dev, dtype=dt)
    gr = grad_r.contiguous() if grad_r is not None and grad_r.numel() else empty_r
    gb = grad_bg_r.contiguous() if grad_bg_r is not None and grad_bg_r.numel() else empty_r
    fn = nat.get_backend_function("maxwell_tm", "born_backward_bggrad", pb.stencil, dt, dev)
    fn(nat.ptr(pb.ca), nat.ptr(pb.cb), nat.ptr(pb.cq), nat.ptr(dca), nat.ptr(dcb),
       nat.ptr(pb.f), nat.ptr(df), nat.ptr(gr), nat.ptr(gb), *_tm._snap_ptrs(snaps),
       nat.ptr(scattered[0]), nat.ptr(scattered[1]), 0, S, *[nat.ptr(t) for t in lam],
       *[nat.ptr(t) for t in eta], nat.ptr(g_f0), nat.ptr(g_df), nat.ptr(g_ca), nat.ptr(g_cb),
       nat.ptr(g_dca), nat.ptr(g_dcb), *[nat.ptr(t) for t in mem], 0, nat.ptr(work), 0, 0, 0, 0,
       0, nat.ptr(scratch), *_tm._profile_ptrs(pb), nat.ptr(pb.sources_i),
       nat.ptr(pb.receivers_i), pb.rdy, pb.rdx, pb.dt, pb.nt, S, ny, nx, n_src, pb.n_rec,
       pb.grad_interval, snaps.mode, snaps.fmt, snaps.shot_bytes, True, True, False, False,
       pb.batched, pb.batched, pb.batched, pb.nt, pb.pml_y0, pb.pml_x0, pb.pml_y1, pb.pml_x1, 0,
       dev.index or 0, _stream_handle(dev), 0)
    nat.check("maxwell_tm born_backward_bggrad")
    return g_dca, g_dcb, g_df, g_ca, g_cb, g_f0, None, None, None, None


class BornPropagate(torch.autograd.Function):
    """Autograd node of the Born pass over the perturbation (dca, dcb, df) and
    the background (ca, cb, f0) (tm2d_born_autograd.py:38-1210).

    Outputs: the background final state (7), the scattered final state (7),
    the background receivers and the scattered receivers.  The history of
    the background Ey^n (kept when dca or ca needs a gradient) and curl H^n
    (dcb or cb) is stored in the ``storage_mode`` of opts (device, cpu, disk
    or auto)."""

    @staticmethod
    def forward(ctx, dca, dcb, df, ca, cb, f0, pb, tan, same_rec, opts):
        dev, dtype = pb.device, pb.dtype
        need = tuple(t.requires_grad for t in (dca, dcb, df, ca, cb, f0))
        store_ey, store_curl = need[0] or need[3], need[1] or need[4]
        # the background enters the scattered receivers too: with a background
        # gradient wanted, both histories and the scattered ones are kept for
        # the second-order adjoint (born_backward_bggrad, device mode)
        second = need[3] or need[4] or need[5]
        if second:
            store_ey = store_curl = True
        r = torch.zeros((pb.nt, pb.n_shots, pb.n_rec), device=dev, dtype=dtype)
        bg_r = torch.zeros_like(r) if same_rec else torch.empty(0, device=dev, dtype=dtype)
        snaps = side = None
        if store_ey or store_curl:
            mode_name = str(opts.get("storage_mode", "device")).lower()
            if mode_name == "checkpoint":
                raise NotImplementedError("storage_mode='checkpoint' is not built for the Born "
                                          "pass; use 'device', 'cpu', 'disk' or 'auto'")
            fmt, sdtype = stg.compression_format(opts.get("storage_compression", False), dtype)
            k = pb.grad_interval
            n_store = (pb.nt + k - 1) // k
            mode = stg.resolve_mode(
                mode_name, device=dev, n_store=n_store, n_shots=pb.n_shots, ny=pb.ny, nx=pb.nx,
                itemsize=sdtype.itemsize, n_arrays=int(store_ey) + int(store_curl),
                bytes_limit_device=opts.get("storage_bytes_limit_device"),
                bytes_limit_host=opts.get("storage_bytes_limit_host"),
            )
            if mode == stg.STORAGE_NONE:
                raise ValueError("storage_mode='none' is incompatible with Born gradients")
            snaps = stg.allocate(mode, sdtype, fmt, n_store, pb.n_shots, pb.ny, pb.nx, dev,
                                 store_ey, store_curl, path=opts.get("storage_path") or ".")
            if mode in (stg.STORAGE_CPU, stg.STORAGE_DISK):
                side = torch.cuda.Stream(dev)
                snaps.keep.append(side)
        direct, ctx.scattered = (0, 0), None
        if second and snaps is not None and snaps.mode == stg.STORAGE_DEVICE:
            shape = (snaps.ey_dev.shape[0], pb.n_shots, pb.ny, pb.nx)
            ctx.scattered = [torch.empty(shape, device=dev, dtype=snaps.ey_dev.dtype)
                             for _ in range(2)]
            direct = tuple(nat.ptr(t) for t in ctx.scattered)
        _born_forward_call(pb, dca.detach(), dcb.detach(), df.detach(), f0.detach(), tan, r,
                           bg_r, snaps, (store_ey, store_curl), side, direct)
        ctx.pb, ctx.snaps, ctx.side, ctx.need, ctx.opts = pb, snaps, side, need, opts
        ctx.pert = (dca.detach(), dcb.detach(), df.detach())
        ctx.f0 = f0.detach()
        outs = (*pb.fields, *tan)
        for t in outs:
            ctx.mark_non_differentiable(t)
        return (*outs, bg_r, r)

    @staticmethod
    def backward(ctx, *grads):
        pb, snaps, side = ctx.pb, ctx.snaps, ctx.side
        need_dca, need_dcb, need_df, need_ca, need_cb, need_f0 = ctx.need
        grad_bg_r, grad_r = grads[14], grads[15]
        nonzero = lambda g: g is not None and g.numel() > 0 and bool(g.count_nonzero())  # noqa: E731
        out = [None] * 10
        if nonzero(grad_r) and (need_ca or need_cb or need_f0):
            if ctx.scattered is None:
                raise NotImplementedError(
                    "the derivative of the Born receivers in the background model (second "
                    "order, born_backward_bggrad) needs the histories in device storage mode")
            out = list(_born_bggrad_call(pb, ctx.pert, grad_r, grad_bg_r, snaps, ctx.scattered))
            if not ctx.opts.get("retain_history"):
                ctx.snaps = ctx.scattered = None
            return tuple(out)
        if nonzero(grad_r):
            if need_dca or need_dcb or need_df:
                st = _tm._AdjointState(pb, need_dca, need_dcb, scratch=False)
                _born_backward_call(pb, _tm._grad_r(pb, grad_r), st, snaps, need_dca, need_dcb,
                                    side)
                out[0], out[1], out[2] = st.result(pb, need_dca, need_dcb, need_df)
        if nonzero(grad_bg_r) and (need_ca or need_cb or need_f0):
            out[3], out[4], out[5] = _tm._run_backward(
                pb, pb.ca, pb.cb, grad_bg_r, snaps, need_ca, need_cb, need_f0, ctx.opts)
        if not ctx.opts.get("retain_history"):
            ctx.snaps = None
        return tuple(out)


def borntm(
    epsilon: torch.Tensor,
    sigma: torch.Tensor,
    mu: torch.Tensor,
    grid_spacing: float | Sequence[float],
    dt: float,
    source_amplitude: torch.Tensor | None,
    source_location: torch.Tensor | None,
    receiver_location: torch.Tensor | None,
    bg_receiver_location: torch.Tensor | None = None,
    *,
    depsilon: torch.Tensor | None = None,
    dsigma: torch.Tensor | None = None,
    dca: torch.Tensor | None = None,
    dcb: torch.Tensor | None = None,
    stencil: int = 2,
    pml_width: int | Sequence[int] = 20,
    max_vel: float | None = None,
    Ey_0: torch.Tensor | None = None,
    Hx_0: torch.Tensor | None = None,
    Hz_0: torch.Tensor | None = None,
    m_Ey_x_0: torch.Tensor | None = None,
    m_Ey_z_0: torch.Tensor | None = None,
    m_Hx_z_0: torch.Tensor | None = None,
    m_Hz_x_0: torch.Tensor | None = None,
    dEy_0: torch.Tensor | None = None,
    dHx_0: torch.Tensor | None = None,
    dHz_0: torch.Tensor | None = None,
    dm_Ey_x_0: torch.Tensor | None = None,
    dm_Ey_z_0: torch.Tensor | None = None,
    dm_Hx_z_0: torch.Tensor | None = None,
    dm_Hz_x_0: torch.Tensor | None = None,
    nt: int | None = None,
    model_gradient_sampling_interval: int = 1,
    parameterization: str = "epsilon_sigma",
    linearize_source: bool = True,
    storage_mode: str = "device",
    storage_path: str = ".",
    storage_compression: bool | str = False,
    storage_bytes_limit_device: int | None = None,
    storage_bytes_limit_host: int | None = None,
    retain_history: bool = False,
    **_unused,
):
    """2-D TM Born propagator (src/tide/maxwell/tm2d_born.py:26).

    Returns the background final state (7 tensors), the scattered final state
    (7 tensors), the background receiver data and the scattered receiver data
    [nt, n_shots, n_receivers].  Background receivers are recorded at
    bg_receiver_location: in the same pass when it equals receiver_location,
    else by a separate forward; empty when it is None.

    Differentiable in depsilon / dsigma (or dca / dcb) and the source
    amplitude through the scattered receivers, and in epsilon, sigma, mu and
    the source amplitude through the background receivers; the background
    history for those gradients is kept in ``storage_mode`` (device, cpu,
    disk or auto).  retain_history keeps it after a backward pass."""
    if epsilon.ndim != 2:
        raise NotImplementedError("borntm currently supports a single 2D model only.")
    if parameterization not in ("epsilon_sigma", "ca_cb"):
        raise ValueError("parameterization must be 'epsilon_sigma' or 'ca_cb'")
    if epsilon.device.type != "cuda":
        raise nat.NativeError("libtide_b200 runs on CUDA devices only; there is no CPU path.")
    pb, ratio = build_problem(
        epsilon, sigma, mu, grid_spacing, dt, source_amplitude,
        source_location, receiver_location, stencil=stencil, pml_width=pml_width,
        max_vel=max_vel, initial_state=[Ey_0, Hx_0, Hz_0, m_Ey_x_0, m_Ey_z_0, m_Hx_z_0, m_Hz_x_0],
        nt=nt, model_gradient_sampling_interval=model_gradient_sampling_interval,
    )
    dev, dtype = pb.device, pb.dtype
    S = pb.n_shots
    dca_p, dcb_p, df = prepare_born(pb, ratio, grid_spacing, source_amplitude, depsilon=depsilon,
                                    dsigma=dsigma, dca=dca, dcb=dcb,
                                    parameterization=parameterization,
                                    linearize_source=linearize_source)

    size = (S, pb.ny, pb.nx)
    tan = [ph.pad_field(t, pb.fd_pad, size, dev, dtype)
           for t in (dEy_0, dHx_0, dHz_0, dm_Ey_x_0, dm_Ey_z_0, dm_Hx_z_0, dm_Hz_x_0)]
    for wf, dim in zip(tan[3:], (1, 0, 0, 1)):
        ph.zero_interior(wf, pb.fd_pad, pb.pml_width, dim)

    same_rec = bg_receiver_location is not None and receiver_location is not None and (
        bg_receiver_location.shape == receiver_location.shape
        and bool(torch.equal(bg_receiver_location.to(dev), receiver_location.to(dev))))
    storage = dict(storage_mode=storage_mode, storage_path=storage_path,
                   storage_compression=storage_compression,
                   storage_bytes_limit_device=storage_bytes_limit_device,
                   storage_bytes_limit_host=storage_bytes_limit_host,
                   retain_history=retain_history)
    inputs = (dca_p, dcb_p, df, pb.ca, pb.cb, pb.f)
    if torch.is_grad_enabled() and any(t.requires_grad for t in inputs):
        out = BornPropagate.apply(*inputs, pb, tan, same_rec, storage)
        tan, bg_r, r = list(out[7:14]), out[14], out[15]
    else:
        r = torch.zeros((pb.nt, S, pb.n_rec), device=dev, dtype=dtype)
        bg_r = torch.zeros_like(r) if same_rec else torch.empty(0, device=dev, dtype=dtype)
        _born_forward_call(pb, dca_p.detach(), dcb_p.detach(), df.detach(), pb.f.detach(), tan,
                           r, bg_r)
    if not same_rec and bg_receiver_location is not None and bg_receiver_location.numel() > 0:
        from .tm2d import maxwelltm

        bg_r = maxwelltm(
            epsilon, sigma, mu, grid_spacing, dt, source_amplitude,
            source_location, bg_receiver_location, stencil=stencil, pml_width=pml_width,
            max_vel=max_vel, Ey_0=Ey_0, Hx_0=Hx_0, Hz_0=Hz_0, m_Ey_x=m_Ey_x_0,
            m_Ey_z=m_Ey_z_0, m_Hx_z=m_Hx_z_0, m_Hz_x=m_Hz_x_0, nt=nt,
            **(storage if torch.is_grad_enabled() else dict(storage_mode="none")))[-1]
    elif same_rec and ratio > 1:
        bg_r = ph.downsample(bg_r.movedim(0, -1), ratio).movedim(-1, 0)
    if ratio > 1 and r.numel() > 0:
        r = ph.downsample(r.movedim(0, -1), ratio).movedim(-1, 0)
    return (*[pb.crop(t) for t in pb.fields], *[pb.crop(t) for t in tan], bg_r, r)


__all__ = ["borntm", "linearize_material_coefficients", "prepare_born"]
