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

The scattered field is J(m) v, linear in the perturbation.  This build
returns it without an autograd graph: gradients through ``borntm`` (the
reference's born_backward / born_backward_bggrad) are not built.
"""

from __future__ import annotations

from collections.abc import Sequence

import torch

from . import _native as nat
from . import physics as ph
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


@torch.no_grad()
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
    **_unused,
):
    """2-D TM Born propagator (src/tide/maxwell/tm2d_born.py:26).

    Returns the background final state (7 tensors), the scattered final state
    (7 tensors), the background receiver data and the scattered receiver data
    [nt, n_shots, n_receivers].  Background receivers are recorded at
    bg_receiver_location: in the same pass when it equals receiver_location,
    else by a separate forward; empty when it is None."""
    if epsilon.ndim != 2:
        raise NotImplementedError("borntm currently supports a single 2D model only.")
    if parameterization not in ("epsilon_sigma", "ca_cb"):
        raise ValueError("parameterization must be 'epsilon_sigma' or 'ca_cb'")
    if epsilon.device.type != "cuda":
        raise nat.NativeError("libtide_b200 runs on CUDA devices only; there is no CPU path.")
    pb, ratio = build_problem(
        epsilon.detach(), sigma.detach(), mu.detach(), grid_spacing, dt, source_amplitude,
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
    r = torch.zeros((pb.nt, S, pb.n_rec), device=dev, dtype=dtype)
    bg_r = torch.zeros_like(r) if same_rec else torch.empty(0, device=dev, dtype=dtype)
    fn = nat.get_backend_function("maxwell_tm", "born_forward", pb.stencil, dtype, dev)
    ey, hx, hz, mex, mez, mhx, mhz = pb.fields
    fn(
        nat.ptr(pb.ca), nat.ptr(pb.cb), nat.ptr(pb.cq), nat.ptr(dca_p), nat.ptr(dcb_p),
        nat.ptr(pb.f), nat.ptr(df), nat.ptr(ey), nat.ptr(hx), nat.ptr(hz), nat.ptr(mex),
        nat.ptr(mez), nat.ptr(mhx), nat.ptr(mhz), *[nat.ptr(t) for t in tan], nat.ptr(r),
        nat.ptr(bg_r), *[nat.ptr(pb.profiles[n]) for n in _PROFILE_ORDER],
        nat.ptr(pb.sources_i), nat.ptr(pb.receivers_i), pb.rdy, pb.rdx, pb.dt, pb.nt, S,
        pb.ny, pb.nx, pb.n_src if pb.f.numel() else 0, pb.n_rec, 1, pb.batched, pb.batched,
        pb.batched, 0,
        pb.pml_y0, pb.pml_x0, pb.pml_y1, pb.pml_x1, 0, dev.index or 0, _stream_handle(dev),
    )
    nat.check("maxwell_tm born_forward")
    if not same_rec and bg_receiver_location is not None and bg_receiver_location.numel() > 0:
        from .tm2d import maxwelltm

        bg_r = maxwelltm(
            epsilon.detach(), sigma.detach(), mu.detach(), grid_spacing, dt, source_amplitude,
            source_location, bg_receiver_location, stencil=stencil, pml_width=pml_width,
            max_vel=max_vel, Ey_0=Ey_0, Hx_0=Hx_0, Hz_0=Hz_0, m_Ey_x=m_Ey_x_0,
            m_Ey_z=m_Ey_z_0, m_Hx_z=m_Hx_z_0, m_Hz_x=m_Hz_x_0, nt=nt,
            storage_mode="none")[-1]
    elif same_rec and ratio > 1:
        bg_r = ph.downsample(bg_r.movedim(0, -1), ratio).movedim(-1, 0)
    if ratio > 1 and r.numel() > 0:
        r = ph.downsample(r.movedim(0, -1), ratio).movedim(-1, 0)
    return (*[pb.crop(t) for t in pb.fields], *[pb.crop(t) for t in tan], bg_r, r)


__all__ = ["borntm", "linearize_material_coefficients", "prepare_born"]
