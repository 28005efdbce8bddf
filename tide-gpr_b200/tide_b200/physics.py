"""Material coefficients, CPML profiles, padding, CFL, wavelets, resampling.

These are the host-side formulas that turn physical inputs into the arrays
the native kernels consume.  Each follows the reference's published formula
and, because the kernels are checked bit for bit against the reference, the
same floating-point operation order in the model's dtype:

* update coefficients   src/tide/utils.py:13-41  (prepare_parameters)
* Debye coefficients    src/tide/utils.py:117-182 (compile_material_coefficients)
* CPML a/b/k profiles   src/tide/utils.py:220-352, src/tide/staggered.py:6-134
* CFL sub-stepping      src/tide/cfl.py:6-63
* Ricker wavelet        src/tide/wavelets.py:62-82
* padding               src/tide/padding.py:23-166
* band-limited resample src/tide/resampling.py:47-246
"""

from __future__ import annotations

import math
import warnings
from collections.abc import Sequence
from dataclasses import dataclass

import torch

EP0 = 8.8541878128e-12  # vacuum permittivity (F/m)
MU0 = 1.2566370614359173e-06  # vacuum permeability (H/m)
C0 = 1.0 / math.sqrt(EP0 * MU0)  # speed of light in vacuum (m/s)


def prepare_parameters(
    epsilon_r: torch.Tensor, sigma: torch.Tensor, mu_r: torch.Tensor, dt: float
) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    """Return the (ca, cb, cq) Yee update coefficients.

    ca = (1 - s dt / 2e) / (1 + s dt / 2e),  cb = (dt / e) / (1 + s dt / 2e),
    cq = dt / mu, with e = eps_r * EP0 and mu = mu_r * MU0.
    """
    epsilon = epsilon_r * EP0
    mu = mu_r * MU0
    denom = 1.0 + sigma * dt / (2.0 * epsilon)
    ca = (1.0 - sigma * dt / (2.0 * epsilon)) / denom
    cb = (dt / epsilon) / denom
    cq = dt / mu
    return ca, cb, cq


@dataclass(frozen=True, slots=True)
class DebyeDispersion:
    """Multi-pole Debye relaxation: eps(w) = eps_inf + sum_p d_eps_p / (1 + i w tau_p).

    ``delta_epsilon`` and ``tau`` are scalars, model-shaped tensors, or
    ``[n_poles, *model_shape]`` tensors (src/tide/dispersion.py).
    """

    delta_epsilon: torch.Tensor | float
    tau: torch.Tensor | float


def _broadcast_pole_param(value, reference: torch.Tensor, name: str) -> torch.Tensor:
    t = torch.as_tensor(value, device=reference.device, dtype=reference.dtype)
    shape = tuple(reference.shape)
    if t.ndim <= len(shape):
        torch.broadcast_shapes(tuple(t.shape), shape)
        t = t.reshape((1,) + tuple(t.shape))
    elif t.ndim == len(shape) + 1:
        torch.broadcast_shapes(tuple(t.shape[1:]), shape)
    else:
        raise ValueError(f"{name} must be a scalar, model-shaped, or [n_poles, *model_shape]")
    return torch.broadcast_to(t, (t.shape[0], *shape))


def compile_material_coefficients(
    epsilon_r: torch.Tensor,
    sigma: torch.Tensor,
    mu_r: torch.Tensor,
    dt: float,
    dispersion: DebyeDispersion | None = None,
) -> dict:
    """Coefficients for the E/H updates, with Debye polarisation terms if given.

    For Debye media (auxiliary differential equation form):
      a = (2 tau - dt) / (2 tau + dt),  b = EP0 d_eps dt / (2 tau + dt),
      den = eps_inf + s dt / 2 + sum_p b_p,
      ca = (eps_inf - s dt / 2 - sum_p b_p) / den,  cb = dt / den,
      cp = (1 - a) / den.
    """
    if torch.any(epsilon_r <= 0):
        raise ValueError("epsilon must be strictly positive.")
    ca, cb, cq = prepare_parameters(epsilon_r, sigma, mu_r, dt)
    out = {"ca": ca, "cb": cb, "cq": cq, "has_dispersion": False}
    if dispersion is None:
        return out
    d_eps = _broadcast_pole_param(dispersion.delta_epsilon, epsilon_r, "delta_epsilon")
    tau = _broadcast_pole_param(dispersion.tau, epsilon_r, "tau")
    if torch.any(d_eps < 0):
        raise ValueError("delta_epsilon must be non-negative.")
    if torch.any(tau <= 0):
        raise ValueError("tau must be strictly positive.")
    if dt >= float(tau.detach().amin().item()):
        raise ValueError("Debye dispersion requires dt < min(tau).")
    eps_inf = epsilon_r * EP0
    mu = mu_r * MU0
    tau_term = 2.0 * tau + dt
    a = (2.0 * tau - dt) / tau_term
    b = (EP0 * d_eps * dt) / tau_term
    b_sum = b.sum(dim=0)
    den = eps_inf + sigma * dt / 2.0 + b_sum
    out.update(
        ca=(eps_inf - sigma * dt / 2.0 - b_sum) / den,
        cb=dt / den,
        cq=dt / mu,
        has_dispersion=True,
        debye={"a": a, "b": b, "cp": (1.0 - a) / den.unsqueeze(0), "n_poles": int(a.shape[0])},
    )
    return out


# --------------------------------------------------------------------- CPML


def cpml_profile(
    pml_width: Sequence[int],
    pml_start: Sequence[float],
    max_pml: float,
    dt: float,
    n: int,
    dtype: torch.dtype,
    device: torch.device,
    start: float = 0.0,
    n_power: int = 4,
    eps: float = 1e-9,
    grid_spacing: float = 1.0,
    eps_scale: float = EP0,
) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
    """CPML (a, b, kappa) along one axis of n points, sampled at start + i.

    Polynomial grading of order n_power over the layer with
    sigma0 = (n_power + 1) / (150 pi dx), kappa_max = 5, alpha_max = 0.008;
    b = exp(-(sigma / kappa + alpha) dt / EP0),
    a = sigma (b - 1) / (kappa (sigma + kappa alpha) + eps), zero where sigma <= 1e-6.
    """
    k_max, alpha_max = 5.0, 0.008
    a = torch.zeros(n, device=device, dtype=dtype)
    b = torch.zeros(n, device=device, dtype=dtype)
    k = torch.ones(n, device=device, dtype=dtype)
    if max_pml == 0 or (pml_width[0] == 0 and pml_width[1] == 0):
        return a, b, k
    sigma0 = (n_power + 1) / (150.0 * math.pi * grid_spacing)
    x = torch.arange(start, start + n, device=device, dtype=dtype)
    for side in (0, 1):
        if pml_width[side] <= 0:
            continue
        dist = (pml_start[0] - x) if side == 0 else (x - pml_start[1])
        inside = dist >= 0
        frac = torch.clamp(dist / pml_width[side], 0, 1)
        sig = sigma0 * (frac**n_power)
        kap = 1.0 + (k_max - 1.0) * (frac**n_power)
        alp = alpha_max * (1.0 - frac) + 0.1 * alpha_max
        k = torch.where(inside, kap, k)
        bb = torch.exp(-(sig / kap + alp) * dt / eps_scale)
        b = torch.where(inside, bb, b)
        aa = sig * (bb - 1.0) / (kap * (sig + kap * alp) + eps)
        aa = torch.where(sig > 1e-6, aa, torch.zeros_like(aa))
        a = torch.where(inside, aa, a)
    return a, b, k


def set_pml_profiles(
    pml_width: Sequence[int],
    fd_pad: Sequence[int],
    dt: float,
    grid_spacing: Sequence[float],
    dtype: torch.dtype,
    device: torch.device,
    ny: int,
    nx: int,
) -> dict[str, torch.Tensor]:
    """The twelve 1-D profiles of the staggered TM grid.

    Integer-grid profiles (ay, by, ky, ax, bx, kx) sample points i; half-grid
    profiles (ayh, ..., kxh) sample i + 1/2.  The inner edge of each layer
    sits at fd_pad + width from the outer edge.
    """
    pml_start = [
        fd_pad[0] + pml_width[0],
        ny - 1 - fd_pad[1] - pml_width[1],
        fd_pad[2] + pml_width[2],
        nx - 1 - fd_pad[3] - pml_width[3],
    ]
    max_pml = max(
        pml_width[0] * grid_spacing[0],
        pml_width[1] * grid_spacing[0],
        pml_width[2] * grid_spacing[1],
        pml_width[3] * grid_spacing[1],
    )
    out: dict[str, torch.Tensor] = {}
    for axis, n, ws, ps, h in (
        ("y", ny, pml_width[:2], pml_start[:2], grid_spacing[0]),
        ("x", nx, pml_width[2:], pml_start[2:], grid_spacing[1]),
    ):
        for suffix, start in (("", 0.0), ("h", 0.5)):
            a, b, k = cpml_profile(
                ws, ps, max_pml, dt, n, dtype, device, start=start, grid_spacing=h
            )
            out[f"a{axis}{suffix}"] = a.contiguous()
            out[f"b{axis}{suffix}"] = b.contiguous()
            out[f"k{axis}{suffix}"] = k.contiguous()
    return out


def set_pml_profiles_3d(
    pml_width: Sequence[int],
    fd_pad: Sequence[int],
    dt: float,
    grid_spacing: Sequence[float],
    dtype: torch.dtype,
    device: torch.device,
    nz: int,
    ny: int,
    nx: int,
) -> dict[str, torch.Tensor]:
    """The eighteen 1-D profiles of the 3-D Yee grid (src/tide/staggered.py:
    188-330): a, b, kappa on integer points and on half points (suffix h) per
    axis; pml_width and fd_pad are [z0, z1, y0, y1, x0, x1], grid_spacing
    [dz, dy, dx]."""
    sizes = (nz, ny, nx)
    max_pml = max(pml_width[2 * a + s] * grid_spacing[a] for a in range(3) for s in range(2))
    out: dict[str, torch.Tensor] = {}
    for a, name in enumerate("zyx"):
        n = sizes[a]
        ws = pml_width[2 * a:2 * a + 2]
        ps = [fd_pad[2 * a] + ws[0], n - 1 - fd_pad[2 * a + 1] - ws[1]]
        for suffix, start in (("", 0.0), ("h", 0.5)):
            aa, bb, kk = cpml_profile(
                ws, ps, max_pml, dt, n, dtype, device, start=start, grid_spacing=grid_spacing[a]
            )
            out[f"a{name}{suffix}"] = aa.contiguous()
            out[f"b{name}{suffix}"] = bb.contiguous()
            out[f"k{name}{suffix}"] = kk.contiguous()
    return out


# ------------------------------------------------------------------ padding


def _torch_pad_order(pad: Sequence[int]) -> list[int]:
    out: list[int] = []
    for i in range(len(pad) // 2 - 1, -1, -1):
        out.extend([pad[2 * i], pad[2 * i + 1]])
    return out


def replicate_pad(t: torch.Tensor, pad: Sequence[int]) -> torch.Tensor:
    """Replicate-pad the last len(pad)//2 dims of t by pad = [lo0, hi0, lo1,
    hi1, ...] (first padded dim first).  Built from edge slices, expand and
    cat, so its backward (sums over the expanded edges) is deterministic on
    the GPU, unlike the scatter-based backward of the replicate mode of
    torch.nn.functional.pad; the forward values are the same."""
    nd = len(pad) // 2
    for i in range(nd):
        dim = t.ndim - nd + i
        lo, hi = int(pad[2 * i]), int(pad[2 * i + 1])
        if lo == 0 and hi == 0:
            continue
        parts = []
        if lo:
            edge = t.narrow(dim, 0, 1)
            parts.append(edge.expand(*[lo if d == dim else -1 for d in range(t.ndim)]))
        parts.append(t)
        if hi:
            edge = t.narrow(dim, t.shape[dim] - 1, 1)
            parts.append(edge.expand(*[hi if d == dim else -1 for d in range(t.ndim)]))
        t = torch.cat(parts, dim)
    return t


def pad_model(t: torch.Tensor, pad: Sequence[int]) -> torch.Tensor:
    """Replicate-pad a [ny, nx] or [B, ny, nx] model by [y0, y1, x0, x1]."""
    if max(pad) == 0:
        return t.clone()
    return replicate_pad(t, pad).contiguous()


def pad_field(
    t: torch.Tensor | None,
    pad: Sequence[int],
    size: tuple[int, int, int],
    device: torch.device,
    dtype: torch.dtype,
) -> torch.Tensor:
    """Zero-pad an initial wavefield to the padded [S, ny, nx] grid."""
    if t is None or t.numel() == 0:
        return torch.zeros(size, device=device, dtype=dtype)
    if t.ndim == 2:
        t = t[None].expand(size[0], -1, -1)
    t = t.to(device=device, dtype=dtype)
    if tuple(t.shape) == size:
        return t.clone().contiguous()
    return torch.nn.functional.pad(t, _torch_pad_order(pad)).contiguous()


def zero_interior(t: torch.Tensor, fd_pad: Sequence[int], pml_width: Sequence[int], dim: int) -> None:
    """Zero a CPML memory outside its absorbing strips along `dim` (0=y, 1=x)."""
    n = t.shape[1 + dim]
    lo = fd_pad[2 * dim] + pml_width[2 * dim]
    hi = n - pml_width[2 * dim + 1] - fd_pad[2 * dim + 1]
    if dim == 0:
        t[:, lo:hi, :].fill_(0)
    else:
        t[:, :, lo:hi].fill_(0)


# ---------------------------------------------------------------- CFL / time


def cfl_condition(
    grid_spacing: float | Sequence[float], dt: float, max_vel: float, c_max: float = 1.0,
    eps: float = 1e-15,
) -> tuple[float, int]:
    """Largest stable internal dt and the integer sub-step ratio for `dt`."""
    if isinstance(grid_spacing, (int, float)):
        grid_spacing = [float(grid_spacing), float(grid_spacing)]
    if max_vel <= 0:
        raise ValueError("max_vel must be positive")
    max_dt = (c_max / math.sqrt(sum(1 / d**2 for d in grid_spacing)) / (max_vel**2 + eps)) * max_vel
    step_ratio = math.ceil(abs(dt) / max_dt)
    if step_ratio >= 2:
        warnings.warn(
            f"CFL condition requires {step_ratio} internal time steps per user time step.",
            stacklevel=2,
        )
    return dt / step_ratio, step_ratio


def ricker(
    freq: float,
    length: int,
    dt: float,
    peak_time: float | None = None,
    dtype: torch.dtype | None = None,
    device: torch.device | str | None = None,
) -> torch.Tensor:
    """Zero-phase Ricker wavelet with unit peak, (1 - 2 (pi f t)^2) exp(-(pi f t)^2)."""
    if peak_time is None:
        peak_time = 1.0 / freq
    t = torch.arange(
        int(length), dtype=torch.get_default_dtype() if dtype is None else dtype, device=device
    )
    t = t * dt - peak_time
    ph2 = (math.pi * freq * t).square()
    return (1.0 - 2.0 * ph2) * torch.exp(-ph2)


def upsample(signal: torch.Tensor, step_ratio: int) -> torch.Tensor:
    """Band-limited (FFT) upsampling of the last axis by an integer factor."""
    if signal.numel() == 0 or step_ratio == 1:
        return signal
    nt = signal.shape[-1]
    up = nt * step_ratio
    sf = torch.fft.rfft(signal, norm="ortho") * math.sqrt(step_ratio)
    if sf.shape[-1] > 1:
        sf = sf.clone()
        sf[..., -1] = 0
    pad = up // 2 + 1 - sf.shape[-1]
    if pad > 0:
        sf = torch.nn.functional.pad(sf, (0, pad))
    return torch.fft.irfft(sf, n=up, norm="ortho")


def downsample(signal: torch.Tensor, step_ratio: int) -> torch.Tensor:
    """Band-limited (FFT) downsampling of the last axis by an integer factor."""
    if signal.numel() == 0 or step_ratio == 1:
        return signal
    nt = signal.shape[-1] // step_ratio
    sf = torch.fft.rfft(signal, norm="ortho")[..., : nt // 2 + 1]
    if sf.shape[-1] > 1:
        sf = sf.clone()
        sf[..., -1] = 0
    return torch.fft.irfft(sf, n=nt, norm="ortho") / math.sqrt(step_ratio)


def normalize_spacing_2d(spacing: float | Sequence[float]) -> list[float]:
    if isinstance(spacing, (int, float)):
        return [float(spacing)] * 2
    s = list(spacing)
    if len(s) == 1:
        return [float(s[0])] * 2
    if len(s) != 2:
        raise ValueError("2D grid_spacing must have length 1 or 2")
    return [float(s[0]), float(s[1])]


def normalize_pml_width_2d(width: int | Sequence[int]) -> list[int]:
    if isinstance(width, int):
        return [width] * 4
    w = list(width)
    if len(w) == 1:
        return w * 4
    if len(w) == 2:
        return [w[0], w[0], w[1], w[1]]
    if len(w) != 4:
        raise ValueError("2D pml_width must have length 1, 2 or 4")
    return [int(v) for v in w]
