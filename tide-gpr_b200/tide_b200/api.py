"""Operator-level public API: value objects, MaxwellTM, Maxwell3D, linearization.

Mirrors src/tide/maxwell/contracts.py:24-201, results.py:12-90,
operators.py:26-255 and linearization.py:36-232 (the vjp half; the Born jvp
is not built here).  A user of the reference switches with
``import tide_b200 as tide``.
"""

from __future__ import annotations

from collections.abc import Iterable
from dataclasses import dataclass
from enum import StrEnum
from typing import Literal

import torch

from . import _native as nat
from . import physics as ph
from .storage import StorageOptions
from .tm2d import Callback, maxwelltm
from . import em3d


class BackendPreference(StrEnum):
    AUTO = "auto"
    NATIVE = "native"
    REFERENCE = "reference"


class FallbackPolicy(StrEnum):
    ERROR = "error"
    REFERENCE = "reference"


def _check(ok: bool, message: str) -> None:
    """Raise ValueError(message) unless ok (value-object invariants)."""
    if not ok:
        raise ValueError(message)


def _as_tuple(v) -> tuple:
    return (v,) if isinstance(v, (int, float)) else tuple(v)


@dataclass(frozen=True, slots=True)
class CPML:
    """Convolutional PML boundary configuration."""

    width: int | tuple[int, ...] = 20

    def __post_init__(self) -> None:
        w = _as_tuple(self.width)
        _check(len(w) > 0 and min(w) >= 0, "CPML width(s) must be given and be >= 0.")


@dataclass(frozen=True, slots=True)
class Discretization:
    spacing: float | tuple[float, ...]
    dt: float
    stencil: int = 2
    boundary: CPML = CPML()
    max_velocity: float | None = None

    def __post_init__(self) -> None:
        h = _as_tuple(self.spacing)
        _check(len(h) > 0 and min(h) > 0, "Grid spacing must be > 0 along every axis.")
        _check(self.dt > 0, "dt must be > 0.")
        _check(self.stencil in (2, 4, 6, 8), f"stencil {self.stencil} is not 2, 4, 6 or 8.")
        _check(self.max_velocity is None or self.max_velocity > 0,
               "max_velocity, when given, must be > 0.")


@dataclass(frozen=True, slots=True)
class Acquisition:
    source_location: torch.Tensor | None
    receiver_location: torch.Tensor | None

    @property
    def n_shots(self) -> int:
        for t in (self.source_location, self.receiver_location):
            if t is not None:
                return int(t.shape[0])
        return 1

    @property
    def n_receivers(self) -> int:
        return 0 if self.receiver_location is None else int(self.receiver_location.shape[1])

    @property
    def spatial_ndim(self) -> int | None:
        for t in (self.source_location, self.receiver_location):
            if t is not None:
                return int(t.shape[-1])
        return None


@dataclass(frozen=True, slots=True)
class Experiment:
    acquisition: Acquisition
    source_amplitude: torch.Tensor | None
    nt: int | None = None
    source_component: str = "ey"
    receiver_component: str = "ey"

    def __post_init__(self) -> None:
        _check(self.nt is None or self.nt > 0, "nt, when given, must be > 0.")
        _check(self.nt is not None or self.source_amplitude is not None,
               "Without source amplitudes the number of steps nt must be given.")


@dataclass(frozen=True, slots=True)
class EMModel:
    epsilon: torch.Tensor
    sigma: torch.Tensor
    mu: torch.Tensor
    dispersion: ph.DebyeDispersion | None = None

    def __post_init__(self) -> None:
        ts = (self.epsilon, self.sigma, self.mu)
        for what in ("shape", "device", "dtype"):
            _check(len({getattr(t, what) for t in ts}) == 1,
                   f"The epsilon, sigma and mu tensors differ in {what}.")


@dataclass(frozen=True, slots=True)
class Observers:
    forward: Callback | None = None
    backward: Callback | None = None
    frequency: int = 1

    def __post_init__(self) -> None:
        _check(self.frequency > 0, "Observer frequency must be >= 1.")


@dataclass(frozen=True, slots=True)
class ExecutionOptions:
    backend: BackendPreference = BackendPreference.AUTO
    fallback: FallbackPolicy = FallbackPolicy.ERROR
    reference_mode: Literal["eager", "jit", "compile"] = "eager"
    n_threads: int | None = None


@dataclass(frozen=True, slots=True)
class TMState:
    Ey: torch.Tensor
    Hx: torch.Tensor
    Hz: torch.Tensor
    m_Ey_x: torch.Tensor
    m_Ey_z: torch.Tensor
    m_Hx_z: torch.Tensor
    m_Hz_x: torch.Tensor

    @classmethod
    def from_tensors(cls, tensors) -> TMState:
        _check(len(tensors) == 7, f"A TM state has 7 tensors (Ey, Hx, Hz and four CPML "
                                  f"memories); {len(tensors)} were given.")
        return cls(*tensors)


@dataclass(frozen=True, slots=True)
class EM3DState:
    """Final (or initial) 3-D state: six fields and the twelve CPML memories
    on the model + CPML region (results.py EM3DState)."""

    Ex: torch.Tensor
    Ey: torch.Tensor
    Ez: torch.Tensor
    Hx: torch.Tensor
    Hy: torch.Tensor
    Hz: torch.Tensor
    m_hz_y: torch.Tensor
    m_hy_z: torch.Tensor
    m_hx_z: torch.Tensor
    m_hz_x: torch.Tensor
    m_hy_x: torch.Tensor
    m_hx_y: torch.Tensor
    m_ey_z: torch.Tensor
    m_ez_y: torch.Tensor
    m_ez_x: torch.Tensor
    m_ex_z: torch.Tensor
    m_ex_y: torch.Tensor
    m_ey_x: torch.Tensor

    @classmethod
    def from_tensors(cls, tensors) -> EM3DState:
        _check(len(tensors) == 18, f"A 3-D state has 18 tensors (six fields, twelve CPML "
                                   f"memories); {len(tensors)} were given.")
        return cls(*tensors)

    def tensors(self) -> tuple:
        return tuple(getattr(self, n) for n in em3d.STATE_NAMES)


@dataclass(frozen=True, slots=True)
class ForwardResult:
    receiver_data: torch.Tensor
    final_state: TMState | EM3DState


@dataclass(frozen=True, slots=True)
class EMDirection:
    """A direction in model space (contracts.py:143-166)."""

    epsilon: torch.Tensor | None = None
    sigma: torch.Tensor | None = None
    mu: torch.Tensor | None = None

    def validate_for(self, model: EMModel) -> None:
        given = {n: getattr(self, n) for n in ("epsilon", "sigma", "mu")
                 if getattr(self, n) is not None}
        _check(bool(given), "The direction is empty: give epsilon, sigma and/or mu.")
        for n, d in given.items():
            m = getattr(model, n)
            _check((d.shape, d.device, d.dtype) == (m.shape, m.device, m.dtype),
                   f"The {n} direction differs from the model's {n} in shape, device or dtype.")


@dataclass(frozen=True, slots=True)
class TangentResult:
    """Receiver data and final scattered state of one tangent propagation
    (results.py:67-72)."""

    receiver_data: torch.Tensor
    final_state: TMState | EM3DState


@dataclass(frozen=True, slots=True)
class EMGradient:
    epsilon: torch.Tensor | None
    sigma: torch.Tensor | None
    mu: torch.Tensor | None = None


class MaxwellTM:
    """Differentiable 2-D TM Maxwell operator on the B200 native path."""

    def __init__(
        self,
        discretization: Discretization,
        experiment: Experiment,
        *,
        execution: ExecutionOptions = ExecutionOptions(),
        storage: StorageOptions = StorageOptions(),
        model_gradient_sampling_interval: int = 1,
    ) -> None:
        if experiment.acquisition.spatial_ndim not in {None, 2}:
            raise ValueError("MaxwellTM requires two-dimensional acquisition coordinates.")
        if execution.backend is BackendPreference.REFERENCE:
            raise NotImplementedError(
                "tide_b200 has no reference (torch) backend; the native CUDA path is the product."
            )
        self.discretization = discretization
        self.experiment = experiment
        self.execution = execution
        self.storage = storage
        self.model_gradient_sampling_interval = model_gradient_sampling_interval

    def forward(
        self, model: EMModel, *, state: TMState | None = None, observers: Observers = Observers(),
        retain_history: bool = False,
    ) -> ForwardResult:
        if model.epsilon.ndim not in {2, 3}:
            raise ValueError("MaxwellTM model tensors must be 2-D or batched 3-D tensors.")
        init = (None,) * 7 if state is None else (
            state.Ey, state.Hx, state.Hz, state.m_Ey_x, state.m_Ey_z, state.m_Hx_z, state.m_Hz_x)
        d, e = self.discretization, self.experiment
        out = maxwelltm(
            model.epsilon, model.sigma, model.mu,
            grid_spacing=d.spacing, dt=d.dt, source_amplitude=e.source_amplitude,
            source_location=e.acquisition.source_location,
            receiver_location=e.acquisition.receiver_location,
            stencil=d.stencil, pml_width=d.boundary.width, max_vel=d.max_velocity,
            Ey_0=init[0], Hx_0=init[1], Hz_0=init[2], m_Ey_x=init[3], m_Ey_z=init[4],
            m_Hx_z=init[5], m_Hz_x=init[6], nt=e.nt,
            model_gradient_sampling_interval=self.model_gradient_sampling_interval,
            forward_callback=observers.forward, backward_callback=observers.backward,
            callback_frequency=observers.frequency,
            storage_mode=self.storage.mode.value, storage_path=self.storage.path,
            storage_compression=self.storage.compression,
            storage_bytes_limit_device=self.storage.bytes_limit_device,
            storage_bytes_limit_host=self.storage.bytes_limit_host,
            storage_chunk_steps=self.storage.chunk_steps,
            dispersion=model.dispersion, retain_history=retain_history,
        )
        return ForwardResult(receiver_data=out[-1], final_state=TMState.from_tensors(out[:-1]))

    __call__ = forward

    def linearize(
        self,
        model: EMModel,
        *,
        storage: StorageOptions | None = None,
        targets: Iterable[str] = ("epsilon", "sigma"),
    ) -> LinearizedMaxwellTM:
        return LinearizedMaxwellTM(self, model, storage=storage or self.storage, targets=targets)


class LinearizedMaxwellTM:
    """Linearization of MaxwellTM at a model: primal data and exact VJPs.

    Follows src/tide/maxwell/linearization.py:36-160: the primal runs once
    with the requested targets differentiable and keeps its autograd graph
    (snapshots), and each vjp is one native adjoint pass.
    """

    def __init__(self, operator: MaxwellTM, model: EMModel, *, storage: StorageOptions,
                 targets: Iterable[str]) -> None:
        self.operator = operator
        self.targets = tuple(targets)
        for t in self.targets:
            if t not in ("epsilon", "sigma"):
                raise ValueError(f"unsupported linearization target {t!r}")
        eps = model.epsilon.detach().requires_grad_("epsilon" in self.targets)
        sig = model.sigma.detach().requires_grad_("sigma" in self.targets)
        self._inputs = {"epsilon": eps, "sigma": sig}
        self.model = EMModel(eps, sig, model.mu.detach(), model.dispersion)
        op = MaxwellTM(operator.discretization, operator.experiment, execution=operator.execution,
                       storage=storage,
                       model_gradient_sampling_interval=operator.model_gradient_sampling_interval)
        self._result = op(self.model, retain_history=True)

    @property
    def primal(self) -> ForwardResult:
        return ForwardResult(self._result.receiver_data.detach(), self._result.final_state)

    def vjp(self, cotangent: torch.Tensor, *, retain_graph: bool = True) -> EMGradient:
        ins = [self._inputs[t] for t in self.targets]
        grads = torch.autograd.grad(self._result.receiver_data, ins, grad_outputs=cotangent,
                                    retain_graph=retain_graph, allow_unused=True)
        g = dict(zip(self.targets, grads))
        return EMGradient(epsilon=g.get("epsilon"), sigma=g.get("sigma"))

    def jvp(self, direction: EMDirection) -> TangentResult:
        """Apply the Jacobian J(model) to a model direction: the Born scattered
        receiver data and final scattered state (linearization.py:162-229).
        The direction's epsilon / sigma parts are used; a mu part raises."""
        direction.validate_for(self.model)
        if direction.mu is not None:
            raise NotImplementedError("TM2D tangent propagation for mu is not available.")
        fast = self._jvp_from_history(direction)
        if fast is not None:
            return fast
        from .born import borntm

        op = self.operator
        d, e = op.discretization, op.experiment
        # the background enters as values (no history is kept for it); a
        # direction that requires grad is differentiated through the Born pass
        res = borntm(
            self.model.epsilon.detach(), self.model.sigma.detach(), self.model.mu.detach(),
            grid_spacing=d.spacing,
            dt=d.dt, source_amplitude=e.source_amplitude,
            source_location=e.acquisition.source_location,
            receiver_location=e.acquisition.receiver_location,
            bg_receiver_location=e.acquisition.receiver_location,
            depsilon=direction.epsilon, dsigma=direction.sigma, stencil=d.stencil,
            pml_width=d.boundary.width, max_vel=d.max_velocity, nt=e.nt,
            model_gradient_sampling_interval=op.model_gradient_sampling_interval,
        )
        return TangentResult(res[-1], TMState.from_tensors(res[7:14]))

    def _jvp_from_history(self, direction: EMDirection) -> TangentResult | None:
        """The jvp from the primal's kept background history (the reference's
        reusable linearization background, tm2d_born_autograd.py:134-259):
        only the scattered state advances, reading Ey^n and curl H^n of each
        step from the history (born_tangent_forward_with_storage).  Applies
        when that history is a FULL-format device history at sampling
        interval 1 without sub-stepping and the direction needs no gradient;
        the result is then bit-identical to the full Born pass.  None
        otherwise."""
        from . import storage as stg
        from .born import prepare_born
        from .tm2d import _PROFILE_ORDER, _stream_handle

        node = self._result.receiver_data.grad_fn
        if type(node).__name__ != "TMPropagateBackward":
            return None
        snaps, pb = getattr(node, "snaps", None), getattr(node, "pb", None)
        if (snaps is None or pb is None or snaps.mode != stg.STORAGE_DEVICE or snaps.fmt != 0
                or pb.grad_interval != 1 or pb.batched or pb.debye is not None
                or snaps.ey_dev.numel() == 0 or snaps.curl_dev.numel() == 0):
            return None
        if torch.is_grad_enabled() and any(
                t is not None and t.requires_grad for t in (direction.epsilon, direction.sigma)):
            return None
        d, e = self.operator.discretization, self.operator.experiment
        with torch.no_grad():
            dca, dcb, df = prepare_born(pb, 1, d.spacing, e.source_amplitude,
                                        depsilon=direction.epsilon, dsigma=direction.sigma)
            S = pb.n_shots
            tan = [torch.zeros((S, pb.ny, pb.nx), device=pb.device, dtype=pb.dtype)
                   for _ in range(7)]
            r = torch.zeros((pb.nt, S, pb.n_rec), device=pb.device, dtype=pb.dtype)
            fn = nat.get_backend_function("maxwell_tm", "born_tangent_forward_with_storage",
                                          pb.stencil, pb.dtype, pb.device)
            fn(nat.ptr(pb.ca), nat.ptr(pb.cb), nat.ptr(pb.cq), nat.ptr(dca), nat.ptr(dcb),
               nat.ptr(df), *[nat.ptr(t) for t in tan], nat.ptr(r), nat.ptr(snaps.ey_dev),
               nat.ptr(snaps.curl_dev), 0, 0, *[nat.ptr(pb.profiles[n]) for n in _PROFILE_ORDER],
               nat.ptr(pb.sources_i), nat.ptr(pb.receivers_i), pb.rdy, pb.rdx, pb.dt, pb.nt, S,
               pb.ny, pb.nx, pb.n_src if df.numel() else 0, pb.n_rec, 1, 0, S, False, False,
               False, 0, pb.pml_y0, pb.pml_x0, pb.pml_y1, pb.pml_x1, 0, pb.device.index or 0,
               _stream_handle(pb.device))
            nat.check("maxwell_tm born_tangent_forward_with_storage")
        return TangentResult(r, TMState.from_tensors([pb.crop(t) for t in tan]))

    def second_vjp(self, direction: EMDirection, cotangent: torch.Tensor) -> EMGradient:
        """Gradient of <cotangent, J(model) direction> with respect to the
        linearization targets (linearization.py:125-146): a Born pass at the
        differentiable background, back-propagated through the second-order
        Born adjoint (born_backward_bggrad; device storage)."""
        direction.validate_for(self.model)
        if direction.mu is not None:
            raise NotImplementedError("TM2D tangent propagation for mu is not available.")
        from .born import borntm

        op = self.operator
        d, e = op.discretization, op.experiment
        res = borntm(
            self._inputs["epsilon"], self._inputs["sigma"], self.model.mu.detach(),
            grid_spacing=d.spacing, dt=d.dt, source_amplitude=e.source_amplitude,
            source_location=e.acquisition.source_location,
            receiver_location=e.acquisition.receiver_location,
            depsilon=direction.epsilon, dsigma=direction.sigma, stencil=d.stencil,
            pml_width=d.boundary.width, max_vel=d.max_velocity, nt=e.nt,
            model_gradient_sampling_interval=op.model_gradient_sampling_interval,
        )
        r = res[-1]
        if cotangent.shape != r.shape:
            raise ValueError("The cotangent's shape differs from the tangent receiver data's.")
        ins = [self._inputs[t] for t in self.targets]
        grads = torch.autograd.grad(r, ins, grad_outputs=cotangent, allow_unused=True)
        g = dict(zip(self.targets, grads))
        return EMGradient(epsilon=g.get("epsilon"), sigma=g.get("sigma"))


class Maxwell3D:
    """Differentiable full 3-D (Yee) Maxwell operator on the B200 native path
    (operators.py:132-255)."""

    def __init__(
        self,
        discretization: Discretization,
        experiment: Experiment,
        *,
        execution: ExecutionOptions = ExecutionOptions(),
        storage: StorageOptions = StorageOptions(),
        model_gradient_sampling_interval: int = 1,
    ) -> None:
        if experiment.acquisition.spatial_ndim not in {None, 3}:
            raise ValueError("Maxwell3D requires three-dimensional acquisition coordinates.")
        if execution.backend is BackendPreference.REFERENCE:
            raise NotImplementedError(
                "tide_b200 has no reference (torch) backend; the native CUDA path is the product."
            )
        self.discretization = discretization
        self.experiment = experiment
        self.execution = execution
        self.storage = storage
        self.model_gradient_sampling_interval = model_gradient_sampling_interval

    def forward(
        self, model: EMModel, *, state: EM3DState | None = None, observers: Observers = Observers(),
        retain_history: bool = False,
    ) -> ForwardResult:
        if model.epsilon.ndim not in {3, 4}:
            raise ValueError("Maxwell3D model tensors must be 3-D or batched 4-D tensors.")
        init = dict(zip(("Ex_0", "Ey_0", "Ez_0", "Hx_0", "Hy_0", "Hz_0") + em3d.MEM_NAMES,
                        state.tensors() if state is not None else (None,) * 18))
        d, e = self.discretization, self.experiment
        out = em3d.maxwell3d(
            model.epsilon, model.sigma, model.mu,
            grid_spacing=d.spacing, dt=d.dt, source_amplitude=e.source_amplitude,
            source_location=e.acquisition.source_location,
            receiver_location=e.acquisition.receiver_location,
            stencil=d.stencil, pml_width=d.boundary.width, max_vel=d.max_velocity, nt=e.nt,
            model_gradient_sampling_interval=self.model_gradient_sampling_interval,
            source_component=e.source_component, receiver_component=e.receiver_component,
            forward_callback=observers.forward, backward_callback=observers.backward,
            callback_frequency=observers.frequency,
            storage_mode=self.storage.mode.value, storage_path=self.storage.path,
            storage_compression=self.storage.compression,
            storage_chunk_steps=self.storage.chunk_steps, dispersion=model.dispersion,
            retain_history=retain_history, **init,
        )
        return ForwardResult(receiver_data=out[-1], final_state=EM3DState.from_tensors(out[:-1]))

    __call__ = forward

    def linearize(
        self,
        model: EMModel,
        *,
        storage: StorageOptions | None = None,
        targets: Iterable[str] = ("epsilon", "sigma"),
    ) -> LinearizedMaxwell3D:
        return LinearizedMaxwell3D(self, model, storage=storage or self.storage, targets=targets)


class LinearizedMaxwell3D(LinearizedMaxwellTM):
    """Linearization of Maxwell3D at a model: primal data and exact VJPs
    (linearization.py LinearizedMaxwell3D, the vjp half)."""

    def __init__(self, operator: Maxwell3D, model: EMModel, *, storage: StorageOptions,
                 targets: Iterable[str]) -> None:
        self.operator = operator
        self.targets = tuple(targets)
        for t in self.targets:
            if t not in ("epsilon", "sigma"):
                raise ValueError(f"unsupported linearization target {t!r}")
        eps = model.epsilon.detach().requires_grad_("epsilon" in self.targets)
        sig = model.sigma.detach().requires_grad_("sigma" in self.targets)
        self._inputs = {"epsilon": eps, "sigma": sig}
        self.model = EMModel(eps, sig, model.mu.detach(), model.dispersion)
        op = Maxwell3D(operator.discretization, operator.experiment, execution=operator.execution,
                       storage=storage,
                       model_gradient_sampling_interval=operator.model_gradient_sampling_interval)
        self._result = op(self.model, retain_history=True)

    def jvp(self, direction: EMDirection) -> TangentResult:
        """Born scattered receiver data and final scattered state for a model
        direction (linearization.py:232-300); a mu part raises."""
        direction.validate_for(self.model)
        if direction.mu is not None:
            raise NotImplementedError("3-D tangent propagation for mu is not available.")
        # the background enters as values; a direction that requires grad is
        # differentiated through the Born pass
        res = self._born(self.model.epsilon.detach(), self.model.sigma.detach(), direction,
                         bg_receivers=True)
        return TangentResult(res[-1], EM3DState.from_tensors(res[18:36]))

    def _born(self, eps, sig, direction: EMDirection, bg_receivers: bool = False):
        op = self.operator
        d, e = op.discretization, op.experiment
        return em3d.born3d(
            eps, sig, self.model.mu, grid_spacing=d.spacing,
            dt=d.dt, source_amplitude=e.source_amplitude,
            source_location=e.acquisition.source_location,
            receiver_location=e.acquisition.receiver_location,
            bg_receiver_location=e.acquisition.receiver_location if bg_receivers else None,
            depsilon=direction.epsilon, dsigma=direction.sigma, stencil=d.stencil,
            pml_width=d.boundary.width, max_vel=d.max_velocity, nt=e.nt,
            model_gradient_sampling_interval=op.model_gradient_sampling_interval,
            source_component=e.source_component, receiver_component=e.receiver_component,
        )

    def second_vjp(self, direction: EMDirection, cotangent: torch.Tensor) -> EMGradient:
        """Gradient of <cotangent, J(model) direction> with respect to the
        linearization targets (linearization.py:125-146) through the 3-D
        second-order Born adjoint (born_backward_bggrad)."""
        direction.validate_for(self.model)
        if direction.mu is not None:
            raise NotImplementedError("3-D tangent propagation for mu is not available.")
        r = self._born(self._inputs["epsilon"], self._inputs["sigma"], direction)[-1]
        if cotangent.shape != r.shape:
            raise ValueError("The cotangent's shape differs from the tangent receiver data's.")
        ins = [self._inputs[t] for t in self.targets]
        grads = torch.autograd.grad(r, ins, grad_outputs=cotangent, allow_unused=True)
        g = dict(zip(self.targets, grads))
        return EMGradient(epsilon=g.get("epsilon"), sigma=g.get("sigma"))
