"""tide_b200 — B200-native (sm_100a) TM2D time stepping with TIDE's API.

``import tide_b200 as tide`` gives the operator API of the reference
(``MaxwellTM``, ``Maxwell3D``, ``EMModel``, ``Experiment``, ``Acquisition``,
``Discretization``, ``CPML``, ``StorageOptions``, ``operator.linearize``)
and the functionals ``maxwelltm`` and ``maxwell3d``; all propagation runs in
libtide_b200.so.
"""

from .api import (
    CPML,
    Acquisition,
    BackendPreference,
    Discretization,
    EM3DState,
    EMDirection,
    EMGradient,
    EMModel,
    ExecutionOptions,
    Experiment,
    FallbackPolicy,
    ForwardResult,
    LinearizedMaxwell3D,
    LinearizedMaxwellTM,
    Maxwell3D,
    MaxwellTM,
    Observers,
    TangentResult,
    TMState,
)
from .physics import (
    C0,
    EP0,
    MU0,
    DebyeDispersion,
    cfl_condition,
    downsample,
    prepare_parameters,
    ricker,
    upsample,
)
from .storage import StorageMode, StorageOptions
from .born import borntm
from .em3d import born3d, maxwell3d
from .tm2d import CallbackState, maxwelltm, prepare_tm2d, propagate

__all__ = [
    "CPML", "Acquisition", "BackendPreference", "C0", "CallbackState", "DebyeDispersion",
    "Discretization", "EM3DState", "EMDirection", "EMGradient", "EMModel", "EP0", "ExecutionOptions",
    "Experiment", "FallbackPolicy", "ForwardResult", "LinearizedMaxwell3D",
    "LinearizedMaxwellTM", "MU0", "Maxwell3D", "MaxwellTM", "Observers", "TangentResult",
    "StorageMode", "StorageOptions", "TMState", "born3d", "borntm", "cfl_condition", "downsample", "maxwell3d", "maxwelltm",
    "prepare_parameters", "prepare_tm2d", "propagate", "ricker", "upsample",
]
