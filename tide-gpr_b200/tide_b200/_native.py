"""ctypes binding of libtide_b200.so (the sm_100a CUDA library).

Mirrors the reference loader (src/tide/backend_utils.py:82-107, 227-308,
823-877): the same declarative argtype specs, the same symbol naming
``maxwell_tm_{accuracy}_{dtype}_{pass}_{device}``, raw ``data_ptr()`` ints.

There is no CPU fallback: if the library is missing or CUDA is unavailable,
every call raises.  After each native call the library's status word is
checked and a failure raises ``NativeError`` with the library's message.
"""

from __future__ import annotations

import ctypes
import pathlib
from ctypes import c_bool, c_double, c_float, c_int, c_int64, c_void_p

import torch

LIB_NAME = "libtide_b200.so"
LIB_PATH = pathlib.Path(__file__).resolve().parent / LIB_NAME


class NativeError(RuntimeError):
    """A libtide_b200 call reported a failure (bad arguments or a CUDA error)."""


_lib: ctypes.CDLL | None = None
_FLOAT = object()  # placeholder replaced by c_float / c_double per dtype

_P, _I, _B = c_void_p, c_int64, c_bool

_TM_PROFILES = [(_P, 8), (_P, 4), (_P, 2)]  # a/b profiles, k profiles, indices
_TM_TAIL = [(_FLOAT, 3), (_I, 1), (_I, 1), (_I, 2), (_I, 2), (_I, 1)]
_TM_FLAGS = [(_B, 3), (_I, 1), (_I, 4), (_I, 1), (_I, 1)]
_TM_STORAGE = [(_I, 3), (_B, 2)]

SPECS: dict[str, list] = {
    # src/tide/backend_utils.py:256-269
    "maxwell_tm_forward": [
        (_P, 3), (_P, 1), (_P, 3), (_P, 4), (_P, 5), (_P, 1), (_I, 1),
        *_TM_PROFILES, *_TM_TAIL, (_B, 1), *_TM_FLAGS, (_P, 1),
    ],
    # src/tide/backend_utils.py:271-287
    "maxwell_tm_forward_with_storage": [
        (_P, 3), (_P, 1), (_P, 3), (_P, 4), (_P, 1), (_P, 6),
        *_TM_PROFILES, *_TM_TAIL, *_TM_STORAGE, *_TM_FLAGS, (_P, 2),
    ],
    # src/tide/backend_utils.py:336-349
    "maxwell_tm_born_forward": [
        (_P, 3), (_P, 2), (_P, 2), (_P, 3), (_P, 4), (_P, 3), (_P, 4), (_P, 2),
        *_TM_PROFILES, *_TM_TAIL, *_TM_FLAGS, (_P, 1),
    ],
    # src/tide/backend_utils.py:351-370
    "maxwell_tm_born_forward_with_storage": [
        (_P, 3), (_P, 2), (_P, 2), (_P, 3), (_P, 4), (_P, 3), (_P, 4), (_P, 2), (_P, 8),
        *_TM_PROFILES, *_TM_TAIL, *_TM_STORAGE, *_TM_FLAGS, (_P, 2),
    ],
    # src/tide/backend_utils.py:372-384
    "maxwell_tm_born_tangent_forward_with_storage": [
        (_P, 3), (_P, 2), (_P, 1), (_P, 7), (_P, 5), *_TM_PROFILES, *_TM_TAIL, (_I, 1), (_I, 1),
        *_TM_FLAGS, (_P, 1),
    ],
    # src/tide/backend_utils.py:386-405
    "maxwell_tm_born_backward": [
        (_P, 3), (_P, 1), (_P, 3), (_P, 4), (_P, 6), (_P, 1), (_P, 2), (_P, 2), (_P, 2),
        *_TM_PROFILES, *_TM_TAIL, *_TM_STORAGE, *_TM_FLAGS, (_P, 2),
    ],
    # src/tide/backend_utils.py:289-308
    "maxwell_tm_backward": [
        (_P, 3), (_P, 1), (_P, 3), (_P, 4), (_P, 1), (_P, 6), (_P, 1), (_P, 2), (_P, 2),
        *_TM_PROFILES, *_TM_TAIL, *_TM_STORAGE, *_TM_FLAGS, (_P, 2),
    ],
    # src/tide/backend_utils.py:407-440
    "maxwell_tm_born_backward_bggrad": [
        (_P, 3), (_P, 2), (_P, 2), (_P, 2), (_P, 6), (_P, 2), (_P, 1), (_I, 1), (_P, 3), (_P, 3),
        (_P, 2), (_P, 2), (_P, 2), (_P, 15), (_P, 1), *_TM_PROFILES, *_TM_TAIL, *_TM_STORAGE,
        (_B, 2), *_TM_FLAGS, (_P, 2),
    ],
    # src/tide/backend_utils.py:310-334 (backward + background_n_shots)
    "maxwell_tm_background_vjp_reuse": [
        (_P, 3), (_P, 1), (_P, 3), (_P, 4), (_P, 1), (_P, 6), (_P, 1), (_P, 2), (_P, 2),
        *_TM_PROFILES, *_TM_TAIL, (_I, 4), (_B, 2), *_TM_FLAGS, (_P, 2),
    ],
}

_3D_TAIL = [(_FLOAT, 3), (_FLOAT, 1), (_I, 1), (_I, 1), (_I, 3), (_I, 2), (_I, 1)]
_3D_FLAGS = [(_B, 3), (_I, 1), (_I, 6), (_I, 2), (_I, 1), (_I, 1), (_I, 1)]
_3D_STORAGE = [(_I, 3), (_B, 2)]
_3D_PROFILES = [(_P, 12), (_P, 6), (_P, 2)]
_3D_FIELDS = [(_P, 6), (_P, 12)]
SPECS.update({
    # src/tide/backend_utils.py:484-504
    "maxwell_3d_forward": [
        (_P, 3), (_P, 1), *_3D_FIELDS, (_P, 9), (_P, 1), (_I, 1), *_3D_PROFILES, *_3D_TAIL,
        (_B, 1), *_3D_FLAGS, (_P, 1),
    ],
    # src/tide/backend_utils.py:506-524
    "maxwell_3d_forward_with_storage": [
        (_P, 3), (_P, 1), *_3D_FIELDS, (_P, 1), (_P, 18), *_3D_PROFILES, *_3D_TAIL,
        *_3D_STORAGE, *_3D_FLAGS, (_P, 2),
    ],
    # src/tide/backend_utils.py:556-577
    "maxwell_3d_born_forward": [
        (_P, 3), (_P, 2), (_P, 2), *_3D_FIELDS, (_P, 6), (_P, 12), (_P, 2), *_3D_PROFILES,
        *_3D_TAIL, *_3D_FLAGS, (_P, 1),
    ],
    # src/tide/backend_utils.py:579-612
    "maxwell_3d_born_forward_with_storage": [
        (_P, 3), (_P, 2), (_P, 2), *_3D_FIELDS, (_P, 6), (_P, 12), (_P, 2), (_P, 18), (_P, 6),
        *_3D_PROFILES, *_3D_TAIL, *_3D_STORAGE, *_3D_FLAGS, (_P, 2),
    ],
    # src/tide/backend_utils.py:614-633
    "maxwell_3d_born_backward": [
        (_P, 3), (_P, 1), *_3D_FIELDS, (_P, 1), (_P, 18), (_P, 1), (_P, 2), (_P, 2),
        *_3D_PROFILES, *_3D_TAIL, *_3D_STORAGE, *_3D_FLAGS, (_P, 2),
    ],
    # src/tide/backend_utils.py:635-671
    "maxwell_3d_born_backward_bggrad": [
        (_P, 3), (_P, 2), (_P, 2), (_P, 1), *_3D_FIELDS, (_P, 6), (_P, 12), (_P, 1), (_P, 18),
        (_P, 6), (_P, 2), (_P, 4), (_P, 4), (_P, 3), *_3D_PROFILES, *_3D_TAIL, (_I, 3), (_B, 4),
        *_3D_FLAGS, (_P, 2),
    ],
    # src/tide/backend_utils.py:537-556
    "maxwell_3d_backward": [
        (_P, 3), (_P, 1), *_3D_FIELDS, (_P, 1), (_P, 18), (_P, 1), (_P, 4), (_P, 2), (_B, 1),
        *_3D_PROFILES, *_3D_TAIL, *_3D_STORAGE, *_3D_FLAGS, (_P, 2),
    ],
})

ACCURACIES = (2, 4, 6, 8)
ACCURACIES_3D = (2, 4, 6, 8)
DTYPES = {torch.float32: "float", torch.float64: "double"}
PASSES = ("forward", "forward_with_storage", "backward")


def argtypes(template: str, dtype_name: str) -> list:
    ftype = c_float if dtype_name == "float" else c_double
    return [ftype if t is _FLOAT else t for t, n in SPECS[template] for _ in range(n)]


def symbol_name(propagator: str, pass_name: str, accuracy: int, dtype_name: str) -> str:
    return f"{propagator}_{accuracy}_{dtype_name}_{pass_name}_cuda"


def library_path() -> pathlib.Path:
    return LIB_PATH


def load() -> ctypes.CDLL:
    """Load the in-tree library once; raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise NativeError(
            f"{LIB_NAME} is not built (expected at {LIB_PATH}); run "
            "`python -c 'import __graft_entry__ as g; g.build()'` from the repository root."
        )
    lib = ctypes.CDLL(str(LIB_PATH))
    lib.tide_cuda_arches.restype = ctypes.c_char_p
    lib.tide_b200_last_status.restype = c_int
    lib.tide_b200_last_error.restype = ctypes.c_char_p
    lib.tide_b200_clear_error.restype = None
    lib.tide_b200_device_status.restype = c_int
    lib.tide_b200_device_status.argtypes = [c_int64]
    _lib = lib
    return lib


def get_backend_function(
    propagator: str, pass_name: str, accuracy: int, dtype: torch.dtype, device: torch.device
):
    """Resolve a native entry point with its argtypes set (device must be cuda)."""
    if device.type != "cuda":
        raise NativeError(
            f"libtide_b200 runs on CUDA devices only (got {device}); there is no CPU path."
        )
    if not torch.cuda.is_available():
        raise NativeError("CUDA is not available; libtide_b200 cannot run.")
    supported = ACCURACIES_3D if propagator == "maxwell_3d" else ACCURACIES
    if accuracy not in supported:
        raise ValueError(f"Unsupported accuracy {accuracy} for {propagator}; supported: {supported}")
    if dtype not in DTYPES:
        raise TypeError(f"Unsupported dtype {dtype}")
    lib = load()
    name = symbol_name(propagator, pass_name, accuracy, DTYPES[dtype])
    fn = getattr(lib, name)
    fn.argtypes = argtypes(f"{propagator}_{pass_name}", DTYPES[dtype])
    fn.restype = None
    return fn


def check(context: str) -> None:
    """Raise NativeError if the last native call recorded a failure."""
    lib = load()
    if lib.tide_b200_last_status() != 0:
        msg = lib.tide_b200_last_error().decode(errors="replace")
        lib.tide_b200_clear_error()
        raise NativeError(f"{context}: {msg}")


def device_status(device: torch.device) -> int:
    """Synchronise and return (then clear) the device-side error word."""
    lib = load()
    return int(lib.tide_b200_device_status(device.index or 0))


def set_fused_threshold(nbytes: int) -> int:
    """Field bytes (3 * shots * ny * nx * 4) above which the stencil-2 FP32
    forward runs the fused one-launch-per-step kernel (0 = always, negative =
    never); returns the previous setting."""
    lib = load()
    lib.tide_b200_set_fused_threshold.argtypes = [ctypes.c_int64]
    lib.tide_b200_set_fused_threshold.restype = ctypes.c_int64
    return int(lib.tide_b200_set_fused_threshold(int(nbytes)))


def set_tma_mode(mode: int) -> int:
    """One-sweep TMA time steps: 0 never (default), 1 on grids of at least 64
    tiles, 2 whenever eligible; returns the previous mode."""
    lib = load()
    lib.tide_b200_set_tma_mode.argtypes = [ctypes.c_int]
    lib.tide_b200_set_tma_mode.restype = ctypes.c_int
    return int(lib.tide_b200_set_tma_mode(int(mode)))


def set_tma_ctas(max_ctas: int) -> int:
    """Upper bound on the TMA path's persistent CTAs (0: one per SM)."""
    lib = load()
    lib.tide_b200_set_tma_ctas.argtypes = [ctypes.c_int]
    lib.tide_b200_set_tma_ctas.restype = ctypes.c_int
    return int(lib.tide_b200_set_tma_ctas(int(max_ctas)))


def set_step_graphs(on: bool) -> bool:
    """Replay blocks of time steps from one captured CUDA graph (default on);
    returns the previous setting."""
    lib = load()
    lib.tide_b200_set_step_graphs.argtypes = [ctypes.c_int]
    lib.tide_b200_set_step_graphs.restype = ctypes.c_int
    return bool(lib.tide_b200_set_step_graphs(1 if on else 0))


def release_scratch(device: torch.device) -> None:
    """Return the library's cached per-call scratch on `device` to the driver."""
    lib = load()
    lib.tide_b200_release_scratch.argtypes = [c_int64]
    lib.tide_b200_release_scratch.restype = c_int
    if lib.tide_b200_release_scratch(device.index or 0) != 0:
        check("release_scratch")


def graph_replays() -> int:
    """Step-block graph replays issued so far by this process."""
    lib = load()
    lib.tide_b200_graph_replays.restype = ctypes.c_int64
    return int(lib.tide_b200_graph_replays())


def ptr(t: torch.Tensor | None) -> int:
    if t is None or t.numel() == 0:
        return 0
    return t.data_ptr()


def exported_symbols() -> list[str]:
    """Every symbol include/*.h declares (used by the load test)."""
    names = [
        symbol_name("maxwell_tm", p, a, d)
        for a in ACCURACIES
        for d in ("float", "double")
        for p in PASSES
    ] + [
        symbol_name("maxwell_tm", p, a, d)
        for a in ACCURACIES
        for d in ("float", "double")
        for p in ("background_vjp_reuse", "born_forward", "born_forward_with_storage",
                  "born_tangent_forward_with_storage", "born_backward", "born_backward_bggrad")
    ] + [
        symbol_name("maxwell_3d", p, a, d)
        for a in ACCURACIES_3D
        for d in ("float", "double")
        for p in ("born_forward", "born_forward_with_storage", "born_backward",
                  "born_backward_bggrad")
    ] + [
        symbol_name("maxwell_3d", p, a, d)
        for a in ACCURACIES_3D
        for d in ("float", "double")
        for p in PASSES
    ]
    return names + [
        "tide_cuda_arches",
        "tide_b200_last_status",
        "tide_b200_last_error",
        "tide_b200_clear_error",
        "tide_b200_device_status",
        "tide_b200_set_fused_threshold",
        "tide_b200_set_tma_mode",
        "tide_b200_set_tma_ctas",
        "tide_b200_set_step_graphs",
        "tide_b200_graph_replays",
        "tide_b200_launch_count",
        "tide_b200_release_scratch",
        "tide_b200_profile_enable",
        "tide_b200_profile_read",
        "tide_b200_profile_kind_name",
        "maxwell_tm_2_float_forward_noalloc_cuda",
        "tide_b200_serve_create",
        "tide_b200_serve_destroy",
        "tide_b200_serve_bind",
        "tide_b200_serve_release",
        "tide_b200_serve_plan",
        "tide_b200_serve_run",
        "tide_b200_serve_launches",
        "tide_b200_serve_configure",
        "tide_b200_serve_set_direct_streams",
    ] + [f"tide_b200_tm_debye_{p}_{d}" for p in ("forward_with_storage", "backward")
         for d in ("float", "double")]
