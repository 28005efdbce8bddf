"""Snapshot storage policy and buffers for the gradient path.

Modes and formats share the reference's integer codes
(src/tide/storage.py:18-30, src/tide/csrc/storage/storage_utils.h:9-16):

* ``device`` (0): the whole history ``[n_store, S, ny, nx]`` lives in HBM;
* ``cpu`` (1): a 3-slot device ring plus a pinned host history
  ``[n_store, S, ny*nx]``; the native library copies each stored step to the
  host on a side stream while the next steps compute, and streams it back in
  the adjoint (pinned-host offload);
* ``disk`` (2): a 3-slot device ring, a 3-slot pinned staging ring and one
  temporary file per snapshot kind under ``storage_path``; a writer thread in
  the native library writes each staged step, the adjoint reads it back
  (2-D and 3-D paths);
* ``none`` (3): nothing stored (forward only);
* ``auto``: ``device`` when the history fits the device budget, else ``cpu``;
* ``checkpoint`` (this library's addition): no history; the forward keeps the
  full state every ``storage_chunk_steps`` steps (default about sqrt(nt)) and
  the adjoint recomputes each segment's snapshots into a segment-sized device
  buffer, last segment first.  Memory falls from nt to about 2 sqrt(nt)
  snapshots for one extra forward pass; the gradient is bit-identical to the
  ``device`` mode's.

Formats: ``FULL`` (0) stores the field dtype, ``BF16`` (1) stores bfloat16
(float32 fields only).
"""

from __future__ import annotations

import os
import threading
import weakref

from dataclasses import dataclass, field
from enum import StrEnum

import torch

STORAGE_DEVICE = 0
STORAGE_CPU = 1
STORAGE_DISK = 2
STORAGE_NONE = 3
STORAGE_FORMAT_FULL = 0
STORAGE_FORMAT_BF16 = 1
RING_SLOTS = 3


class StorageMode(StrEnum):
    DEVICE = "device"
    CPU = "cpu"
    DISK = "disk"
    NONE = "none"
    AUTO = "auto"
    CHECKPOINT = "checkpoint"


@dataclass(frozen=True, slots=True)
class StorageOptions:
    """Snapshot storage policy (src/tide/core/types.py:66-88)."""

    mode: StorageMode = StorageMode.DEVICE
    path: str = "."
    compression: bool | str = False
    bytes_limit_device: int | None = None
    bytes_limit_host: int | None = None
    chunk_steps: int = 0

    def __post_init__(self) -> None:
        for name, v in (("bytes_limit_device", self.bytes_limit_device),
                        ("bytes_limit_host", self.bytes_limit_host)):
            if v is not None and v < 0:
                raise ValueError(f"{name} must be non-negative when provided.")
        if self.chunk_steps < 0:
            raise ValueError("storage_chunk_steps must be non-negative.")


def compression_format(compression: bool | str | None, dtype: torch.dtype) -> tuple[int, torch.dtype]:
    """Map the public compression flag to (storage_format, stored dtype)."""
    if compression is True:
        kind = "bf16"
    elif compression is False or compression is None:
        kind = "none"
    elif isinstance(compression, str) and compression.strip().lower() in {"none", "false", "off", "0"}:
        kind = "none"
    elif isinstance(compression, str) and compression.strip().lower() in {"bf16", "bfloat16"}:
        kind = "bf16"
    else:
        raise ValueError("storage_compression must be False/True or one of 'none' or 'bf16'.")
    if kind == "none":
        return STORAGE_FORMAT_FULL, dtype
    if dtype != torch.float32:
        raise NotImplementedError("BF16 snapshot storage is only supported for float32.")
    return STORAGE_FORMAT_BF16, torch.bfloat16


def mode_code(mode: str) -> int:
    m = str(mode).lower()
    codes = {"device": STORAGE_DEVICE, "cpu": STORAGE_CPU, "disk": STORAGE_DISK, "none": STORAGE_NONE}
    if m not in codes:
        raise ValueError(f"storage_mode must be 'device', 'cpu', 'disk', 'none', or 'auto', got {mode!r}")
    return codes[m]


@dataclass(slots=True, weakref_slot=True)
class SnapshotBuffers:
    """Device (and host) buffers for the Ey and curl-H histories."""

    mode: int
    fmt: int
    dtype: torch.dtype
    n_store: int
    shot_bytes: int
    ey_dev: torch.Tensor
    ey_host: torch.Tensor
    curl_dev: torch.Tensor
    curl_host: torch.Tensor
    keep: list = field(default_factory=list)
    files: object = None  # DiskFiles of the disk mode


class DiskFiles:
    """Temporary snapshot files of one disk-mode history (one per snapshot
    kind, under the storage path), removed when the history is released, and
    the char* arrays the native calls take (ey_filenames / curl_filenames;
    the six *_fn of the 3-D path)."""

    def __init__(self, directory: str, *want: bool, tags: tuple[str, ...] = ("ey", "curl")):
        import ctypes
        import tempfile

        self.paths: list[str | None] = []
        self.arrays = []
        for want_k, tag in zip(want, tags, strict=True):
            if not want_k:
                self.paths.append(None)
                self.arrays.append(None)
                continue
            fd, path = tempfile.mkstemp(prefix=f"tide_b200_{tag}_", suffix=".bin",
                                        dir=directory or ".")
            os.close(fd)
            self.paths.append(path)
            self.arrays.append((ctypes.c_char_p * 1)(path.encode()))

    def pointer(self, k: int) -> int:
        import ctypes

        a = self.arrays[k]
        return 0 if a is None else ctypes.addressof(a)

    def __del__(self):
        for p in getattr(self, "paths", []):
            if p:
                try:
                    os.remove(p)
                except OSError:
                    pass


class _HistoryPool:
    """Keeps the most recently released device history of each (shape, dtype,
    device) for the next request of the same shape.

    A shot-batched gradient allocates and releases a device history of
    100+ GB per batch.  Returned to torch's caching allocator, that block can
    be split by the next batch's small allocations, after which the next
    history no longer fits and the allocator frees its cache and calls
    cudaMalloc again (a device synchronisation and a large mapping per
    batch).

    Stream order.  A history is written by the storing forward and read by
    the adjoint on the stream that allocated it (autograd runs a backward
    node on its forward's stream), and it is released by a finalizer as soon
    as the host drops it -- possibly while that adjoint is still queued.  So
    ``give`` records an event on the allocating stream (and on the stream
    current at release) and ``take`` makes the requesting stream wait for
    those events before the buffer is handed out; a history is never
    overwritten by a later batch on another stream before its reader ran.
    ``give`` may run on any thread (garbage collection), so every method
    holds a lock.  ``release_history_pool()`` hands the kept buffers back to
    torch."""

    def __init__(self) -> None:
        self._free: dict = {}
        self._lock = threading.Lock()

    def take(self, shape, dtype, device) -> torch.Tensor:
        key = (tuple(shape), dtype, torch.device(device))
        with self._lock:
            kept = self._free.get(key)
            if kept:
                t, events = kept.pop()
            else:
                self._free.clear()  # other shapes go back to torch before a new block
                t, events = None, ()
        if t is None:
            return torch.empty(shape, device=device, dtype=dtype)
        if events:
            cur = torch.cuda.current_stream(t.device)
            for ev in events:
                cur.wait_event(ev)
        return t

    def give(self, t: torch.Tensor, stream=None) -> None:
        events = []
        if t.device.type == "cuda":
            streams = [torch.cuda.current_stream(t.device)]
            if stream is not None and stream != streams[0]:
                streams.append(stream)
            for s in streams:
                ev = torch.cuda.Event()
                ev.record(s)
                events.append(ev)
        key = (tuple(t.shape), t.dtype, t.device)
        with self._lock:
            if key not in self._free:
                self._free = {key: []}  # keep the latest shape only
            self._free[key].append((t, tuple(events)))

    def clear(self) -> None:
        with self._lock:
            self._free.clear()

    def nbytes(self, device) -> int:
        dev = torch.device(device)
        with self._lock:
            return sum(t.numel() * t.element_size() for k, ts in self._free.items()
                       if k[2] == dev for t, _ in ts)


_POOL = _HistoryPool()


def release_history_pool() -> None:
    """Return the kept device snapshot history to torch's allocator."""
    _POOL.clear()


def history_bytes(n_store: int, n_shots: int, ny: int, nx: int, itemsize: int, n_arrays: int) -> int:
    return n_store * n_shots * ny * nx * itemsize * n_arrays


def resolve_mode(
    mode: str,
    *,
    device: torch.device,
    n_store: int,
    n_shots: int,
    ny: int,
    nx: int,
    itemsize: int,
    n_arrays: int,
    bytes_limit_device: int | None,
    bytes_limit_host: int | None,
) -> int:
    m = str(mode).lower()
    if m != "auto":
        code = mode_code(m)
        return code
    total = history_bytes(n_store, n_shots, ny, nx, itemsize, n_arrays)
    limit_dev = bytes_limit_device
    if limit_dev is None:
        free, _ = torch.cuda.mem_get_info(device)
        limit_dev = int(0.8 * (free + _POOL.nbytes(device)))  # the pool's buffers are free to it
    if total <= limit_dev:
        return STORAGE_DEVICE
    if bytes_limit_host is not None and total > bytes_limit_host:
        raise MemoryError(
            f"snapshot history of {total / 1e9:.1f} GB exceeds both budgets; "
            "use storage_mode='checkpoint'"
        )
    return STORAGE_CPU


def allocate(
    mode: int,
    fmt_dtype: torch.dtype,
    fmt: int,
    n_store: int,
    n_shots: int,
    ny: int,
    nx: int,
    device: torch.device,
    want_ey: bool,
    want_curl: bool,
    path: str = ".",
) -> SnapshotBuffers:
    """Buffers of a snapshot history: device mode the whole history on the
    device; cpu mode a 3-slot device ring and the pinned host history; disk
    mode a 3-slot device ring, a 3-slot pinned staging ring and one
    temporary file per snapshot kind under `path`."""
    empty = torch.empty(0, device=device, dtype=fmt_dtype)
    empty_h = torch.empty(0, dtype=fmt_dtype)
    shot_bytes = ny * nx * fmt_dtype.itemsize

    def one(want: bool) -> tuple[torch.Tensor, torch.Tensor]:
        if not want or mode == STORAGE_NONE:
            return empty, empty_h
        if mode == STORAGE_DEVICE:
            return _POOL.take((n_store, n_shots, ny, nx), fmt_dtype, device), empty_h
        ring = torch.empty((RING_SLOTS, n_shots, ny, nx), device=device, dtype=fmt_dtype)
        n_host = RING_SLOTS if mode == STORAGE_DISK else n_store
        host = torch.empty((n_host, n_shots, ny * nx), dtype=fmt_dtype, pin_memory=True)
        return ring, host

    ed, eh = one(want_ey)
    cd, ch = one(want_curl)
    snaps = SnapshotBuffers(mode, fmt, fmt_dtype, n_store, shot_bytes, ed, eh, cd, ch)
    if mode == STORAGE_DEVICE:
        # released histories go back to the pool (see _HistoryPool)
        dev_t = torch.device(device)
        alloc_stream = torch.cuda.current_stream(dev_t) if dev_t.type == "cuda" else None
        for t in (ed, cd):
            if t.numel():
                weakref.finalize(snaps, _POOL.give, t, alloc_stream)
    if mode == STORAGE_DISK and (want_ey or want_curl):
        snaps.files = DiskFiles(path, want_ey, want_curl)
    return snaps
