"""Continuous-batching server for 2-D TM modeling jobs on one GPU.

The reference runs one ``tide.MaxwellTM`` job per call (all of its shots in
one launch per kernel and step, src/tide/csrc/tm2d/maxwell_tm_cuda_inst.cu:
1281-1609) and has no request loop.  ``TMServer`` accepts forward and
forward+gradient jobs of uneven grid sizes, shot counts and nt, and keeps
every admitted job resident on the device (coefficients, wavefields, CPML
memories, adjoint fields, snapshots or checkpoints) until it is done.  Work
advances in chunks of ``chunk_steps`` time steps; each chunk is one replay of
a captured CUDA graph of the native serving engine (include/tide_b200_serve.h)
whose kernels walk the tiles of all resident jobs, whatever their shapes, so
jobs that arrive while others run join at the next chunk boundary as slots
and device memory free up (continuous batching), and a finished job leaves
without waiting for the others.

Each job is planned from its own shape alone (``plan_job``): forward-only;
gradient with its snapshot history in device memory; or gradient by
checkpoint-and-recompute segments; jobs too large for one slot are split into
contiguous shot groups whose gradients are summed in group order.  The
per-cell arithmetic is that of the per-call kernels, so a job's receivers,
loss and gradients are the same bits alone, in any mix, and through
``tide_b200.maxwelltm`` run with the same plan (``run_plain``).

Loss of a gradient job: 0.5 * sum((r - observed)^2) (observed = 0 when not
given); results are returned on the host.
"""

from __future__ import annotations

import ctypes
import gc
import math
import time
from collections import deque
from collections.abc import Iterable, Sequence
from ctypes import c_double, c_int64, c_void_p
from dataclasses import dataclass, field

import torch

from . import _native as nat
from . import physics as ph
from . import storage as stg
from . import tm2d

# Slot phases and plan flags (include/tide_b200_serve.h).
IDLE, FORWARD, FORWARD_STORE, ADJOINT = 0, 1, 2, 3
FLAG_FUSED = 1
DIRECT_CELLS = 1 << 20  # shots x cells from which a group runs the per-call kernels
DIRECT_STREAMS = 8  # streams of those groups


class _CJob(ctypes.Structure):
    """TideServeJob (include/tide_b200_serve.h)."""

    _fields_ = [
        *[(n, c_int64) for n in ("n_shots", "ny", "nx", "nt", "pml_y0", "pml_x0", "pml_y1",
                                 "pml_x1")],
        ("rdy", c_double), ("rdx", c_double),
        *[(n, c_void_p) for n in tm2d._PROFILE_ORDER],
        *[(n, c_void_p) for n in ("ca", "cb", "cq", "ey", "hx", "hz", "m_ey_x", "m_ey_z",
                                  "m_hx_z", "m_hz_x", "f", "r", "sources_i", "receivers_i")],
        ("n_src", c_int64), ("n_rec", c_int64),
        ("lam", c_void_p * 7), ("lam_scratch", c_void_p), ("grad_r", c_void_p),
        ("grad_f", c_void_p), ("grad_ca", c_void_p), ("grad_cb", c_void_p),
        ("step_ratio", c_int64), ("storage_format", c_int64),
    ]


_BOUND = False


def _lib():
    global _BOUND
    lib = nat.load()
    if not _BOUND:
        P, I = c_void_p, c_int64
        sig = {
            "tide_b200_serve_create": ([I, I, I], P),
            "tide_b200_serve_destroy": ([P], None),
            "tide_b200_serve_bind": ([P, ctypes.POINTER(_CJob), I], I),
            "tide_b200_serve_release": ([P, I], I),
            "tide_b200_serve_plan": ([P, I, I, I, I, P, P, I, I, I], I),
            "tide_b200_serve_configure": ([P, I, I], I),
            "tide_b200_serve_set_direct_streams": ([P, I], I),
            "tide_b200_serve_run": ([P, I, I, I], I),
            "tide_b200_serve_launches": ([P], I),
        }
        for name, (args, res) in sig.items():
            fn = getattr(lib, name)
            fn.argtypes, fn.restype = args, res
        _BOUND = True
    return lib


# ------------------------------------------------------------------ jobs


@dataclass
class ModelingJob:
    """One modeling request: a 2-D TM model, its acquisition and what to return.

    Shapes follow ``tide_b200.maxwelltm``: models [ny, nx]; source_amplitude
    [S, n_src, nt]; locations [S, n, 2] (row, column); observed [nt, S, n_rec].
    """

    epsilon: torch.Tensor
    sigma: torch.Tensor
    mu: torch.Tensor
    grid_spacing: float | Sequence[float]
    dt: float
    source_amplitude: torch.Tensor
    source_location: torch.Tensor
    receiver_location: torch.Tensor
    pml_width: int = 20
    gradient: bool = False
    observed: torch.Tensor | None = None
    model_gradient_sampling_interval: int = 1
    arrival: float = 0.0
    job_id: int = -1

    @property
    def n_shots(self) -> int:
        return int(self.source_amplitude.shape[0])

    @property
    def nt(self) -> int:
        return int(self.source_amplitude.shape[-1])

    def padded_shape(self) -> tuple[int, int]:
        w = int(self.pml_width)
        ny, nx = self.epsilon.shape[-2:]
        return int(ny) + 2 * w + 1, int(nx) + 2 * w + 1  # stencil 2: fd pad [1, 0] per axis

    def cell_updates(self) -> float:
        """Cell updates of the job's useful work: forward (and adjoint) steps
        over the padded grid (recomputation is not counted)."""
        ny, nx = self.padded_shape()
        return float(ny * nx * self.n_shots * self.nt * (2 if self.gradient else 1))


@dataclass
class JobResult:
    job_id: int
    receivers: torch.Tensor  # [nt, S, n_rec] (host)
    loss: float | None
    grad_epsilon: torch.Tensor | None  # [ny, nx] (host)
    grad_sigma: torch.Tensor | None
    arrival: float
    admitted: float
    finished: float
    cell_updates: float

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


# ------------------------------------------------------------------ plans


@dataclass(frozen=True)
class JobPlan:
    """How a job runs: its shot groups (contiguous ranges), gradient mode
    ("forward", "device" history or "checkpoint"), checkpoint segment length
    and the device bytes of each group."""

    groups: tuple[tuple[int, int], ...]
    mode: str
    seg_len: int
    group_bytes: tuple[int, ...]


def group_bytes(ny: int, nx: int, S: int, nt: int, n_src: int, n_rec: int, mode: str,
                seg_len: int, k: int, item: int) -> int:
    """Device bytes of one resident shot group (fields, coefficients,
    amplitudes, receivers, adjoint state, snapshots or checkpoints, the
    padded models kept for the gradient's chain rule, and the pitched copy of
    a fused forward)."""
    N = ny * nx
    SN = S * N
    b = 4 * (3 * N + 7 * SN + nt * S * (n_src + n_rec)) + 8 * S * (n_src + n_rec)
    b += 4 * 12 * max(ny, nx) + 4 * 6 * N
    if mode in ("forward", "device") and SN >= DIRECT_CELLS:
        b += 4 * (12 * S * (ny + 2) + 3 * (ny + 2)) * (nx + 64)
    if mode == "forward":
        return b
    b += 4 * (11 * SN + nt * S * (n_rec + n_src) + 2 * N) + 4 * 6 * N
    if mode == "device":
        return b + 2 * (-(-nt // k)) * SN * item
    n_seg = -(-nt // seg_len)
    return b + n_seg * 7 * SN * 4 + 2 * (-(-seg_len // k)) * SN * item


def plan_job(ny: int, nx: int, S: int, nt: int, n_src: int, n_rec: int, gradient: bool, k: int,
             *, item: int, history_limit: int, group_limit: int, chunk_steps: int) -> JobPlan:
    """Plan a job from its own shape (never from the mix)."""
    k = max(1, min(k, nt)) if nt > 0 else 1
    unit = chunk_steps * k // math.gcd(chunk_steps, k)
    if not gradient:
        mode, seg = "forward", 0
    else:
        hist = 2 * (-(-nt // k)) * S * ny * nx * item
        mode = "device" if hist <= history_limit else "checkpoint"
        seg = 0
        if mode == "checkpoint":
            # segment length minimising checkpoints (7 arrays per segment) plus
            # one segment of snapshots (2 arrays per stored step)
            best = math.sqrt(nt * 7 * 4 * k / (2 * item))
            seg = max(unit, int(round(best / unit)) * unit)
    n_groups = 1
    while True:
        sizes = [S // n_groups + (1 if g < S % n_groups else 0) for g in range(n_groups)]
        nb = [group_bytes(ny, nx, s, nt, n_src, n_rec, mode, seg, k, item) for s in sizes]
        if max(nb) <= group_limit or n_groups == S:
            break
        n_groups += 1
    groups, lo = [], 0
    for s in sizes:
        groups.append((lo, lo + s))
        lo += s
    return JobPlan(tuple(groups), mode, seg, tuple(nb))


def select_admissions(sizes: Sequence[int], resident_bytes: int, n_resident: int, budget: int,
                      max_slots: int, bypassed: int, max_bypass: int) -> tuple[list[int], int]:
    """Which queued groups (sizes in arrival order) to admit now: first fit in
    arrival order within the byte budget and the slot count; groups behind an
    oldest group that does not fit may pass it for at most max_bypass rounds,
    after which nothing passes it until it is admitted.  Returns the indices
    and the updated pass count."""
    take: list[int] = []
    used, slots = resident_bytes, n_resident
    blocked = False
    for i, b in enumerate(sizes):
        fits = slots < max_slots and used + b <= budget
        if not fits:
            if not blocked:
                blocked = True
                bypassed += 1
            continue
        if blocked and bypassed > max_bypass:
            break
        take.append(i)
        used += b
        slots += 1
    if not blocked:
        bypassed = 0
    return take, bypassed


@dataclass
class Segment:
    """A run of one phase: forward steps start .. start+steps-1, or adjoint
    steps start-1 down to start-steps; q0 is the first store index of the
    snapshot buffer; hooks run on the host before its first chunk."""

    phase: int
    start: int
    steps: int
    q0: int = 0
    hooks: tuple[str, ...] = ()


def program(mode: str, nt: int, k: int, seg_len: int) -> list[Segment]:
    """Segments of one shot group, in execution order."""
    if mode == "forward":
        return [Segment(FORWARD, 0, nt)]
    if mode == "device":
        return [Segment(FORWARD_STORE, 0, nt), Segment(ADJOINT, nt, nt, 0, ("grad_r",))]
    starts = list(range(0, nt, seg_len))
    segs = [Segment(FORWARD, s, min(seg_len, nt - s), 0, (f"save:{i}",))
            for i, s in enumerate(starts)]
    for i in range(len(starts) - 1, -1, -1):
        s = starts[i]
        n = min(seg_len, nt - s)
        hooks = (f"restore:{i}",) + (("grad_r",) if i == len(starts) - 1 else ())
        segs.append(Segment(FORWARD_STORE, s, n, s // k, hooks))
        segs.append(Segment(ADJOINT, s + n, n, s // k))
    return segs


# ------------------------------------------------------------------ tasks


class _Task:
    """One shot group of a job on the device."""

    def __init__(self, job: ModelingJob, plan: JobPlan, g: int):
        self.job = job
        self.plan = plan
        self.g = g
        self.lo, self.hi = plan.groups[g]
        self.bytes = plan.group_bytes[g]
        ny, nx = job.padded_shape()
        self.cells = (self.hi - self.lo) * ny * nx  # shots x cells of the group
        nt = job.nt
        k = max(1, min(job.model_gradient_sampling_interval, nt)) if nt > 0 else 1
        self.segments = program(plan.mode, nt, k, plan.seg_len)
        self.seg = 0
        self.pos = 0
        self.adj_steps = 0
        self.slot = -1
        self.admitted = 0.0
        self.done_event: torch.cuda.Event | None = None
        self.out: dict = {}  # device buffers while resident
        self.result: dict = {}  # host results once finished
        self.state: _JobState | None = None

    @property
    def finished_stepping(self) -> bool:
        return self.seg >= len(self.segments)

    def remaining_steps(self) -> int:
        if self.finished_stepping:
            return 0
        return sum(s.steps for s in self.segments[self.seg:]) - self.pos

    def next_plan(self, C: int) -> tuple[Segment, int, int, bool] | None:
        """(segment, t0 for this chunk, steps this chunk, first chunk of segment)."""
        if self.finished_stepping:
            return None
        s = self.segments[self.seg]
        n = min(C, s.steps - self.pos)
        t0 = s.start + self.pos if s.phase != ADJOINT else s.start - self.pos
        return s, t0, n, self.pos == 0

    def advance(self, n: int) -> None:
        s = self.segments[self.seg]
        if s.phase == ADJOINT:
            self.adj_steps += n
        self.pos += n
        if self.pos >= s.steps:
            self.seg += 1
            self.pos = 0


@dataclass
class _JobState:
    job: ModelingJob
    plan: JobPlan
    tasks: list[_Task]
    admitted: float = math.inf
    pending: int = 0
    results: list = field(default_factory=list)


# ------------------------------------------------------------------ server


class TMServer:
    """Persistent request loop over the native serving engine (one GPU).

    memory_budget: device bytes for resident jobs (default 85 % of free
    memory less 2 GiB for the library's per-call scratch); max_slots:
    resident shot groups; chunk_steps: time steps per chunk (the
    continuous-batching granularity); use_graphs: replay a captured CUDA
    graph per chunk; storage_compression: BF16 snapshots for every gradient
    job of this server; history_limit / group_limit: planning thresholds
    (default budget/8 and budget/4); direct_cells: shots x cells from which a
    group runs the per-call kernels on its own stream (and, with fused, the
    fused forward step) instead of the shared tile walk; direct_streams: the
    streams those groups are spread over (1: one after another, each with its
    fields in L2 between its kernels).
    """

    def __init__(self, device: torch.device | str = "cuda", *, memory_budget: int | None = None,
                 max_slots: int = 64, chunk_steps: int = 32, use_graphs: bool = True,
                 storage_compression: bool = False, history_limit: int | None = None,
                 group_limit: int | None = None, max_bypass: int = 8, depth: int = 2,
                 direct_cells: int = DIRECT_CELLS, fused: bool = True, priority: bool = True,
                 max_weight: int = 4, direct_streams: int = DIRECT_STREAMS):
        self.device = torch.device(device)
        if self.device.type != "cuda":
            raise nat.NativeError("TMServer runs on a CUDA device only")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        # the server budgets device memory itself from the free memory: the
        # histories of earlier gradient calls (some held only by reference
        # cycles until a collection) and torch's cached blocks go back to the
        # driver first
        gc.collect()
        stg.release_history_pool()
        torch.cuda.synchronize(self.device)
        torch.cuda.empty_cache()
        nat.release_scratch(self.device)
        self.fmt, self.sdtype = stg.compression_format(storage_compression, torch.float32)
        self.item = self.sdtype.itemsize
        if memory_budget is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            memory_budget = int(0.85 * free) - (2 << 30)  # headroom for per-call scratch
        self.budget = int(memory_budget)
        self.history_limit = int(history_limit if history_limit is not None else self.budget // 8)
        self.group_limit = int(group_limit if group_limit is not None else self.budget // 4)
        self.max_slots = int(max_slots)
        self.C = int(chunk_steps)
        self.use_graphs = bool(use_graphs)
        self.max_bypass = int(max_bypass)
        self.depth = max(1, int(depth))
        self.lib = _lib()
        self.engine = self.lib.tide_b200_serve_create(self.device.index, self.max_slots, self.fmt)
        nat.check("serve create")
        if not self.engine:
            raise nat.NativeError("serve create failed")
        self.lib.tide_b200_serve_configure(self.engine, int(direct_cells), int(fused))
        nat.check("serve configure")
        if self.lib.tide_b200_serve_set_direct_streams(self.engine, int(direct_streams)) < 0:
            nat.check("serve set_direct_streams")
        self.direct_cells = int(direct_cells)
        self.priority = bool(priority)
        self.max_weight = max(1, int(max_weight))
        self.stream = torch.cuda.Stream(self.device)
        self.queue: deque[_Task] = deque()
        self.resident: list[_Task] = []
        self.finishing: list[_Task] = []
        self.resident_bytes = 0
        self.inflight: deque[torch.cuda.Event] = deque()
        self.completed: list[JobResult] = []
        self.t0 = time.perf_counter()
        self.bypassed = 0
        self.chunks = 0
        self.stats = {"admitted": 0, "chunks": 0, "max_resident": 0, "max_bytes": 0,
                      "deferred_oom": 0}

    # -------------------------------------------------------------- public

    def close(self) -> None:
        if getattr(self, "engine", None):
            torch.cuda.synchronize(self.device)
            self.lib.tide_b200_serve_destroy(self.engine)
            self.engine = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass

    def now(self) -> float:
        return time.perf_counter() - self.t0

    def plan(self, job: ModelingJob) -> JobPlan:
        ny, nx = job.padded_shape()
        return plan_job(ny, nx, job.n_shots, job.nt, int(job.source_location.shape[1]),
                        int(job.receiver_location.shape[1]), job.gradient,
                        job.model_gradient_sampling_interval, item=self.item,
                        history_limit=self.history_limit, group_limit=self.group_limit,
                        chunk_steps=self.C)

    def submit(self, job: ModelingJob) -> None:
        """Queue a job (its arrival time is taken as now if not set)."""
        plan = self.plan(job)
        if max(plan.group_bytes) > self.budget:
            raise MemoryError(f"job {job.job_id} needs {max(plan.group_bytes) / 1e9:.1f} GB per "
                              f"shot group; the budget is {self.budget / 1e9:.1f} GB")
        js = _JobState(job, plan, [])
        js.tasks = [_Task(job, plan, g) for g in range(len(plan.groups))]
        js.pending = len(js.tasks)
        for t in js.tasks:
            t.state = js
            self.queue.append(t)

    def idle(self) -> bool:
        return not self.queue and not self.resident and not self.finishing

    def step(self) -> list[JobResult]:
        """Admit, run one chunk, retire; returns the jobs completed since the
        last call."""
        with torch.cuda.stream(self.stream):
            self._admit()
            if self.resident:
                self._run_chunk()
            self._collect(block=not self.resident and bool(self.finishing))
        out, self.completed = self.completed, []
        return out

    def serve(self, jobs: Iterable[ModelingJob], *, realtime: bool = True) -> list[JobResult]:
        """Run a stream of jobs to completion.  With realtime, a job is
        submitted when the wall clock passes its arrival time (seconds from
        the start of the call); else all are submitted at once."""
        pending = sorted(jobs, key=lambda j: j.arrival)
        self.t0 = time.perf_counter()
        results: list[JobResult] = []
        i = 0
        while i < len(pending) or not self.idle():
            now = self.now()
            while i < len(pending) and (not realtime or pending[i].arrival <= now):
                if not realtime:
                    pending[i].arrival = 0.0
                self.submit(pending[i])
                i += 1
            if self.idle():
                time.sleep(max(0.0, min(0.01, pending[i].arrival - self.now())))
                continue
            results.extend(self.step())
        return results

    def launches(self) -> int:
        return int(self.lib.tide_b200_serve_launches(self.engine))

    # -------------------------------------------------------------- admission

    def _admit(self) -> None:
        now = self.now()
        arrived = [t for t in self.queue if t.job.arrival <= now]
        take, self.bypassed = select_admissions(
            [t.bytes for t in arrived], self.resident_bytes, len(self.resident), self.budget,
            self.max_slots, self.bypassed, self.max_bypass)
        for i in take:
            if not self._load_or_defer(arrived[i]):
                break  # device memory is fragmented: the rest waits for a job to leave
            self.queue.remove(arrived[i])
        self.stats["max_resident"] = max(self.stats["max_resident"], len(self.resident))
        self.stats["max_bytes"] = max(self.stats["max_bytes"], self.resident_bytes)

    def _load_or_defer(self, t: _Task) -> bool:
        """Load a task admitted by the byte budget.  The budget counts bytes,
        but torch's caching allocator can be too fragmented to place a large
        block: then the cached blocks go back to the driver and the load is
        tried once more; if it still fails the task stays queued while other
        jobs are resident (False), and the error propagates when none is."""
        for attempt in range(2):
            try:
                self._load(t)
                return True
            except torch.OutOfMemoryError:
                t.out.clear()  # drop what the failed load allocated
                torch.cuda.synchronize(self.device)
                torch.cuda.empty_cache()
                if attempt == 1 and self.resident:
                    self.stats["deferred_oom"] += 1
                    return False
                if attempt == 1:
                    raise
        return False

    def _load(self, t: _Task) -> None:
        """Prepare a shot group on the device and bind it to a slot."""
        job, dev = t.job, self.device
        sl = slice(t.lo, t.hi)
        grad = job.gradient
        eps = job.epsilon.to(dev, torch.float32)
        sig = job.sigma.to(dev, torch.float32)
        if grad:
            eps = eps.detach().requires_grad_(True)
            sig = sig.detach().requires_grad_(True)
        with torch.set_grad_enabled(grad):
            pb, ratio = tm2d.build_problem(
                eps, sig, job.mu.to(dev, torch.float32), job.grid_spacing, job.dt,
                job.source_amplitude[sl].to(dev, torch.float32),
                job.source_location[sl].to(dev), job.receiver_location[sl].to(dev),
                stencil=2, pml_width=job.pml_width,
                model_gradient_sampling_interval=job.model_gradient_sampling_interval,
            )
        if ratio != 1:
            raise ValueError(f"job {job.job_id}: dt exceeds the CFL limit (sub-step ratio "
                             f"{ratio}); the served path needs dt within it")
        S, N = pb.n_shots, pb.ny * pb.nx
        z = lambda *shape: torch.zeros(shape, device=dev, dtype=torch.float32)  # noqa: E731
        r = z(pb.nt, S, pb.n_rec) if pb.n_rec > 0 else z(0)
        o = t.out
        o.update(pb=pb, r=r, eps=eps, sig=sig, ratio=ratio)
        cj = _CJob()
        cj.n_shots, cj.ny, cj.nx, cj.nt = S, pb.ny, pb.nx, pb.nt
        cj.pml_y0, cj.pml_x0, cj.pml_y1, cj.pml_x1 = pb.pml_y0, pb.pml_x0, pb.pml_y1, pb.pml_x1
        cj.rdy, cj.rdx = pb.rdy, pb.rdx
        for name in tm2d._PROFILE_ORDER:
            setattr(cj, name, nat.ptr(pb.profiles[name]))
        cj.ca, cj.cb, cj.cq = nat.ptr(pb.ca), nat.ptr(pb.cb), nat.ptr(pb.cq)
        (cj.ey, cj.hx, cj.hz, cj.m_ey_x, cj.m_ey_z, cj.m_hx_z,
         cj.m_hz_x) = [nat.ptr(f) for f in pb.fields]
        cj.f, cj.r = nat.ptr(pb.f), nat.ptr(r)
        cj.sources_i, cj.receivers_i = nat.ptr(pb.sources_i), nat.ptr(pb.receivers_i)
        cj.n_src, cj.n_rec = pb.n_src, pb.n_rec
        cj.step_ratio, cj.storage_format = pb.grad_interval, self.fmt
        if grad:
            lam = [z(S, pb.ny, pb.nx) for _ in range(7)]
            scratch = z(4, S, pb.ny, pb.nx)
            grad_r = z(pb.nt, S, pb.n_rec) if pb.n_rec > 0 else z(0)
            grad_f = z(pb.nt, S, pb.n_src) if pb.n_src > 0 else z(0)
            gca, gcb = z(pb.ny, pb.nx), z(pb.ny, pb.nx)
            k = pb.grad_interval
            if t.plan.mode == "device":
                n_slots = -(-pb.nt // k)
            else:
                n_slots = -(-t.plan.seg_len // k)
                o["ckpt"] = [[torch.empty_like(f) for f in pb.fields]
                             for _ in range(-(-pb.nt // t.plan.seg_len))]
            snaps = [torch.empty((n_slots, S, pb.ny, pb.nx), device=dev, dtype=self.sdtype)
                     for _ in range(2)]
            o.update(lam=lam, scratch=scratch, grad_r=grad_r, grad_f=grad_f, gca=gca, gcb=gcb,
                     snaps=snaps)
            for i, a in enumerate(lam):
                cj.lam[i] = nat.ptr(a)
            cj.lam_scratch = nat.ptr(scratch)
            cj.grad_r, cj.grad_f = nat.ptr(grad_r), nat.ptr(grad_f)
            cj.grad_ca, cj.grad_cb = nat.ptr(gca), nat.ptr(gcb)
        slot = int(self.lib.tide_b200_serve_bind(self.engine, ctypes.byref(cj),
                                                 self.stream.cuda_stream))
        nat.check("serve bind")
        if slot < 0:
            raise nat.NativeError("serve bind failed")
        t.slot = slot
        t.admitted = self.now()
        t.state.admitted = min(t.state.admitted, t.admitted)
        self.resident.append(t)
        self.resident_bytes += t.bytes
        self.stats["admitted"] += 1

    # -------------------------------------------------------------- chunks

    def _hook(self, t: _Task, name: str) -> None:
        o = t.out
        fields = o["pb"].fields
        if name == "grad_r":
            obs = t.job.observed
            r = o["r"]
            if r.numel():
                if obs is not None:
                    o["grad_r"].copy_(r - obs[:, t.lo:t.hi].to(r.device, r.dtype))
                else:
                    o["grad_r"].copy_(r)
        elif name.startswith("save:"):
            for dst, src in zip(o["ckpt"][int(name[5:])], fields):
                dst.copy_(src)
        elif name.startswith("restore:"):
            for dst, src in zip(fields, o["ckpt"][int(name[8:])]):
                dst.copy_(src)

    def _weights(self) -> dict:
        """Steps per chunk of each resident group, in units of chunk_steps:
        groups on their own streams (per-call kernels) with more remaining
        steps than the median run up to max_weight chunks' worth, so the
        longest jobs (checkpointed gradients: three passes) are not left to
        finish alone after the others."""
        if not self.priority:
            return {}
        rem = sorted(t.remaining_steps() for t in self.resident)
        if not rem:
            return {}
        ref = max(1, rem[len(rem) // 2])
        w = {}
        for t in self.resident:
            if t.cells >= self.direct_cells >= 0:
                w[id(t)] = max(1, min(self.max_weight, t.remaining_steps() // ref))
        return w

    def _run_chunk(self) -> None:
        C = self.C
        planned = []
        weights = self._weights()
        for t in self.resident:
            p = t.next_plan(C * weights.get(id(t), 1))
            if p is None:
                continue
            seg, t0, n, first = p
            if first:
                for h in seg.hooks:
                    self._hook(t, h)
            ey = cu = None
            if seg.phase in (FORWARD_STORE, ADJOINT):
                ey, cu = (nat.ptr(s) for s in t.out["snaps"])
            # fields of forward-only and device-history forwards are not read
            # afterwards (checkpoint segments copy theirs)
            flags = FLAG_FUSED if (seg.phase != ADJOINT and
                                   t.plan.mode in ("forward", "device")) else 0
            self.lib.tide_b200_serve_plan(self.engine, t.slot, seg.phase, t0, n, ey, cu, seg.q0,
                                          t.adj_steps, flags)
            nat.check("serve plan")
            planned.append((t, n))
        if not planned:
            return
        # the engine's own scratch (pitched copies, tile lists) comes from the
        # driver: torch's cached blocks go back when the driver runs short
        if torch.cuda.mem_get_info(self.device)[0] < (4 << 30):
            torch.cuda.empty_cache()
        rc = self.lib.tide_b200_serve_run(self.engine, C, int(self.use_graphs),
                                          self.stream.cuda_stream)
        nat.check("serve run")
        if rc != 0:
            raise nat.NativeError("serve run failed")
        self.chunks += 1
        self.stats["chunks"] += 1
        for t, n in planned:
            t.advance(n)
        ev = torch.cuda.Event()
        ev.record(self.stream)
        self.inflight.append(ev)
        while len(self.inflight) > self.depth:
            self.inflight.popleft().synchronize()
        for t in [t for t in self.resident if t.finished_stepping]:
            self._finish(t)

    def _finish(self, t: _Task) -> None:
        """Enqueue a finished group's gradient chain rule and host copies;
        release its slot (the engine frees it once its chunks are done)."""
        o, job = t.out, t.job
        pb = o["pb"]
        r = o["r"]
        res = {"r": r.to("cpu", non_blocking=True) if r.numel() else r.cpu()}
        if job.gradient:
            d = r - job.observed[:, t.lo:t.hi].to(r.device, r.dtype) if job.observed is not None else r
            loss = 0.5 * (d**2).sum()
            outs, grads = [pb.ca, pb.cb], [o["gca"].unsqueeze(0), o["gcb"].unsqueeze(0)]
            if pb.n_src > 0 and pb.f.requires_grad:
                outs.append(pb.f)
                grads.append(o["grad_f"].reshape(-1))
            ge, gs = torch.autograd.grad(outs, [o["eps"], o["sig"]], grads, allow_unused=True)
            res.update(loss=loss.to("cpu", non_blocking=True),
                       ge=ge.to("cpu", non_blocking=True) if ge is not None else None,
                       gs=gs.to("cpu", non_blocking=True) if gs is not None else None)
        ev = torch.cuda.Event()
        ev.record(self.stream)
        t.done_event = ev
        t.result = res
        self.lib.tide_b200_serve_release(self.engine, t.slot)
        nat.check("serve release")
        self.resident.remove(t)
        self.resident_bytes -= t.bytes
        t.out = {}
        self.finishing.append(t)

    def _collect(self, block: bool) -> None:
        for t in list(self.finishing):
            if block:
                t.done_event.synchronize()
            elif not t.done_event.query():
                continue
            self.finishing.remove(t)
            js = t.state
            js.results.append((t.g, t.result))
            js.pending -= 1
            if js.pending == 0:
                self.completed.append(self._assemble(js))
                # when torch's cache has grown past the budget (freed blocks
                # kept by the caching allocator), a finished job's blocks go
                # back to the driver, where the library's per-call scratch
                # (stream-ordered pool) can use them; otherwise they stay
                # cached (returning them synchronises the device)
                if torch.cuda.memory_reserved(self.device) > self.budget:
                    torch.cuda.empty_cache()

    def _assemble(self, js: _JobState) -> JobResult:
        job = js.job
        parts = [res for _, res in sorted(js.results, key=lambda x: x[0])]
        r = torch.cat([p["r"] for p in parts], dim=1) if parts[0]["r"].numel() else parts[0]["r"]
        loss = ge = gs = None
        if job.gradient:
            loss = 0.0
            for p in parts:
                loss += float(p["loss"])
                if p["ge"] is not None:
                    ge = p["ge"] if ge is None else ge + p["ge"]
                if p["gs"] is not None:
                    gs = p["gs"] if gs is None else gs + p["gs"]
        return JobResult(job.job_id, r, loss, ge, gs, job.arrival, js.admitted, self.now(),
                         job.cell_updates())


# ------------------------------------------------------------------ plain path


def run_plain(job: ModelingJob, plan: JobPlan, device: torch.device | str = "cuda",
              storage_compression: bool = False) -> JobResult:
    """The same job through ``tide_b200.maxwelltm`` one shot group at a time
    (the per-job path the server is compared with); the result's `finished`
    (and latency) is the job's own wall time."""
    dev = torch.device(device)
    t_start = time.perf_counter()
    rs, loss, ge, gs = [], None, None, None
    mode = {"forward": "device", "device": "device", "checkpoint": "checkpoint"}[plan.mode]
    for lo, hi in plan.groups:
        eps = job.epsilon.to(dev, torch.float32)
        sig = job.sigma.to(dev, torch.float32)
        if job.gradient:
            eps = eps.detach().requires_grad_(True)
            sig = sig.detach().requires_grad_(True)
        with torch.set_grad_enabled(job.gradient):
            out = tm2d.maxwelltm(
                eps, sig, job.mu.to(dev, torch.float32), job.grid_spacing, job.dt,
                job.source_amplitude[lo:hi].to(dev, torch.float32),
                job.source_location[lo:hi].to(dev), job.receiver_location[lo:hi].to(dev),
                pml_width=job.pml_width,
                model_gradient_sampling_interval=job.model_gradient_sampling_interval,
                storage_mode=mode, storage_compression=storage_compression,
                storage_chunk_steps=plan.seg_len,
            )
        r = out[-1]
        rs.append(r.detach().cpu())
        if job.gradient:
            d = r - job.observed[:, lo:hi].to(dev, r.dtype) if job.observed is not None else r
            lg = 0.5 * (d**2).sum()
            g1, g2 = torch.autograd.grad(lg, [eps, sig])
            loss = float(lg.detach()) if loss is None else loss + float(lg.detach())
            ge = g1.cpu() if ge is None else ge + g1.cpu()
            gs = g2.cpu() if gs is None else gs + g2.cpu()
    torch.cuda.synchronize(dev)
    t_end = time.perf_counter()
    return JobResult(job.job_id, torch.cat(rs, dim=1), loss, ge, gs, 0.0, 0.0, t_end - t_start,
                     job.cell_updates())


# ------------------------------------------------------------------ stream


def mixed_stream(n_jobs: int, seed: int = 3, rate: float | None = None, *,
                 nz_range=(128, 1024), nx_range=(256, 2048), nt_range=(1000, 6000),
                 shots_range=(1, 32), gradient_fraction: float = 0.3, pml: int = 20,
                 dx: float = 0.02, freq: float = 400e6, nt_scale: float = 1.0) -> list[ModelingJob]:
    """Seeded mixed-size 2-D TM job stream (synthetic): nz and nx log-uniform,
    nt and shots uniform, layered eps_r (6 layers in [3, 25]) and sigma
    ([0, 0.01] S/m), 30 % forward+gradient, Poisson arrivals at `rate` jobs/s
    (all at t = 0 when rate is None).  nt_scale shortens every job (for
    bounded benchmark samples; 1.0 is the full stream)."""
    g = torch.Generator().manual_seed(seed)

    def u() -> float:
        return float(torch.rand((), generator=g, dtype=torch.float64))

    jobs, t = [], 0.0
    for i in range(n_jobs):
        nz = int(math.exp(math.log(nz_range[0]) + u() * math.log(nz_range[1] / nz_range[0])))
        nx = int(math.exp(math.log(nx_range[0]) + u() * math.log(nx_range[1] / nx_range[0])))
        nt = nt_range[0] + int(u() * (nt_range[1] - nt_range[0] + 1))
        nt = max(1, int(round(nt * nt_scale)))
        S = shots_range[0] + int(u() * (shots_range[1] - shots_range[0] + 1))
        grad = u() < gradient_fraction
        layer_eps = 3.0 + 22.0 * torch.rand(6, generator=g, dtype=torch.float64)
        layer_sig = 0.01 * torch.rand(6, generator=g, dtype=torch.float64)
        rows = torch.clamp(torch.arange(nz) * 6 // nz, max=5)
        eps = layer_eps[rows][:, None].expand(nz, nx).to(torch.float32).contiguous()
        sig = layer_sig[rows][:, None].expand(nz, nx).to(torch.float32).contiguous()
        mu = torch.ones((nz, nx), dtype=torch.float32)
        vmax = ph.C0 / math.sqrt(float(layer_eps.min()))
        dt = 0.9 / math.sqrt(2.0 / dx**2) / vmax
        amp = ph.ricker(freq, nt, dt, dtype=torch.float32).view(1, 1, nt).repeat(S, 1, 1)
        row = min(10, nz - 1)
        src = torch.tensor([[[row, int((s + 0.5) * nx / S)]] for s in range(S)])
        n_rec = max(1, min(256, nx // 4))
        rec = torch.tensor([[[row, int(j * nx / n_rec)] for j in range(n_rec)]] * S)
        if rate is not None:
            t += -math.log(max(u(), 1e-12)) / rate
        jobs.append(ModelingJob(eps, sig, mu, dx, dt, amp, src, rec, pml_width=pml,
                                gradient=grad, arrival=t, job_id=i))
    return jobs


def percentile(values: Sequence[float], q: float) -> float:
    """q-th percentile (0-100) with linear interpolation between order statistics."""
    v = sorted(values)
    if not v:
        return math.nan
    pos = (len(v) - 1) * q / 100.0
    lo = int(math.floor(pos))
    hi = min(lo + 1, len(v) - 1)
    return v[lo] + (v[hi] - v[lo]) * (pos - lo)


__all__ = ["JobPlan", "JobResult", "ModelingJob", "Segment", "TMServer", "group_bytes",
           "mixed_stream", "percentile", "plan_job", "program", "run_plain",
           "select_admissions"]
