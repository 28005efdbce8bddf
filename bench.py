"""Benchmark: 2-D TM forward + exact adjoint, FP32, config-2 workload.

Workload (one bench step = one full gradient evaluation):
  model 512 x 1024 (padded 553 x 1065 with CPML 20, stencil 2), dx = 0.02 m,
  dt = 0.9 x CFL, nt = 4000, 64 shots (sources on row 10 every 16 cells,
  256 receivers on row 10 every 4 cells, Ricker 400 MHz), eps_r = 6 layers
  U[3, 25] + smoothed N(0, 0.5) noise, sigma U[0, 0.01] per layer, seed 2.
  Loss 0.5 * sum(r^2); gradients w.r.t. eps and sigma.  Snapshots of Ey and
  curl H are stored on the device (FP32 by default, --storage bf16); the 64
  shots run in shot batches that fit HBM.
Metric: cell-updates per second (one padded cell of one shot advanced one
internal step, forward or adjoint): 2 * 64 * 553 * 1065 * 4000 = 3.02e11 per
step.

The default run adds a "serving" object: the first --serve-jobs jobs of the
seeded mixed-size stream (config 3) through the continuous-batching server
(tide_b200.serve) and one after another through the per-job API, plus a
Poisson-arrival run for p50/p99 latency.

Arms:
  default          the B200 library through the public tide_b200 API.
  --impl reference the reference's own CPU backend (compiled from its sources
                   with OpenMP) on the host cores, on a bounded sample of the
                   same workload.

Run with torchrun for N > 1 GPUs: the 64 shots of the evaluation are split
over the ranks (strided, as the reference's workflow/distributed.py does),
each rank back-propagates its shots in batches, and the partial eps/sigma
gradients are summed with one NCCL all-reduce (strong scaling: the job is
fixed, `value` counts its cell-updates once).
"""

from __future__ import annotations

import argparse
import ctypes
import gc
import json
import math
import os
import pathlib
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np
import torch

ROOT = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "tide-gpr_b200"))

import tide_b200 as tide  # noqa: E402
from tide_b200 import _native as nat  # noqa: E402
from tide_b200 import storage as stg  # noqa: E402

METRIC = "2D TM cell-updates/s fwd+adj (% of HBM roofline); served p50/p99 latency"
UNIT = "cell-updates/s"
PEAKS = ROOT / "MEASURED_PEAKS.json"
FALLBACK_HBM_GBS = 6650.0

# ---------------------------------------------------------------- workload


def config2(seed: int = 2, shots: int = 64, nt: int = 4000, device="cpu"):
    """Seeded config-2 model and acquisition (synthetic; no dataset)."""
    from scipy.ndimage import gaussian_filter

    ny, nx, dx = 512, 1024, 0.02
    rng = np.random.default_rng(seed)
    layer_eps = rng.uniform(3.0, 25.0, size=6)
    layer_sig = rng.uniform(0.0, 0.01, size=6)
    rows = np.minimum(np.arange(ny) * 6 // ny, 5)
    eps = layer_eps[rows][:, None] * np.ones((1, nx))
    sig = layer_sig[rows][:, None] * np.ones((1, nx))
    eps = eps + gaussian_filter(rng.normal(0.0, 0.5, size=(ny, nx)), sigma=8)
    eps = np.maximum(eps, 1.0)
    vmax = tide.C0 / math.sqrt(float(eps.min()))
    max_dt = 1.0 / math.sqrt(2.0 / dx**2) / vmax
    dt = 0.9 * max_dt
    amp = tide.ricker(400e6, nt, dt, dtype=torch.float64).view(1, 1, nt).repeat(shots, 1, 1)
    src = torch.tensor([[[10, 8 + 16 * i]] for i in range(shots)])
    rec = torch.tensor([[[10, 2 + 4 * j] for j in range(256)]] * shots)
    f32 = torch.float32
    return dict(
        eps=torch.from_numpy(eps).to(f32).to(device), sig=torch.from_numpy(sig).to(f32).to(device),
        mu=torch.ones((ny, nx), dtype=f32, device=device), amp=amp.to(f32).to(device),
        src=src.to(device), rec=rec.to(device), dx=dx, dt=dt, nt=nt, shots=shots, ny=ny, nx=nx,
        pml=20,
    )


PADDED = (553, 1065)


def cell_updates(shots: int, nt: int) -> float:
    return 2.0 * shots * PADDED[0] * PADDED[1] * nt


# ---------------------------------------------------------------- helpers


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL,
            )
        except FileNotFoundError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path).read().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        return {
            "sm_mhz": statistics.median(sm) if sm else None,
            "sm_max_mhz": max(smax) if smax else None,
            "reasons": sorted(reasons),
            "samples": len(sm),
        }


def hbm_peak() -> tuple[float, str]:
    try:
        return float(json.loads(PEAKS.read_text())["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def lib():
    L = nat.load()
    L.tide_b200_profile_enable.argtypes = [ctypes.c_int, ctypes.c_int]
    L.tide_b200_profile_read.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
    L.tide_b200_profile_read.restype = ctypes.c_int
    L.tide_b200_profile_kind_name.restype = ctypes.c_char_p
    L.tide_b200_launch_count.restype = ctypes.c_int64
    return L


def read_profile(L) -> dict:
    ms = (ctypes.c_double * 16)()
    n = (ctypes.c_int64 * 16)()
    k = L.tide_b200_profile_read(ms, n, 16)
    return {L.tide_b200_profile_kind_name(i).decode(): (ms[i], n[i]) for i in range(k)}


# Algorithmic bytes per cell (one shot, one step) of each stencil kernel,
# single sweep: fields each read/written once, model coefficients once per
# launch (shared by the S shots of a launch), CPML memories only in their
# strips (read + write), snapshot bytes where the kernel stores or reads them,
# and the model-shaped gradient read-modify-write once per launch.
def kernel_bytes_per_cell(kind: str, S: int, snap_bytes: int, rho_x: float, rho_y: float) -> float:
    f = 4.0
    strips = 2 * f * (rho_x + rho_y)  # two CPML memories (one per axis), read + write
    if kind == "fwd_h":  # read Ey; RMW Hx, Hz; cq; m_ey_x, m_ey_z
        return 5 * f + f / S + strips
    if kind == "fwd_e":  # read Hx, Hz; RMW Ey; ca, cb; m_hx_z, m_hz_x; store Ey^t, curl H^t
        return 4 * f + 2 * f / S + strips + 2 * snap_bytes
    if kind == "fwd_step":  # fused: read + write Ey, Hx, Hz; ca, cb, cq; four memories; snapshots
        return 6 * f + 3 * f / S + 2 * strips + 2 * snap_bytes
    if kind == "adj_e":  # read lEy; RMW lHx, lHz; cb; adjoint memories (read cur, write next)
        return 5 * f + f / S + strips
    if kind == "adj_h":  # read lHx, lHz; RMW lEy; ca, cq; memories; 2 snapshots; 2 gradients
        return 4 * f + 2 * f / S + strips + 2 * snap_bytes + 2 * 2 * f / S
    if kind == "adj_step":  # fused adjoint: read + write lEy, lHx, lHz; coefficients; memories;
        return 6 * f + 3 * f / S + 2 * strips + 2 * snap_bytes + 2 * 2 * f / S  # snapshots; grads
    raise KeyError(kind)


# ---------------------------------------------------------------- B200 arm


# DRAM bytes per cell (one shot, one step) moved by each kernel in an ncu
# capture (dram__bytes_read.sum + dram__bytes_write.sum) on the config-2 grid
# with 8-shot launches; None where not captured.
TRAFFIC_B_PER_CELL = {"adj_h": 23.6}


def shot_batches(shots: int, snap_bytes: int, device) -> int:
    per_shot = 2 * snap_bytes * PADDED[0] * PADDED[1] * 4000
    free, _ = torch.cuda.mem_get_info(device)
    budget = int(0.88 * free) - (4 << 30)
    b = max(1, min(shots, budget // per_shot))
    while shots % b:
        b -= 1
    return b


def _shot_take(t: torch.Tensor, ids: torch.Tensor) -> torch.Tensor:
    """Rows `ids` (CPU int64, ascending) of a per-shot tensor: a view for a
    contiguous range, a gathered copy otherwise."""
    lo, n = int(ids[0]), int(ids.numel())
    if int(ids[-1]) - lo + 1 == n:
        return t[lo:lo + n]
    return t.index_select(0, ids.to(t.device))


def sharded_gradient(eps, sig, n_shots: int, batch: int, batch_fn, ctx):
    """One gradient evaluation of an n_shots acquisition across the ranks of
    `ctx` (shot-parallel, as the reference's workflow/distributed.py:151,260-274):
    each rank takes its strided share of the shots (rank_shot_indices), runs
    them in batches of `batch` through batch_fn(eps, sig, ids) -- which
    back-propagates into eps.grad / sig.grad and returns the batch loss --
    and the partial gradients and losses are then summed over the ranks (the
    path's one exchange).  Every rank returns the full gradient [2, ny, nx]
    and the full loss, equal to a single-rank evaluation of all shots up to
    the order of the shot sum."""
    from tide_b200 import distributed as tdist

    e = eps.detach().requires_grad_(True)
    s = sig.detach().requires_grad_(True)
    ids = tdist.rank_shot_indices(n_shots, ctx=ctx, device="cpu")
    loss = torch.zeros((), dtype=eps.dtype, device=eps.device)
    for b in ids.split(max(1, int(batch))):
        loss = loss + batch_fn(e, s, b)
    tdist.all_reduce_gradients([e, s], ctx=ctx)
    loss = tdist.all_reduce_tensor(loss, ctx=ctx)
    if e.grad is None:
        e.grad = torch.zeros_like(e)
    if s.grad is None:
        s.grad = torch.zeros_like(s)
    return torch.stack([e.grad, s.grad]), loss


def run_b200(args) -> None:
    from tide_b200 import distributed as tdist

    ctx = tdist.init_distributed(device="cuda", timeout_s=600.0)  # NCCL when WORLD_SIZE > 1
    world, rank, dev = ctx.world_size, ctx.rank, ctx.device
    L = lib()
    snap_bytes = 2 if args.storage == "bf16" else 4
    cfg = config2(shots=args.shots, nt=args.nt)
    S_total = args.shots
    S_rank = int(tdist.rank_shot_indices(S_total, ctx=ctx, device="cpu").numel())
    batch = args.batch or shot_batches(S_rank, snap_bytes, dev)
    # snapshot format and shot batch of the step (the BF16 leg switches them)
    mode = {"compression": args.storage == "bf16", "batch": batch}

    # host (pinned) copies for the end-to-end leg, device copies for `value`
    host = {k: (v.pin_memory() if torch.is_tensor(v) else v) for k, v in cfg.items()}
    dev_in = {k: (v.to(dev) if torch.is_tensor(v) else v) for k, v in cfg.items()}

    def step(inp, copy_in: bool):
        if copy_in:
            d = {k: (v.to(dev, non_blocking=True) if torch.is_tensor(v) else v) for k, v in inp.items()}
        else:
            d = inp

        def batch_fn(eps, sig, ids):
            out = tide.maxwelltm(
                eps, sig, d["mu"], d["dx"], d["dt"], _shot_take(d["amp"], ids),
                _shot_take(d["src"], ids), _shot_take(d["rec"], ids),
                stencil=2, pml_width=d["pml"], storage_mode="device",
                storage_compression=mode["compression"],
            )
            r = out[-1]
            loss = 0.5 * (r * r).sum()
            loss.backward()
            return loss.detach()

        return sharded_gradient(d["eps"], d["sig"], S_total, mode["batch"], batch_fn, ctx)

    def timed(n_steps, copy_in):
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
        torch.cuda.synchronize(dev)
        st = torch.cuda.current_stream(dev)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        h2d = d2h = 0
        for _ in range(n_steps):
            g, loss = step(host if copy_in else dev_in, copy_in)
            if copy_in:
                h2d = sum(v.numel() * v.element_size() for v in host.values() if torch.is_tensor(v))
                g_h = g.to("cpu", non_blocking=False)
                l_h = loss.to("cpu")
                d2h = g_h.numel() * g_h.element_size() + l_h.numel() * l_h.element_size()
        e1.record(st)
        torch.cuda.synchronize(dev)
        ms = e0.elapsed_time(e1)
        if world > 1:
            import torch.distributed as dist

            t = torch.tensor([ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
            dist.barrier()
        return ms, h2d, d2h

    for _ in range(args.warmup):
        step(dev_in, False)
    torch.cuda.synchronize(dev)

    clocks = ClockSampler(dev.index or 0)
    clocks.start()
    L.tide_b200_profile_enable(1 if args.profile_every > 0 else 0, max(1, args.profile_every))
    read_profile(L)
    launches0 = L.tide_b200_launch_count()
    replays0 = nat.graph_replays()
    ms, _, _ = timed(args.steps, copy_in=False)
    launches = L.tide_b200_launch_count() - launches0
    replays = nat.graph_replays() - replays0
    L.tide_b200_profile_enable(0, 1)
    prof = read_profile(L)
    clk = clocks.stop()
    e2e_ms, h2d, d2h = timed(max(1, args.e2e_steps), copy_in=True)
    # config 2's BF16 snapshot variant: the same step and shot batches with
    # BF16 histories (half the snapshot bytes)
    bf16_leg = None
    if args.bf16_steps > 0 and args.storage == "fp32":
        def fresh():  # the FP32 history goes back to the driver before the switch
            torch.cuda.synchronize(dev)
            gc.collect()
            stg.release_history_pool()
            torch.cuda.empty_cache()

        fresh()
        mode.update(compression=True)
        try:
            step(dev_in, False)  # warm-up: allocates the BF16 history
            torch.cuda.synchronize(dev)
            L.tide_b200_profile_enable(1 if args.profile_every > 0 else 0,
                                       max(1, args.profile_every))
            read_profile(L)
            b_ms, _, _ = timed(args.bf16_steps, copy_in=False)
            L.tide_b200_profile_enable(0, 1)
            bprof = read_profile(L)
        except torch.OutOfMemoryError as exc:  # reported in the line; the rest still runs
            L.tide_b200_profile_enable(0, 1)
            bf16_leg = {"error": str(exc).splitlines()[0]}
        finally:
            mode.update(compression=False)
            fresh()
        if bf16_leg is None:
            bk = {}
            for k in ("fwd_h", "fwd_e", "adj_e", "adj_h"):
                if bprof.get(k, (0, 0))[1] > 0:
                    avg = bprof[k][0] / bprof[k][1]
                    bpc = kernel_bytes_per_cell(k, batch, 2, 41 / PADDED[1], 41 / PADDED[0])
                    gbs = bpc * batch * PADDED[0] * PADDED[1] / (avg / 1e3) / 1e9
                    bk[k] = {"avg_launch_ms": round(avg, 5), "achieved_gbs": round(gbs, 1),
                             "frac": round(gbs / hbm_peak()[0], 4)}
            bf16_leg = {
                "value": cell_updates(S_total, args.nt) * args.bf16_steps / (b_ms / 1e3),
                "unit": UNIT, "steps": args.bf16_steps, "ms_per_step": b_ms / args.bf16_steps,
                "shot_batch": batch, "kernels": bk,
                "note": "same step and shot batches with BF16 snapshot histories; kernel "
                        "fractions use 2-byte snapshots in the byte model"}
    # the same step with every time step launched from the host (no graphs)
    eager_ms = None
    if args.graphs_off_steps > 0:
        prev = nat.set_step_graphs(False)
        try:
            eager_ms, _, _ = timed(args.graphs_off_steps, copy_in=False)
        finally:
            nat.set_step_graphs(prev)

    units = cell_updates(S_total, args.nt)  # the whole job; its shots are split over the ranks
    value = units * args.steps / (ms / 1e3)
    e2e_value = units * max(1, args.e2e_steps) / (e2e_ms / 1e3)

    # roofline of the dominant kernel
    peak, peak_kind = hbm_peak()
    rho_x, rho_y = 41 / PADDED[1], 41 / PADDED[0]
    shares = {k: v[0] for k, v in prof.items() if v[1] > 0}
    dom = max(shares, key=shares.get) if shares else None
    roof = None
    if dom:
        avg_ms = prof[dom][0] / prof[dom][1]
        bpc = kernel_bytes_per_cell(dom, batch, snap_bytes, rho_x, rho_y)
        bytes_launch = bpc * batch * PADDED[0] * PADDED[1]
        achieved = bytes_launch / (avg_ms / 1e3) / 1e9
        roof = {
            "kernel": dom, "bound": "hbm", "achieved": round(achieved, 1), "peak": peak,
            "peak_source": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
            "traffic": (TRAFFIC_B_PER_CELL[dom] * batch * PADDED[0] * PADDED[1]
                        if dom in TRAFFIC_B_PER_CELL else None),
            "algorithmic_bytes_per_launch": bytes_launch,
            "avg_launch_ms": avg_ms,
            "kernel_ms_share": {k: round(v / sum(shares.values()), 4) for k, v in shares.items()},
        }
    # GPU busy time: sampled mean duration of each step kernel x its launches
    # per step (nt per shot batch), against the measured step time
    n_batches = -(-S_rank // batch)
    kernel_ms = sum(prof[k][0] / prof[k][1] * args.nt * n_batches
                    for k in ("fwd_h", "fwd_e", "adj_e", "adj_h") if prof.get(k, (0, 0))[1] > 0)
    graphs = {
        "replays": int(replays), "block_steps": 64,
        "kernel_ms_per_step": round(kernel_ms, 2),
        "kernel_share_of_step": round(kernel_ms / (ms / args.steps), 4) if kernel_ms else None,
        "ms_per_step_graphs_off": (eager_ms / args.graphs_off_steps) if eager_ms else None,
        "graphs_off_steps": args.graphs_off_steps,
    }

    tma_leg = None
    serving = em3d_leg = debye_leg = None
    # the other legs budget device memory themselves: kept histories (some
    # held only by reference cycles until a collection) go back to the driver
    torch.cuda.synchronize(dev)
    gc.collect()
    stg.release_history_pool()
    torch.cuda.empty_cache()
    if rank == 0 and world == 1 and args.serve_jobs > 0:
        serving = serve_bench(args)
    sweep = None
    if rank == 0 and world == 1 and args.serve_sweep_jobs > 0:
        try:
            sweep = serve_sweep(args)
        except nat.NativeError as exc:  # reported in the line; the other legs still run
            sweep = {"error": str(exc)}
            torch.cuda.synchronize(dev)
            torch.cuda.empty_cache()
    if rank == 0 and world == 1 and args.em3d_nt > 0:
        em3d_leg = em3d_bench(args)
    if rank == 0 and world == 1 and args.debye_nt > 0:
        debye_leg = debye_bench(args)
    if rank == 0 and world == 1 and args.tma_nt > 0:  # after the legs that budget memory
        tma_leg = tma_bench(args, dev, batch, snap_bytes)
    if rank == 0:
        cpu = cpu_baseline(args) if not args.no_cpu_baseline else None
        parity = parity_report(args, dev) if not args.no_cpu_baseline and args.parity_nt > 0 else None
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded config-2 model and acquisition)",
            "config": {
                "workload": "config2: 2D TM fwd+adj, 512x1024 (553x1065 padded), CPML 20, "
                            f"stencil 2, nt={args.nt}, {S_total} shots, snapshots {args.storage} on device",
                "shots": S_total, "shot_batch": batch, "nt": args.nt,
                "cell_updates_per_step": units, "l2": "per-step working set (snapshot history) >> L2",
                "parallelism": f"shot-parallel dp{world}: {S_rank} shots per rank in batches "
                               f"of {batch}, one all-reduce of the eps/sigma gradient",
            },
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches), "step_graphs": graphs,
            "roofline": roof, "cpu_baseline": cpu, "parity": parity, "clocks": clk,
            "tma_path": tma_leg, "bf16_snapshots": bf16_leg,
            "serving": serving, "serving_sweep": sweep,
            "em3d": em3d_leg, "debye": debye_leg,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()


def tma_bench(args, dev, batch: int, snap_bytes: int) -> dict:
    """The one-sweep TMA time steps (opt-in, tide_b200_set_tma_mode) against
    the default per-call kernels on one batch of the same workload: first
    `batch` shots, tma_nt steps, fwd + adj through the public API, CUDA-event
    device time of the whole evaluation and per-kernel event samples."""
    cfg = config2(shots=batch, nt=args.tma_nt, device=dev)
    L = lib()
    peak, peak_kind = hbm_peak()
    rho_x, rho_y = 41 / PADDED[1], 41 / PADDED[0]

    def once():
        eps = cfg["eps"].detach().requires_grad_(True)
        sig = cfg["sig"].detach().requires_grad_(True)
        out = tide.maxwelltm(eps, sig, cfg["mu"], cfg["dx"], cfg["dt"], cfg["amp"], cfg["src"],
                             cfg["rec"], stencil=2, pml_width=cfg["pml"], storage_mode="device",
                             storage_compression=args.storage == "bf16")
        (0.5 * (out[-1] * out[-1]).sum()).backward()
        return torch.stack([eps.grad, sig.grad])

    res = {}
    grads = {}
    for name, mode in (("default", 0), ("tma", 2)):
        prev = nat.set_tma_mode(mode)
        try:
            once()
            once()  # warm-up (pool, tensor maps)
            ms, g = _timed_gpu(once, dev)
            L.tide_b200_profile_enable(1, 10)
            read_profile(L)
            once()
            torch.cuda.synchronize(dev)
            L.tide_b200_profile_enable(0, 1)
            prof = {k: v for k, v in read_profile(L).items() if v[1] > 0}
        finally:
            nat.set_tma_mode(prev)
        grads[name] = g
        kern = {}
        for k, (tot, n) in prof.items():
            avg = tot / n
            bpc = kernel_bytes_per_cell(k, batch, snap_bytes, rho_x, rho_y)
            ach = bpc * batch * PADDED[0] * PADDED[1] / (avg / 1e3) / 1e9
            kern[k] = {"avg_launch_ms": round(avg, 5), "achieved_gbs": round(ach, 1),
                       "frac": round(ach / peak, 4)}
        res[name] = {"ms_per_eval": ms,
                     "cell_updates_per_s": 2.0 * batch * PADDED[0] * PADDED[1] * args.tma_nt / (ms / 1e3),
                     "kernels": kern}
    d = grads["tma"] - grads["default"]
    res["grad_bitwise_equal"] = bool(torch.equal(grads["tma"], grads["default"]))
    res["grad_max_abs_diff"] = float(d.abs().max())
    res["workload"] = (f"config2 grid, {batch} shots, nt={args.tma_nt}, snapshots {args.storage} "
                       "on device; fwd+adj through the public API")
    res["peak"] = {"hbm_gbs": peak, "source": peak_kind}
    return res


# ---------------------------------------------------------------- serving


def serve_bench(args) -> dict:
    """Served mixed-size stream (seeded, synthetic): the first `serve_jobs`
    jobs of the 2000-job stream (nz, nx log-uniform, nt and shots uniform,
    30 % forward+gradient), unchanged in size.  Three runs: all jobs queued at
    t = 0 through the server (capacity), the same jobs one after another
    through the per-job public API with the same plans (plain), and Poisson
    arrivals at `serve_load` x the served capacity (p50/p99 latency)."""
    from tide_b200 import serve as sv

    dev = torch.device("cuda", torch.cuda.current_device())
    torch.cuda.empty_cache()
    jobs = sv.mixed_stream(args.serve_jobs, seed=3)
    cells = sum(j.cell_updates() for j in jobs)
    L = lib()
    with sv.TMServer(dev, chunk_steps=args.serve_chunk) as srv:
        srv.serve([sv.mixed_stream(1, seed=11, nt_scale=0.02)[0]], realtime=False)  # capture
        torch.cuda.synchronize(dev)
        l0 = srv.launches()
        t0 = time.perf_counter()
        res = srv.serve(jobs, realtime=False)
        torch.cuda.synchronize(dev)
        t_served = time.perf_counter() - t0
        launches = srv.launches() - l0
        stats = dict(srv.stats)
        plans = {j.job_id: srv.plan(j) for j in jobs}
        budget = srv.budget
    assert len(res) == len(jobs)
    torch.cuda.empty_cache()
    n_plain = min(len(jobs), args.serve_plain_jobs)
    lp0 = L.tide_b200_launch_count()
    t0 = time.perf_counter()
    for j in jobs[:n_plain]:
        sv.run_plain(j, plans[j.job_id], dev)
    torch.cuda.synchronize(dev)
    t_plain = time.perf_counter() - t0
    plain_launches = L.tide_b200_launch_count() - lp0
    cells_plain = sum(j.cell_updates() for j in jobs[:n_plain])
    torch.cuda.empty_cache()
    rate = args.serve_load * len(jobs) / t_served
    stream = sv.mixed_stream(args.serve_jobs, seed=3, rate=rate)
    with sv.TMServer(dev, chunk_steps=args.serve_chunk) as srv:
        srv.serve([sv.mixed_stream(1, seed=11, nt_scale=0.02)[0]], realtime=False)
        t0 = time.perf_counter()
        res2 = srv.serve(stream, realtime=True)
        t_stream = time.perf_counter() - t0
    lat = [r.latency for r in res2]
    served = cells / t_served
    plain = cells_plain / t_plain
    modes = {}
    for p in plans.values():
        modes[p.mode] = modes.get(p.mode, 0) + 1
    return {
        "workload": f"served mixed-size 2D TM stream, seed 3, first {len(jobs)} of 2000 jobs "
                    "(full sizes: nz 128-1024, nx 256-2048 log-uniform, nt 1000-6000, shots 1-32, "
                    "30 % forward+gradient), CPML 20, stencil 2, FP32",
        "jobs": len(jobs), "cell_updates": cells,
        "served_cell_updates_per_s": served, "served_s": t_served,
        "plain_cell_updates_per_s": plain, "plain_s": t_plain, "plain_jobs": n_plain,
        "served_over_plain": served / plain,
        "poisson_rate_jobs_per_s": rate, "load": args.serve_load,
        "stream_cell_updates_per_s": cells / t_stream,
        "latency_p50_s": sv.percentile(lat, 50), "latency_p99_s": sv.percentile(lat, 99),
        "latency_max_s": max(lat),
        "chunk_steps": args.serve_chunk, "memory_budget_gb": round(budget / 1e9, 1),
        "max_resident_groups": stats["max_resident"], "chunks": stats["chunks"],
        "engine_launches": launches, "plain_launches": int(plain_launches), "plans": modes,
        "timing": "wall clock around host-to-host runs (models and sources in host memory, "
                  "results copied back), torch.cuda.synchronize at the end",
    }


def serve_sweep(args) -> dict:
    """Load sweep of the served stream on a bounded sample: the first
    `serve_sweep_jobs` jobs of the seeded 2000-job stream with every nt
    scaled by `serve_sweep_nt_scale` (sizes, shots and the forward/gradient
    mix unchanged).  Capacity (all jobs at t = 0) through the server, the
    same jobs one after another through the per-job path (plain), then
    Poisson arrivals at each load of `serve_sweep_loads` x the served
    capacity with p50 / p99 latency per load."""
    from tide_b200 import serve as sv

    dev = torch.device("cuda", torch.cuda.current_device())
    torch.cuda.empty_cache()
    n, scale = args.serve_sweep_jobs, args.serve_sweep_nt_scale
    jobs = sv.mixed_stream(n, seed=3, nt_scale=scale)
    cells = sum(j.cell_updates() for j in jobs)
    with sv.TMServer(dev, chunk_steps=args.serve_chunk) as srv:
        srv.serve([sv.mixed_stream(1, seed=11, nt_scale=0.02)[0]], realtime=False)  # capture
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        srv.serve(jobs, realtime=False)
        torch.cuda.synchronize(dev)
        t_served = time.perf_counter() - t0
        plans = {j.job_id: srv.plan(j) for j in jobs}
    torch.cuda.empty_cache()
    t0 = time.perf_counter()
    for j in jobs:
        sv.run_plain(j, plans[j.job_id], dev)
    torch.cuda.synchronize(dev)
    t_plain = time.perf_counter() - t0
    loads = {}
    for load in [float(v) for v in args.serve_sweep_loads.split(",") if v]:
        rate = load * n / t_served
        stream = sv.mixed_stream(n, seed=3, rate=rate, nt_scale=scale)
        torch.cuda.empty_cache()
        with sv.TMServer(dev, chunk_steps=args.serve_chunk) as srv:
            srv.serve([sv.mixed_stream(1, seed=11, nt_scale=0.02)[0]], realtime=False)
            t0 = time.perf_counter()
            res = srv.serve(stream, realtime=True)
            t_stream = time.perf_counter() - t0
        lat = [r.latency for r in res]
        loads[str(load)] = {"rate_jobs_per_s": rate, "latency_p50_s": sv.percentile(lat, 50),
                            "latency_p99_s": sv.percentile(lat, 99), "latency_max_s": max(lat),
                            "stream_cell_updates_per_s": cells / t_stream}
    sizes = [j.cell_updates() for j in jobs]
    return {
        "workload": f"served 2D TM stream, seed 3, first {n} of 2000 jobs, nt x {scale} "
                    "(nz 128-1024, nx 256-2048 log-uniform, shots 1-32, 30 % forward+gradient), "
                    "CPML 20, stencil 2, FP32",
        "jobs": n, "cell_updates": cells,
        "cell_updates_per_job_p10_p50_p90": [sv.percentile(sizes, q) for q in (10, 50, 90)],
        "served_cell_updates_per_s": cells / t_served, "served_s": t_served,
        "plain_cell_updates_per_s": cells / t_plain, "plain_s": t_plain,
        "served_over_plain": t_plain / t_served, "loads": loads,
        "timing": "wall clock around host-to-host runs, torch.cuda.synchronize at the end",
    }


# ---------------------------------------------------------------- 3-D and Debye legs


def config4(seed: int = 4, shots: int = 4, nt: int = 1500, device="cpu"):
    """Seeded config-4 model and acquisition (synthetic): 128^3, dx 0.02 m,
    eps_r in 6 horizontal layers U[1, 16] with 8 ellipsoid inclusions (radii
    5-20 cells, eps_r U[1, 30]), sigma U[0, 0.005] S/m per layer, dt at 0.9 x
    the 3-axis CFL limit, Ez dipole Ricker 500 MHz, 64 receivers on the top
    plane."""
    n, dx = 128, 0.02
    rng = np.random.default_rng(seed)
    layer_eps = rng.uniform(1.0, 16.0, size=6)
    layer_sig = rng.uniform(0.0, 0.005, size=6)
    rows = np.minimum(np.arange(n) * 6 // n, 5)
    eps = np.broadcast_to(layer_eps[rows][:, None, None], (n, n, n)).copy()
    sig = np.broadcast_to(layer_sig[rows][:, None, None], (n, n, n)).copy()
    z, y, x = np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij")
    for _ in range(8):
        c = rng.uniform(0, n, size=3)
        r = rng.uniform(5, 20, size=3)
        e = rng.uniform(1.0, 30.0)
        inside = ((z - c[0]) / r[0]) ** 2 + ((y - c[1]) / r[1]) ** 2 + ((x - c[2]) / r[2]) ** 2 <= 1
        eps[inside] = e
    vmax = tide.C0 / math.sqrt(float(eps.min()))
    dt = 0.9 * dx / (math.sqrt(3.0) * vmax)
    amp = tide.ricker(500e6, nt, dt, dtype=torch.float64).view(1, 1, nt).repeat(shots, 1, 1)
    src = torch.tensor([[[12, 32 + 64 * (i // 2), 32 + 64 * (i % 2)]] for i in range(shots)])
    rec = torch.tensor([[[0, 8 + 16 * (j // 8), 8 + 16 * (j % 8)] for j in range(64)]] * shots)
    f32 = torch.float32
    return dict(
        eps=torch.from_numpy(eps).to(f32).to(device), sig=torch.from_numpy(sig).to(f32).to(device),
        mu=torch.ones((n, n, n), dtype=f32, device=device), amp=amp.to(f32).to(device),
        src=src.to(device), rec=rec.to(device), dx=dx, dt=dt, nt=nt, shots=shots, pml=12,
    )


PADDED3 = 153  # 128 + 2 x 12 CPML + 1 fd pad


# Algorithmic bytes per cell (one shot, one step) of each 3-D kernel, FP32
# fields: six field components each read or read-modify-written once, the
# model coefficients once per launch of S shots, the two CPML memories of
# each axis read + written in that axis's strips (strip fraction rho per
# axis), snapshots (six components of snap_bytes) where stored or read, and
# the per-shot coefficient-gradient buffers read-modify-written by the
# gradient pass.
def em3d_bytes_per_cell(kind: str, S: int, snap_bytes: int, rho: float) -> float:
    f = 4.0
    strips = 2 * 2 * f * 3 * rho  # 2 memories per axis, read + write, 3 axes
    if kind == "em3d_fwd_h":  # read Ex, Ey, Ez; RMW Hx, Hy, Hz; cq
        return 9 * f + f / S + strips
    if kind == "em3d_fwd_e":  # read H; RMW E; ca, cb; store E^t and curl H^t
        return 9 * f + 2 * f / S + strips + 6 * snap_bytes
    if kind == "em3d_adj_e":  # read lambda_E; RMW lambda_H; cb; adjoint memories; and the
        # previous stored step's gradient term: six snapshots, two per-shot gradients RMW
        return 9 * f + f / S + strips + 6 * snap_bytes + 2 * 2 * f
    if kind == "em3d_adj_h":  # read lambda_H; RMW lambda_E; ca, cq; adjoint memories
        return 9 * f + 2 * f / S + strips
    if kind == "em3d_grad":  # last step's term: lambda_E, six snapshots, two gradients RMW
        return 3 * f + 6 * snap_bytes + 2 * 2 * f
    raise KeyError(kind)


def _timed_gpu(fn, dev):
    """Device time (CUDA events on the current stream) of fn(), ms."""
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    out = fn()
    e1.record()
    torch.cuda.synchronize(dev)
    return e0.elapsed_time(e1), out


def em3d_bench(args) -> dict:
    """Config-4 leg: 3-D fwd+adj with BF16 snapshots, (a) checkpoint segments
    with recomputation at the full nt, (b) the history in pinned host memory
    (host-link bound) on the first em3d_host_nt steps, with the checkpoint
    gradient of the same steps compared to it; plus the box's H2D/D2H
    bandwidth for a 1 GiB pinned copy."""
    from tide_b200 import em3d

    dev = torch.device("cuda", torch.cuda.current_device())
    torch.cuda.empty_cache()

    def run(cfg, mode):
        eps = cfg["eps"].detach().requires_grad_(True)
        sig = cfg["sig"].detach().requires_grad_(True)
        out = em3d.maxwell3d(eps, sig, cfg["mu"], cfg["dx"], cfg["dt"], cfg["amp"], cfg["src"],
                             cfg["rec"], pml_width=cfg["pml"], source_component="ez",
                             receiver_component="ez", storage_mode=mode, storage_compression=True)
        r = out[-1]
        (0.5 * (r * r).sum()).backward()
        return eps.grad, sig.grad

    full = config4(shots=4, nt=args.em3d_nt, device=dev)
    run(dict(full, amp=full["amp"][..., :64]), "checkpoint")  # warm-up
    ms_ck, _ = _timed_gpu(lambda: run(full, "checkpoint"), dev)
    units = 2.0 * full["shots"] * PADDED3 ** 3 * args.em3d_nt
    seg = em3d.checkpoint_steps(args.em3d_nt, 1, None)
    # per-kernel device times: CUDA events around every 10th step's launches
    # (on the launching stream, inside the library) during one more evaluation
    L = lib()
    L.tide_b200_profile_enable(1, 10)
    read_profile(L)
    run(full, "checkpoint")
    torch.cuda.synchronize(dev)
    L.tide_b200_profile_enable(0, 1)
    prof = {k: v for k, v in read_profile(L).items() if k.startswith("em3d_") and v[1] > 0}
    peak, peak_kind = hbm_peak()
    rho = 27 / PADDED3  # 13 + 14 compact strip cells per axis
    cells = full["shots"] * PADDED3 ** 3
    kernels = {}
    for k, (tot, n) in prof.items():
        bpc = em3d_bytes_per_cell(k, full["shots"], 2, rho)
        if k == "em3d_fwd_e":  # checkpoint mode: half the sampled launches store snapshots
            bpc -= 0.5 * 6 * 2
        avg = tot / n
        ach = bpc * cells / (avg / 1e3) / 1e9
        kernels[k] = {"avg_launch_ms": avg, "launches_sampled": n, "bytes_per_cell": round(bpc, 2),
                      "achieved_gbs": round(ach, 1), "frac": round(ach / peak, 4)}
    share = {k: v[0] for k, v in prof.items()}
    dom = max(share, key=share.get) if share else None
    roof3 = None
    if dom:
        roof3 = {"kernel": dom, "bound": "hbm", "achieved": kernels[dom]["achieved_gbs"],
                 "peak": peak, "peak_source": peak_kind, "unit": "GB/s",
                 "frac": kernels[dom]["frac"], "traffic": None,
                 "algorithmic_bytes_per_launch": kernels[dom]["bytes_per_cell"] * cells,
                 "avg_launch_ms": kernels[dom]["avg_launch_ms"],
                 "kernel_ms_share": {k: round(v / sum(share.values()), 4) for k, v in share.items()},
                 "kernels": kernels}
    torch.cuda.empty_cache()
    short = dict(full, amp=full["amp"][..., : args.em3d_host_nt])
    run(short, "cpu")  # warm-up: the pinned host history is allocated once and then cached
    ms_host, g_host = _timed_gpu(lambda: run(short, "cpu"), dev)
    _, g_ck = _timed_gpu(lambda: run(short, "checkpoint"), dev)
    rel = lambda a, b: float((a - b).norm() / b.norm())  # noqa: E731
    units_short = 2.0 * full["shots"] * PADDED3 ** 3 * args.em3d_host_nt
    hist_step = 6 * full["shots"] * PADDED3 ** 3 * 2
    # host link: 1 GiB pinned <-> device
    h = torch.empty(1 << 28, dtype=torch.float32, pin_memory=True)
    d = torch.empty(1 << 28, dtype=torch.float32, device=dev)
    d.copy_(h, non_blocking=True)
    ms_h2d, _ = _timed_gpu(lambda: d.copy_(h, non_blocking=True), dev)
    ms_d2h, _ = _timed_gpu(lambda: h.copy_(d, non_blocking=True), dev)
    del h, d
    torch.cuda.empty_cache()
    return {
        "workload": f"config4: 3-D Yee fwd+adj, 128^3 ({PADDED3}^3 padded), CPML 12, 4 shots, "
                    "Ez dipole Ricker 500 MHz, 64 receivers on the top plane, BF16 snapshots",
        "checkpoint_bf16": {"nt": args.em3d_nt, "segment_steps": seg, "ms_per_eval": ms_ck,
                            "cell_updates_per_s": units / (ms_ck / 1e3),
                            "note": "fwd + recomputed fwd with storage + adjoint; cell-updates "
                                    "count fwd+adj only"},
        "host_bf16": {"nt": args.em3d_host_nt, "ms_per_eval": ms_host,
                      "cell_updates_per_s": units_short / (ms_host / 1e3),
                      "history_bytes_per_step": hist_step,
                      "history_gb_full_nt": hist_step * args.em3d_nt / 1e9},
        "link": {"h2d_gbs": (1 << 30) / (ms_h2d / 1e3) / 1e9,
                 "d2h_gbs": (1 << 30) / (ms_d2h / 1e3) / 1e9, "bytes": 1 << 30},
        "grad_rel_l2_checkpoint_vs_host": {"eps": rel(g_ck[0], g_host[0]),
                                            "sigma": rel(g_ck[1], g_host[1])},
        "roofline": roof3,
        "timing": "CUDA events around each whole evaluation (public API, device inputs)",
    }


def config5(seed: int = 5, shots: int = 128, nt: int = 8000, device="cpu"):
    """Seeded config-5 Debye model (synthetic): 2048 x 4096, dx 0.02 m,
    eps_inf U[3, 10], delta_eps U[0, 5], tau U[1e-10, 1e-9] s as Gaussian-
    smoothed (8 cells) random fields, sigma 0, dt at 0.9 x the CFL limit of
    eps_inf, sources on row 10 every 32 cells, 256 receivers on row 10,
    Ricker 400 MHz."""
    from scipy.ndimage import gaussian_filter

    ny, nx, dx = 2048, 4096, 0.02
    rng = np.random.default_rng(seed)

    def field(lo, hi):
        u = gaussian_filter(rng.uniform(0.0, 1.0, size=(ny, nx)), sigma=8)
        u = (u - u.min()) / max(float(u.max() - u.min()), 1e-12)
        return lo + (hi - lo) * u

    eps_inf, deps, tau = field(3.0, 10.0), field(0.0, 5.0), field(1e-10, 1e-9)
    vmax = tide.C0 / math.sqrt(float(eps_inf.min()))
    dt = 0.9 / math.sqrt(2.0 / dx**2) / vmax
    amp = tide.ricker(400e6, nt, dt, dtype=torch.float64).view(1, 1, nt).repeat(shots, 1, 1)
    src = torch.tensor([[[10, 16 + 32 * i]] for i in range(shots)])
    rec = torch.tensor([[[10, 8 + 16 * j] for j in range(256)]] * shots)
    f32 = torch.float32
    t = lambda a: torch.from_numpy(a).to(f32).to(device)  # noqa: E731
    return dict(eps=t(eps_inf), sig=torch.zeros((ny, nx), dtype=f32, device=device),
                mu=torch.ones((ny, nx), dtype=f32, device=device), deps=t(deps), tau=t(tau),
                amp=amp.to(f32).to(device), src=src.to(device), rec=rec.to(device), dx=dx, dt=dt,
                nt=nt, shots=shots, pml=30)


def debye_bench(args) -> dict:
    """Config-5 leg: Debye-medium fwd+adj (gradients in eps_inf, sigma,
    delta_eps, tau) on the full 2109 x 4157 padded grid with checkpoint
    segments, for the first debye_shots shots and debye_nt steps."""
    dev = torch.device("cuda", torch.cuda.current_device())
    torch.cuda.empty_cache()
    c = config5(shots=args.debye_shots, nt=args.debye_nt, device=dev)

    def run(cfg):
        eps = cfg["eps"].detach().requires_grad_(True)
        sig = cfg["sig"].detach().requires_grad_(True)
        deps = cfg["deps"].detach().requires_grad_(True)
        tau = cfg["tau"].detach().requires_grad_(True)
        out = tide.maxwelltm(eps, sig, cfg["mu"], cfg["dx"], cfg["dt"], cfg["amp"], cfg["src"],
                             cfg["rec"], stencil=2, pml_width=cfg["pml"], storage_mode="checkpoint",
                             dispersion=tide.DebyeDispersion(deps, tau))
        r = out[-1]
        (0.5 * (r * r).sum()).backward()
        return eps.grad

    run(dict(c, amp=c["amp"][..., :16]))  # warm-up
    ms, _ = _timed_gpu(lambda: run(c), dev)
    padded = (2048 + 61) * (4096 + 61)
    units = 2.0 * args.debye_shots * padded * args.debye_nt
    torch.cuda.empty_cache()
    return {
        "workload": "config5: 2-D TM 1-pole Debye fwd+adj, 2048x4096 (2109x4157 padded), CPML 30, "
                    f"{args.debye_shots} of 128 shots, nt={args.debye_nt} of 8000, checkpoint "
                    "segments, FP32 snapshots",
        "ms_per_eval": ms, "cell_updates_per_s": units / (ms / 1e3),
        "segment_steps": int(round(args.debye_nt ** 0.5)),
        "timing": "CUDA events around one whole evaluation (public API, device inputs)",
    }


# ---------------------------------------------------------------- CPU arm


def _ref_lib():
    p = ROOT / "oracle" / "_ref" / "libtide_ref_cpu.so"
    if p.exists():
        return ctypes.CDLL(str(p)), "reference"
    return None, "port"


def cpu_sample(n_shots: int, nt: int, threads: int):
    """Time fwd+adj of the reference CPU backend on a config-2 sample."""
    from tide_b200.tm2d import prepare_tm2d

    lib, kind = _ref_lib()
    cfg = config2(shots=n_shots, nt=nt)
    pb = prepare_tm2d(cfg["eps"], cfg["sig"], cfg["mu"], cfg["dx"], cfg["dt"], cfg["amp"],
                      cfg["src"], cfg["rec"], stencil=2, pml_width=20)
    prof = [pb.profiles[n] for n in ("ay", "by", "ayh", "byh", "ax", "bx", "axh", "bxh",
                                      "ky", "kyh", "kx", "kxh")]
    P = lambda t: 0 if t is None or t.numel() == 0 else t.data_ptr()  # noqa: E731
    S, ny, nx = pb.n_shots, pb.ny, pb.nx
    r = torch.zeros((nt, S, pb.n_rec))
    ey_st = torch.empty((nt, S, ny, nx))
    cu_st = torch.empty((nt, S, ny, nx))
    if lib is None:
        raise RuntimeError("reference CPU backend not built (oracle/_ref); run build()")
    fwd = lib.maxwell_tm_2_float_forward_with_storage_cpu
    fwd.argtypes = nat.argtypes("maxwell_tm_forward_with_storage", "float")
    bwd = lib.maxwell_tm_2_float_backward_cpu
    bwd.argtypes = nat.argtypes("maxwell_tm_backward", "float")
    ey, hx, hz, mex, mez, mhx, mhz = pb.fields
    t0 = time.perf_counter()
    fwd(P(pb.ca), P(pb.cb), P(pb.cq), P(pb.f), P(ey), P(hx), P(hz), P(mex), P(mez), P(mhx),
        P(mhz), P(r), P(ey_st), 0, 0, P(cu_st), 0, 0, *[P(t) for t in prof], P(pb.sources_i),
        P(pb.receivers_i), pb.rdy, pb.rdx, pb.dt, nt, S, ny, nx, pb.n_src, pb.n_rec, 1, 0, 0,
        ny * nx * 4, True, True, False, False, False, 0, pb.pml_y0, pb.pml_x0, pb.pml_y1,
        pb.pml_x1, threads, 0, 0, 0)
    lam = [torch.zeros((S, ny, nx)) for _ in range(7)]
    scratch = torch.zeros((4, S, ny, nx))
    gca, gcb = torch.zeros((ny, nx)), torch.zeros((ny, nx))
    sca, scb = torch.zeros((S, ny, nx)), torch.zeros((S, ny, nx))
    gf = torch.zeros((nt, S, pb.n_src))
    bwd(P(pb.ca), P(pb.cb), P(pb.cq), P(r), *[P(t) for t in lam], P(scratch), P(ey_st), 0, 0,
        P(cu_st), 0, 0, P(gf), P(gca), P(gcb), P(sca), P(scb), *[P(t) for t in prof],
        P(pb.sources_i), P(pb.receivers_i), pb.rdy, pb.rdx, pb.dt, nt, S, ny, nx, pb.n_src,
        pb.n_rec, 1, 0, 0, ny * nx * 4, True, True, False, False, False, nt, pb.pml_y0, pb.pml_x0,
        pb.pml_y1, pb.pml_x1, threads, 0, 0, 0)
    sec = time.perf_counter() - t0
    return cell_updates(n_shots, nt) / sec, sec, kind


def cpu_baseline(args) -> dict:
    threads = os.cpu_count() or 1
    try:
        v, sec, kind = cpu_sample(args.cpu_shots, args.cpu_nt, threads)
    except Exception as exc:  # noqa: BLE001
        return {"value": None, "unit": UNIT, "cores": threads, "kind": "reference",
                "sample": f"unavailable: {exc}"}
    return {
        "value": v, "unit": UNIT, "cores": threads, "kind": kind,
        "sample": f"reference CPU backend (OpenMP build, {threads} threads), config-2 geometry, "
                  f"{args.cpu_shots} shots x nt={args.cpu_nt} fwd+adj in {sec:.2f} s",
    }


def parity_report(args, dev) -> dict:
    """Accuracy beside the speed (part of the CPU-baseline leg: the CPU
    checkers run here only to check the GPU results): config-1 receivers
    against the reference CPU backend's FP32 and FP64 runs, and the eps /
    sigma gradient of a config-2 sample (full grid, the first
    --parity-shots shots, --parity-nt steps) against the C oracle's exact
    adjoint in FP32 and FP64, plus the BF16-snapshot gradient error."""
    sys.path.insert(0, str(ROOT / "tests"))
    try:
        import parity_config2 as pc2

        t0 = time.perf_counter()
        c1 = pc2.config1_errors(dev)
        c2 = pc2.config2_sample_errors(config2(shots=args.parity_shots, nt=args.parity_nt), dev)
        sec = time.perf_counter() - t0
    except Exception as exc:  # noqa: BLE001
        return {"unavailable": f"{type(exc).__name__}: {exc}"}
    return {
        "config1_receivers": c1,
        "config2_sample": dict(c2, sample=f"config-2 model and acquisition, 553x1065 padded, "
                                          f"first {args.parity_shots} shots, nt={args.parity_nt}, "
                                          "loss 0.5|r|^2, FP32 public API vs C oracle exact "
                                          "adjoint (reference summation order)"),
        "bar": "FP32 relative L2 <= 1e-5 against the FP32 checkers; FP64 figures are the "
               "FP32 error statement; BF16 snapshots: gradient error reported",
        "seconds": round(sec, 1),
    }


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    for _ in range(args.warmup):
        cpu_sample(args.cpu_shots, max(8, args.cpu_nt // 8), threads)
    vals, secs = [], []
    kind = "reference"
    for _ in range(args.steps):
        v, sec, kind = cpu_sample(args.cpu_shots, args.cpu_nt, threads)
        vals.append(v)
        secs.append(sec)
    value = cell_updates(args.cpu_shots, args.cpu_nt) * len(vals) / sum(secs)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * sum(secs) / len(secs),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded config-2 model and acquisition)",
        "config": {
            "workload": "config2 sample: 2D TM fwd+adj on the 553x1065 padded grid, "
                        f"{args.cpu_shots} shots x nt={args.cpu_nt} per step",
            "shots": args.cpu_shots, "nt": args.cpu_nt,
        },
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": f"{args.cpu_shots} shots x nt={args.cpu_nt} per step"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--shots", type=int, default=64)
    ap.add_argument("--nt", type=int, default=4000)
    ap.add_argument("--batch", type=int, default=0)
    ap.add_argument("--storage", default="fp32", choices=["fp32", "bf16"])
    ap.add_argument("--e2e-steps", type=int, default=1)
    ap.add_argument("--cpu-shots", type=int, default=4)
    ap.add_argument("--cpu-nt", type=int, default=64)
    ap.add_argument("--no-cpu-baseline", action="store_true",
                    help="skip the CPU baseline and the accuracy checks")
    ap.add_argument("--parity-shots", type=int, default=2)
    ap.add_argument("--parity-nt", type=int, default=250,
                    help="steps of the config-2 accuracy sample (0: skip)")
    ap.add_argument("--profile-every", type=int, default=2048,
                    help="time every n-th step's kernels with events in the timed region "
                         "(0: off; the roofline needs it); the 64-step block holding a timed "
                         "step runs as ordinary launches, the others replay a CUDA graph")
    ap.add_argument("--bf16-steps", type=int, default=2,
                    help="steps timed with BF16 snapshot histories (config 2's BF16 variant; "
                         "0: skip)")
    ap.add_argument("--graphs-off-steps", type=int, default=1,
                    help="steps timed again with the step graphs off (0: skip)")
    ap.add_argument("--serve-jobs", type=int, default=32,
                    help="jobs of the served mixed-size stream (0: skip the serving runs)")
    ap.add_argument("--serve-plain-jobs", type=int, default=32)
    ap.add_argument("--serve-chunk", type=int, default=32)
    ap.add_argument("--serve-load", type=float, default=0.8)
    ap.add_argument("--serve-sweep-jobs", type=int, default=200,
                    help="jobs of the bounded serving load sweep (0: skip)")
    ap.add_argument("--serve-sweep-nt-scale", type=float, default=0.05)
    ap.add_argument("--serve-sweep-loads", default="0.5,0.8,1.0")
    ap.add_argument("--tma-nt", type=int, default=400,
                    help="steps of the TMA-path comparison leg (0: skip)")
    ap.add_argument("--em3d-nt", type=int, default=1500,
                    help="steps of the 3-D (config 4) leg, checkpointed (0: skip)")
    ap.add_argument("--em3d-host-nt", type=int, default=60,
                    help="steps of the 3-D leg with the BF16 history in pinned host memory")
    ap.add_argument("--debye-nt", type=int, default=256,
                    help="steps of the Debye (config 5) leg (0: skip)")
    ap.add_argument("--debye-shots", type=int, default=8)
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "b200":
        print("warning: fewer than 3 warm-up steps", file=sys.stderr)
    if args.impl == "reference":
        run_reference(args)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
