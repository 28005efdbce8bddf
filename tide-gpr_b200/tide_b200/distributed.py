"""Shot-parallel helpers: one process per GPU, shots sharded across ranks.

Shots are independent given a shared model, so a fwd+adj pass shards them
across ranks with no data-path communication; the one exchange is the sum of
the model gradients (and of the loss) per gradient evaluation.  Mirrors the
reference's shot-parallel workflow helpers (src/tide/workflow/distributed.py:
16-300: context, strided shot ownership, mini-batches of the local shard,
gradient / scalar all-reduce, receiver gather on one rank).  The collective
backend is NCCL for CUDA devices and gloo on CPU.
"""

from __future__ import annotations

import datetime
import os
from dataclasses import dataclass

import torch
import torch.distributed as dist


@dataclass(frozen=True)
class DistributedContext:
    """Where this worker runs and whether a process group is active."""

    enabled: bool = False
    rank: int = 0
    world_size: int = 1
    local_rank: int = 0
    device: torch.device = torch.device("cpu")
    backend: str | None = None

    @property
    def is_main(self) -> bool:
        return self.rank == 0


def _env(name: str, default: int) -> int:
    v = os.environ.get(name)
    if v is None:
        return default
    try:
        return int(v)
    except ValueError as exc:
        raise ValueError(f"{name} must be an integer, got {v!r}") from exc


def init_distributed(*, enabled: bool = True, device: str | torch.device | None = None,
                     backend: str | None = None, timeout_s: float = 300.0) -> DistributedContext:
    """Join the process group described by RANK / WORLD_SIZE / LOCAL_RANK /
    MASTER_ADDR / MASTER_PORT (torchrun's variables).  A world of one, or
    enabled=False, returns a disabled context without a process group."""
    local = _env("LOCAL_RANK", 0)
    if device is None or str(device) == "auto":
        dev = torch.device("cuda", local) if torch.cuda.is_available() else torch.device("cpu")
    else:
        dev = torch.device(device)
        if dev.type == "cuda" and dev.index is None:
            dev = torch.device("cuda", local)
    if dev.type == "cuda":
        if not torch.cuda.is_available() or (dev.index or 0) >= torch.cuda.device_count():
            raise RuntimeError(f"CUDA device {dev} is not available to local rank {local}")
        torch.cuda.set_device(dev)
    world = _env("WORLD_SIZE", 1)
    rank = _env("RANK", 0)
    if not enabled or world <= 1:
        return DistributedContext(rank=rank, world_size=world, local_rank=local, device=dev)
    if not dist.is_available():
        raise RuntimeError("torch.distributed is not available")
    be = backend or ("nccl" if dev.type == "cuda" else "gloo")
    if not dist.is_initialized():
        dist.init_process_group(be, rank=rank, world_size=world,
                                timeout=datetime.timedelta(seconds=timeout_s))
    return DistributedContext(True, dist.get_rank(), dist.get_world_size(), local, dev,
                              dist.get_backend())


def destroy_distributed(ctx: DistributedContext | None) -> None:
    if ctx is not None and ctx.enabled and dist.is_initialized():
        dist.destroy_process_group()


def barrier(ctx: DistributedContext | None) -> None:
    if ctx is not None and ctx.enabled:
        dist.barrier()


def rank_shot_indices(n_shots: int, *, ctx: DistributedContext | None = None, rank: int | None = None,
                      world_size: int | None = None, device=None) -> torch.Tensor:
    """Global shot ids owned by a rank: every world_size-th shot starting at
    the rank (balanced to within one shot; order preserved)."""
    if n_shots < 0:
        raise ValueError("n_shots must be non-negative")
    if ctx is not None and ctx.enabled:
        r, w = ctx.rank, ctx.world_size
    else:
        r = 0 if rank is None else int(rank)
        w = 1 if world_size is None else int(world_size)
    if w <= 0 or not 0 <= r < w:
        raise ValueError(f"need 0 <= rank < world_size, got rank={r}, world_size={w}")
    if device is None and ctx is not None:
        device = ctx.device
    return torch.arange(r, int(n_shots), w, device=device, dtype=torch.long)


def split_rank_shots(n_shots: int, batch_size: int, **kw) -> list[torch.Tensor]:
    """The rank's shot ids in mini-batches of at most batch_size."""
    if batch_size <= 0:
        raise ValueError("batch_size must be positive")
    return list(rank_shot_indices(n_shots, **kw).split(int(batch_size)))


def local_shot_positions(global_ids: torch.Tensor, local_ids: torch.Tensor) -> torch.Tensor:
    """Positions of global shot ids inside a sorted local shard."""
    if global_ids.ndim != 1 or local_ids.ndim != 1:
        raise ValueError("shot ids must be 1-D")
    g = global_ids.detach().cpu().long()
    loc = local_ids.detach().cpu().long()
    if loc.numel() > 1 and bool((loc[1:] < loc[:-1]).any()):
        raise ValueError("local shot ids must be sorted ascending")
    pos = torch.searchsorted(loc, g)
    ok = pos < loc.numel()
    ok[ok.clone()] = loc[pos[ok]] == g[ok]
    if not bool(ok.all()):
        raise ValueError(f"shot ids not in the local shard: {g[~ok].tolist()}")
    return pos.to(global_ids.device)


def all_reduce_gradients(params, *, ctx: DistributedContext | None) -> None:
    """Sum .grad of every parameter that requires grad across ranks (a
    missing .grad counts as zeros), in place."""
    if ctx is None or not ctx.enabled:
        return
    for p in params:
        if not p.requires_grad:
            continue
        if p.grad is None:
            p.grad = torch.zeros_like(p)
        dist.all_reduce(p.grad, op=dist.ReduceOp.SUM)


def all_reduce_tensor(t: torch.Tensor, *, ctx: DistributedContext | None,
                      op=dist.ReduceOp.SUM) -> torch.Tensor:
    """A reduced copy of t (t itself when not distributed)."""
    if ctx is None or not ctx.enabled:
        return t
    out = t.clone()
    dist.all_reduce(out, op=op)
    return out


def all_reduce_float(v: float, *, ctx: DistributedContext | None, device=None) -> float:
    if ctx is None or not ctx.enabled:
        return float(v)
    t = torch.tensor(float(v), dtype=torch.float64, device=device or ctx.device)
    dist.all_reduce(t)
    return float(t.item())


def gather_receiver_shards(local: torch.Tensor, local_ids: torch.Tensor, n_shots: int, *,
                           ctx: DistributedContext | None, dst: int = 0,
                           shot_dim: int = 1) -> torch.Tensor | None:
    """Assemble [.., n_shots, ..] receiver data on rank dst from the ranks'
    shards (shot dimension `shot_dim`, [nt, shots, n_rec] by default);
    other ranks get None."""
    if ctx is None or not ctx.enabled:
        return local
    payload = (local.detach().cpu(), local_ids.detach().cpu().long())
    objs = [None] * ctx.world_size if ctx.rank == dst else None
    dist.gather_object(payload, object_gather_list=objs, dst=dst)
    if ctx.rank != dst:
        return None
    shape = list(local.shape)
    shape[shot_dim] = int(n_shots)
    full = torch.zeros(shape, dtype=local.dtype)
    seen = torch.zeros(int(n_shots), dtype=torch.bool)
    for shard, ids in objs:
        if ids.numel():
            full.index_copy_(shot_dim, ids, shard)
            seen[ids] = True
    if not bool(seen.all()):
        raise RuntimeError(f"receiver shards missing shots {(~seen).nonzero().flatten().tolist()}")
    return full
