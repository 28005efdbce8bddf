"""Shot-parallel (multi-rank) host logic on CPU: two gloo ranks.

Each rank runs the CPU oracle on its shot shard; the summed model gradient
must equal the single-process gradient over all shots (FP64, relative L2
<= 1e-12: only the order of the shot sum changes) and the gathered
receivers must equal the full run's bit for bit.  A rank that fails before a
collective makes the other rank's collective end with an error instead of
hanging (short process-group timeout).
"""

from __future__ import annotations

import os
import socket

import pytest
import torch
import torch.multiprocessing as mp

from tide_b200 import distributed as tdist


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _subset(pb, ids):
    """The prepared problem restricted to shots `ids` (a copy)."""
    from cases import clone_problem

    q = clone_problem(pb)
    S = pb.n_shots
    q.n_shots = len(ids)
    q.sources_i = pb.sources_i[ids].contiguous()
    q.receivers_i = pb.receivers_i[ids].contiguous()
    q.f = pb.f.reshape(pb.nt, S, -1)[:, ids].contiguous().reshape(-1)
    q.fields = [t[ids].contiguous() for t in pb.fields]
    if pb.batched:
        q.ca, q.cb, q.cq = (t[ids].contiguous() for t in (pb.ca, pb.cb, pb.cq))
    return q


def _problem():
    from cases import random_problem

    return random_problem(41, 18, 22, 5, 30, dtype=torch.float64, pml=4, n_rec=3)


def _fwd_adj(oracle, pb):
    S, ny, nx, nt = pb.n_shots, pb.ny, pb.nx, pb.nt
    store = (torch.zeros((nt, S, ny, nx), dtype=pb.dtype), torch.zeros((nt, S, ny, nx), dtype=pb.dtype))
    r = torch.zeros((nt, S, pb.n_rec), dtype=pb.dtype)
    oracle.forward(pb, pb.ca, pb.cb, pb.f, r, store=store, need_ca=True, need_cb=True)
    grad_r = r.clone()  # d(0.5 |r|^2)/dr
    gca, gcb, _, _ = oracle.backward(pb, pb.ca, pb.cb, grad_r, store)
    return r, gca, gcb


def _worker(rank, world, port, out_dir, fail_rank):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.join(os.path.dirname(here), "tide-gpr_b200"))
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    from oracle_harness import Oracle

    ctx = tdist.init_distributed(device="cpu", timeout_s=20.0)
    try:
        if rank == fail_rank:
            raise SystemExit(3)  # leaves before the collective
        pb = _problem()
        ids = tdist.rank_shot_indices(pb.n_shots, ctx=ctx)
        r, gca, gcb = _fwd_adj(Oracle(), _subset(pb, ids))
        g = tdist.all_reduce_tensor(torch.stack([gca, gcb]), ctx=ctx)
        full_r = tdist.gather_receiver_shards(r, ids, pb.n_shots, ctx=ctx)
        loss = tdist.all_reduce_float(0.5 * float((r * r).sum()), ctx=ctx)
        torch.save({"g": g, "r": full_r, "loss": loss}, os.path.join(out_dir, f"rank{rank}.pt"))
    except RuntimeError as exc:  # collective ended because a peer left
        torch.save({"error": str(exc)}, os.path.join(out_dir, f"rank{rank}.pt"))
    finally:
        tdist.destroy_distributed(ctx)


def test_rank_shot_partition_pure():
    ids = [tdist.rank_shot_indices(10, rank=r, world_size=3).tolist() for r in range(3)]
    assert ids == [[0, 3, 6, 9], [1, 4, 7], [2, 5, 8]]
    assert sorted(sum(ids, [])) == list(range(10))
    batches = tdist.split_rank_shots(10, 2, rank=0, world_size=3)
    assert [b.tolist() for b in batches] == [[0, 3], [6, 9]]
    pos = tdist.local_shot_positions(torch.tensor([6, 0]), torch.tensor([0, 3, 6, 9]))
    assert pos.tolist() == [2, 0]
    with pytest.raises(ValueError):
        tdist.local_shot_positions(torch.tensor([1]), torch.tensor([0, 3]))
    with pytest.raises(ValueError):
        tdist.rank_shot_indices(4, rank=2, world_size=2)


def test_two_rank_gradient_equals_single_process(tmp_path, oracle):
    port = _free_port()
    mp.spawn(_worker, args=(2, port, str(tmp_path), -1), nprocs=2, join=True)
    res = [torch.load(tmp_path / f"rank{r}.pt") for r in range(2)]
    r_full, gca, gcb = _fwd_adj(oracle, _problem())
    g = torch.stack([gca, gcb])
    for rr in res:
        err = float((rr["g"] - g).norm() / g.norm())
        assert err <= 1e-12, err
        assert abs(rr["loss"] - 0.5 * float((r_full * r_full).sum())) <= 1e-12 * abs(rr["loss"])
    assert torch.equal(res[0]["r"], r_full)
    assert res[1]["r"] is None


def test_rank_leaving_before_collective_is_an_error_not_a_hang(tmp_path):
    port = _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_worker, args=(r, 2, port, str(tmp_path), 1)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert not p.is_alive(), "a rank hung"
    assert procs[1].exitcode == 3
    out = torch.load(tmp_path / "rank0.pt")
    assert "error" in out
