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


# ---------------------------------------------------------------- bench step


def _bench_case(dtype):
    from tide_b200 import physics as ph

    g = torch.Generator().manual_seed(7)
    ny, nx, S, nt = 16, 20, 5, 30
    eps = (2.0 + 4.0 * torch.rand((ny, nx), generator=g, dtype=torch.float64)).to(dtype)
    sig = (0.004 * torch.rand((ny, nx), generator=g, dtype=torch.float64)).to(dtype)
    mu = torch.ones((ny, nx), dtype=dtype)
    dt = 3e-11
    amp = ph.ricker(900e6, nt, dt, dtype=dtype).view(1, 1, nt).repeat(S, 1, 1)
    amp = amp * (1.0 + torch.arange(S, dtype=dtype)).view(S, 1, 1)
    src = torch.tensor([[[4, 3 + 3 * i]] for i in range(S)])
    rec = torch.tensor([[[5, 2 + 4 * j] for j in range(4)]] * S)
    return dict(eps=eps, sig=sig, mu=mu, dx=0.02, dt=dt, amp=amp, src=src, rec=rec, S=S)


def _bench_batch_fn(c):
    """bench.py's per-batch step with the C oracle (CPU) in place of the GPU
    propagator: forward, loss 0.5 |r|^2, backward into eps/sigma."""
    from oracle_harness import Oracle, OracleTM
    from tide_b200.tm2d import prepare_tm2d

    oracle = Oracle()

    def fn(eps, sig, ids):
        pb = prepare_tm2d(eps, sig, c["mu"], c["dx"], c["dt"], c["amp"][ids], c["src"][ids],
                          c["rec"][ids], stencil=2, pml_width=4)
        r = OracleTM.apply(pb.ca, pb.cb, pb.f, pb, oracle, 1, 0)
        loss = 0.5 * (r * r).sum()
        loss.backward()
        return loss.detach()

    return fn


def _bench_worker(rank, world, port, out_dir, dtype):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, here)
    sys.path.insert(0, os.path.dirname(here))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "tide-gpr_b200"))
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank),
                      MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import bench

    ctx = tdist.init_distributed(device="cpu", timeout_s=30.0)
    try:
        c = _bench_case(dtype)
        g, loss = bench.sharded_gradient(c["eps"], c["sig"], c["S"], 2, _bench_batch_fn(c), ctx)
        torch.save({"g": g, "loss": loss}, os.path.join(out_dir, f"bench{rank}.pt"))
    finally:
        tdist.destroy_distributed(ctx)


@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-12), (torch.float32, 1e-5)])
def test_bench_step_sharded_equals_single_rank(tmp_path, dtype, tol):
    """bench.py's multi-GPU step: the ranks split the shots, each
    back-propagates its shard in batches and the eps/sigma gradients are
    summed once.  The two-rank gradient and loss equal the single-rank ones
    (only the order of the shot sum changes: FP64 1e-12, FP32 1e-5 relative
    L2)."""
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench

    port = _free_port()
    mp.spawn(_bench_worker, args=(2, port, str(tmp_path), dtype), nprocs=2, join=True)
    c = _bench_case(dtype)
    g1, loss1 = bench.sharded_gradient(c["eps"], c["sig"], c["S"], 2, _bench_batch_fn(c), None)
    assert float(g1.norm()) > 0
    for rank in range(2):
        res = torch.load(tmp_path / f"bench{rank}.pt")
        err = float((res["g"] - g1).norm() / g1.norm())
        assert err <= tol, (rank, err)
        assert abs(float(res["loss"]) - float(loss1)) <= tol * abs(float(loss1))
