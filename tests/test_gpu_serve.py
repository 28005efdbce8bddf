"""Serving loop on the GPU: continuous batching gives each job the same bits
alone, in a mix and through the per-job public API.

Jobs of different grid shapes, shot counts, nt, gradient sampling intervals
and plans (forward only, gradient with device history, gradient by
checkpoint segments, shot groups) are served together; every receiver trace,
loss and epsilon/sigma gradient must be bit-identical to the same job served
alone and to ``run_plain`` (``tide_b200.maxwelltm`` with the same plan).  The
FP32 bar (relative L2 <= 1e-5) is asserted next to each equality.
"""

from __future__ import annotations

import copy

import pytest
import torch

from oracle_harness import rel_l2
from tide_b200 import serve as sv

pytestmark = pytest.mark.gpu
TOL = 1e-5
MB = 1 << 20
CFG = dict(memory_budget=512 * MB, history_limit=1 * MB, group_limit=3 * MB,
           chunk_steps=16, max_slots=8)


def _job(seed, ny, nx, S, nt, grad, k=1, n_rec=5, observed=True):
    g = torch.Generator().manual_seed(seed)
    layers = 2.0 + 10.0 * torch.rand(4, generator=g, dtype=torch.float64)
    rows = torch.clamp(torch.arange(ny) * 4 // ny, max=3)
    eps = (layers[rows][:, None] + 0.3 * torch.rand((ny, nx), generator=g, dtype=torch.float64))
    sig = 0.004 * torch.rand((ny, nx), generator=g, dtype=torch.float64)
    dx = 0.02
    dt = 0.9 / (2.0 / dx**2) ** 0.5 / (299792458.0 / float(eps.min()) ** 0.5)
    t = torch.arange(nt, dtype=torch.float64) * dt
    amp = torch.sin(2 * torch.pi * 7e8 * t) * torch.exp(-((t - 2e-9) / 8e-10) ** 2)
    amp = (amp.view(1, 1, nt) * (1 + 0.1 * torch.arange(S)).view(S, 1, 1)).float()
    src = torch.stack([torch.randint(0, ny, (S, 1), generator=g),
                       torch.randint(0, nx, (S, 1), generator=g)], -1)
    rec = torch.stack([torch.randint(0, ny, (S, n_rec), generator=g),
                       torch.randint(0, nx, (S, n_rec), generator=g)], -1)
    obs = (0.01 * torch.randn((nt, S, n_rec), generator=g)).float() if (grad and observed) else None
    return sv.ModelingJob(eps.float(), sig.float(), torch.ones((ny, nx)), dx, dt, amp, src, rec,
                          pml_width=5, gradient=grad, observed=obs,
                          model_gradient_sampling_interval=k, job_id=seed)


def _jobs():
    return [
        _job(1, 30, 40, 1, 50, False),
        _job(2, 37, 53, 3, 71, True),             # checkpoint, shot groups
        _job(3, 24, 33, 1, 45, True, k=2),        # device history, k = 2
        _job(4, 45, 29, 2, 64, False, n_rec=1),
        _job(5, 33, 61, 2, 90, True, k=3),        # checkpoint, k = 3
        _job(6, 28, 28, 1, 33, True, observed=False),
    ]


def _same(a, b, what):
    if a is None or b is None:
        assert a is None and b is None, what
        return
    if isinstance(a, float):
        assert a == b, f"{what}: {a} != {b}"
        return
    err = rel_l2(a, b)
    assert err <= TOL, f"{what}: rel l2 {err}"
    assert torch.equal(a, b), f"{what}: not bit-identical (rel l2 {err})"


def _check(x, y, tag):
    _same(x.receivers, y.receivers, f"{tag} receivers")
    _same(x.loss, y.loss, f"{tag} loss")
    _same(x.grad_epsilon, y.grad_epsilon, f"{tag} grad eps")
    _same(x.grad_sigma, y.grad_sigma, f"{tag} grad sigma")


def _serve(jobs, **kw):
    cfg = dict(CFG, **kw)
    with sv.TMServer("cuda", **cfg) as srv:
        out = {r.job_id: r for r in srv.serve([copy.copy(j) for j in jobs], realtime=False)}
        plans = {j.job_id: srv.plan(j) for j in jobs}
        launches = srv.launches()
    return out, plans, launches


def test_plans_cover_every_mode(cuda_device):
    with sv.TMServer("cuda", **CFG) as srv:
        plans = [srv.plan(j) for j in _jobs()]
    modes = [p.mode for p in plans]
    assert {"forward", "device", "checkpoint"} <= set(modes)
    assert any(len(p.groups) > 1 for p in plans)


def test_mix_equals_alone_and_plain(cuda_device):
    jobs = _jobs()
    mix, plans, launches = _serve(jobs)
    assert sorted(mix) == [j.job_id for j in jobs]
    assert launches > 0
    for job in jobs:
        alone, _, _ = _serve([job])
        _check(mix[job.job_id], alone[job.job_id], f"job {job.job_id} mix vs alone")
        plain = sv.run_plain(job, plans[job.job_id])
        _check(mix[job.job_id], plain, f"job {job.job_id} served vs plain")


def test_graph_and_eager_chunks_agree(cuda_device):
    jobs = _jobs()[:4]
    a, _, _ = _serve(jobs, use_graphs=True)
    b, _, _ = _serve(jobs, use_graphs=False, chunk_steps=7)
    for j in jobs:
        _check(a[j.job_id], b[j.job_id], f"job {j.job_id} graph vs eager")


def test_bf16_snapshots_match_plain(cuda_device):
    jobs = [j for j in _jobs() if j.gradient][:3]
    out, plans, _ = _serve(jobs, storage_compression=True)
    for j in jobs:
        plain = sv.run_plain(j, plans[j.job_id], storage_compression=True)
        _check(out[j.job_id], plain, f"job {j.job_id} bf16")


def test_poisson_arrivals_realtime(cuda_device):
    jobs = _jobs()
    for i, j in enumerate(jobs):
        j.arrival = 0.02 * i
    ref, _, _ = _serve(jobs)
    with sv.TMServer("cuda", **CFG) as srv:
        res = srv.serve([copy.copy(j) for j in jobs], realtime=True)
        assert srv.stats["max_resident"] >= 1
    assert len(res) == len(jobs)
    for r in res:
        assert r.finished >= r.admitted >= r.arrival - 1e-9
        _check(r, ref[r.job_id], f"job {r.job_id} realtime")


@pytest.mark.parametrize("fused_threshold", [0, -1])
def test_direct_slots_match_table_and_plain(cuda_device, fused_threshold):
    """Groups at or above direct_cells run the per-call kernels (pair, or the
    fused pitched forward when allowed) on the engine's streams next to the
    table walk of the small groups: same bits as the table walk and as the
    per-job path."""
    from tide_b200 import _native as nat

    jobs = _jobs()
    ref, plans, _ = _serve(jobs, direct_cells=-1)
    old = nat.set_fused_threshold(fused_threshold)
    try:
        mixed, _, _ = _serve(jobs, direct_cells=3000)
        alone, _, _ = _serve(jobs[1:2], direct_cells=3000)
        plain = sv.run_plain(jobs[4], plans[jobs[4].job_id])
    finally:
        nat.set_fused_threshold(old)
    for j in jobs:
        _check(mixed[j.job_id], ref[j.job_id], f"job {j.job_id} direct vs table")
    _check(alone[jobs[1].job_id], ref[jobs[1].job_id], "direct alone")
    _check(mixed[jobs[4].job_id], plain, "direct vs plain")
