"""Host logic of the serving loop (CPU only): job plans, segment programs,
chunk stepping, admission and the seeded job stream."""

from __future__ import annotations

import pytest
import torch

from tide_b200 import serve as sv

GB = 1 << 30
KW = dict(item=4, history_limit=16 * GB, group_limit=32 * GB, chunk_steps=32)


def test_plan_modes_and_groups():
    fwd = sv.plan_job(300, 600, 8, 3000, 1, 150, False, 1, **KW)
    assert fwd.mode == "forward" and fwd.groups == ((0, 8),)
    small = sv.plan_job(100, 200, 2, 500, 1, 50, True, 1, **KW)
    assert small.mode == "device" and small.seg_len == 0
    ck = sv.plan_job(300, 600, 8, 6000, 1, 150, True, 3, **KW)
    assert ck.mode == "checkpoint"
    assert ck.seg_len % 32 == 0 and ck.seg_len % 3 == 0
    big = sv.plan_job(1066, 2090, 32, 6000, 1, 256, True, 1, **KW)
    assert len(big.groups) > 1
    assert big.groups[0][0] == 0 and big.groups[-1][1] == 32
    assert all(a[1] == b[0] for a, b in zip(big.groups, big.groups[1:]))
    assert max(big.group_bytes) <= KW["group_limit"]
    # the plan depends on the job alone
    assert sv.plan_job(1066, 2090, 32, 6000, 1, 256, True, 1, **KW) == big


def test_group_bytes_monotone():
    a = sv.group_bytes(200, 300, 4, 1000, 1, 10, "device", 0, 1, 4)
    b = sv.group_bytes(200, 300, 4, 1000, 1, 10, "device", 0, 1, 2)
    c = sv.group_bytes(200, 300, 4, 1000, 1, 10, "checkpoint", 64, 1, 4)
    f = sv.group_bytes(200, 300, 4, 1000, 1, 10, "forward", 0, 1, 4)
    assert f < c < b < a


@pytest.mark.parametrize("nt,k,seg", [(100, 1, 32), (100, 3, 48), (96, 2, 32), (7, 1, 32)])
def test_checkpoint_program_covers_every_step(nt, k, seg):
    segs = sv.program("checkpoint", nt, k, seg)
    fwd = [s for s in segs if s.phase == sv.FORWARD]
    assert [s.start for s in fwd] == list(range(0, nt, seg))
    assert sum(s.steps for s in fwd) == nt
    assert all(s.hooks == (f"save:{i}",) for i, s in enumerate(fwd))
    rest = segs[len(fwd):]
    assert len(rest) == 2 * len(fwd)
    adj_steps = []
    for i in range(len(fwd)):
        rec, adj = rest[2 * i], rest[2 * i + 1]
        idx = len(fwd) - 1 - i
        assert rec.phase == sv.FORWARD_STORE and adj.phase == sv.ADJOINT
        assert rec.hooks[0] == f"restore:{idx}"
        assert ("grad_r" in rec.hooks) == (i == 0)
        assert rec.start == fwd[idx].start and rec.steps == fwd[idx].steps
        assert adj.start == rec.start + rec.steps and adj.steps == rec.steps
        assert rec.q0 == adj.q0 == rec.start // k
        adj_steps += list(range(adj.start - 1, adj.start - 1 - adj.steps, -1))
    assert adj_steps == list(range(nt - 1, -1, -1))


def test_device_program():
    segs = sv.program("device", 50, 1, 0)
    assert [(s.phase, s.start, s.steps, s.hooks) for s in segs] == [
        (sv.FORWARD_STORE, 0, 50, ()), (sv.ADJOINT, 50, 50, ("grad_r",))]
    assert [(s.phase, s.start, s.steps) for s in sv.program("forward", 9, 1, 0)] == [
        (sv.FORWARD, 0, 9)]


def _job(S=3, nt=70, grad=True, k=1):
    eps = torch.full((20, 30), 4.0)
    amp = torch.zeros((S, 1, nt))
    src = torch.zeros((S, 1, 2), dtype=torch.long)
    rec = torch.zeros((S, 2, 2), dtype=torch.long)
    return sv.ModelingJob(eps, torch.zeros_like(eps), torch.ones_like(eps), 0.02, 1e-11, amp,
                          src, rec, pml_width=5, gradient=grad,
                          model_gradient_sampling_interval=k)


def test_task_stepping_in_chunks():
    job = _job(nt=70)
    plan = sv.JobPlan(((0, 3),), "checkpoint", 32, (0,))
    t = sv._Task(job, plan, 0)
    seen = []
    while not t.finished_stepping:
        seg, t0, n, first = t.next_plan(16)
        seen.append((seg.phase, t0, n, first))
        t.advance(n)
    fwd = [x for x in seen if x[0] == sv.FORWARD]
    assert [x[1] for x in fwd] == [0, 16, 32, 48, 64]
    assert [x[3] for x in fwd] == [True, False, True, False, True]
    adj = [x for x in seen if x[0] == sv.ADJOINT]
    assert adj[0][1] == 70 and adj[0][2] == 6  # last segment [64, 70)
    assert t.adj_steps == 70
    # adjoint chunks count down from each segment's end
    assert [x[1] for x in adj] == [70, 64, 48, 32, 16]


def test_select_admissions_fifo_first_fit_and_bypass_limit():
    take, byp = sv.select_admissions([5, 3, 4], 0, 0, 10, 8, 0, 2)
    assert take == [0, 1] and byp == 1  # 4 does not fit behind 5+3: counted as blocked
    take, byp = sv.select_admissions([8, 1, 1], 5, 1, 10, 8, 0, 2)
    assert take == [1, 2] and byp == 1  # the 8 is blocked, smaller groups pass it
    take, byp = sv.select_admissions([8, 1, 1], 5, 1, 10, 8, 2, 2)
    assert take == [] and byp == 3  # passed too often: nothing passes it any more
    take, byp = sv.select_admissions([8, 1], 0, 0, 10, 8, 3, 2)
    assert take == [0, 1] and byp == 0
    take, _ = sv.select_admissions([1, 1, 1], 0, 6, 10, 8, 0, 2)
    assert take == [0, 1]  # slot limit


def test_percentile():
    v = [5.0, 1.0, 3.0, 2.0, 4.0]
    assert sv.percentile(v, 50) == 3.0
    assert sv.percentile(v, 0) == 1.0 and sv.percentile(v, 100) == 5.0
    assert sv.percentile(v, 25) == 2.0
    assert abs(sv.percentile(list(range(101)), 99) - 99.0) < 1e-12


def test_mixed_stream_is_seeded_and_in_range():
    a = sv.mixed_stream(40, seed=3, rate=10.0)
    b = sv.mixed_stream(40, seed=3, rate=10.0)
    for x, y in zip(a, b):
        assert x.epsilon.shape == y.epsilon.shape and x.nt == y.nt and x.arrival == y.arrival
        assert torch.equal(x.epsilon, y.epsilon)
    for j in a:
        nz, nx = j.epsilon.shape
        assert 128 <= nz <= 1024 and 256 <= nx <= 2048
        assert 1000 <= j.nt <= 6000 and 1 <= j.n_shots <= 32
        assert float(j.epsilon.min()) >= 3.0 and float(j.epsilon.max()) <= 25.0
    arr = [j.arrival for j in a]
    assert arr == sorted(arr) and arr[0] > 0
    frac = sum(j.gradient for j in sv.mixed_stream(400, seed=3)) / 400
    assert 0.22 < frac < 0.38


def test_load_defers_on_allocator_oom(monkeypatch):
    """A load the byte budget admits but the fragmented allocator cannot place
    is retried once after the cache goes back to the driver, then deferred
    while other jobs are resident, and raised when none is."""
    import torch

    monkeypatch.setattr(torch.cuda, "synchronize", lambda *a, **k: None)
    monkeypatch.setattr(torch.cuda, "empty_cache", lambda: None)

    class Task:
        def __init__(self):
            self.out = {}

    class Busy:
        device = "cuda:0"

        def __init__(self, resident, fail):
            self.resident, self.fail, self.calls = resident, fail, 0
            self.stats = {"deferred_oom": 0}

        def _load(self, t):
            self.calls += 1
            t.out["partial"] = 1
            if self.calls <= self.fail:
                raise torch.OutOfMemoryError("fragmented")

    s, t = Busy(["resident job"], fail=2), Task()
    assert sv.TMServer._load_or_defer(s, t) is False
    assert s.calls == 2 and s.stats["deferred_oom"] == 1 and t.out == {}
    s = Busy([], fail=2)
    with pytest.raises(torch.OutOfMemoryError):
        sv.TMServer._load_or_defer(s, Task())
    s = Busy(["resident job"], fail=1)
    assert sv.TMServer._load_or_defer(s, Task()) is True and s.calls == 2
