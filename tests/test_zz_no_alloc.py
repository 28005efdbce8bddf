"""The allocation-free forward (maxwell_tm_2_float_forward_noalloc_cuda).

Callers that may not allocate device memory while the solver runs (allocator
or memory-pool callbacks, applications that reserve all device memory up
front) use this entry point: its per-call scratch lives in a fixed device
array inside the library.  These tests call it through the C ABI and check it
against the regular forward on two calls in a row (the second call must not be
disturbed by what the first left in the shared array), and check that a
problem larger than the array is refused with a message.

This file is collected last on purpose; it also passes on its own.
"""

from __future__ import annotations

import pytest
import torch

from cases import clone_problem, random_problem
from oracle_harness import rel_l2
from tide_b200 import _native as nat
from tide_b200 import tm2d

pytestmark = pytest.mark.gpu
TOL = 1e-5  # FP32 parity bar: relative L2


def _noalloc_fn():
    lib = nat.load()
    fn = lib.maxwell_tm_2_float_forward_noalloc_cuda
    fn.argtypes = nat.argtypes("maxwell_tm_forward", "float")
    fn.restype = None
    return fn


def _call(fn, pb, r, start_t, nt):
    ey, hx, hz, mex, mez, mhx, mhz = pb.fields
    prof = [nat.ptr(pb.profiles[n]) for n in tm2d._PROFILE_ORDER]
    fn(
        nat.ptr(pb.ca), nat.ptr(pb.cb), nat.ptr(pb.cq), nat.ptr(pb.f),
        nat.ptr(ey), nat.ptr(hx), nat.ptr(hz), nat.ptr(mex), nat.ptr(mez), nat.ptr(mhx), nat.ptr(mhz),
        0, 0, 0, 0, 0, nat.ptr(r), 0, *prof, nat.ptr(pb.sources_i), nat.ptr(pb.receivers_i),
        pb.rdy, pb.rdx, pb.dt, nt, pb.n_shots, pb.ny, pb.nx, pb.n_src, pb.n_rec, 1, False,
        pb.batched, pb.batched, pb.batched, start_t, pb.pml_y0, pb.pml_x0, pb.pml_y1, pb.pml_x1,
        0, pb.device.index or 0, int(torch.cuda.current_stream(pb.device).cuda_stream),
    )
    nat.check("noalloc forward")


def test_noalloc_forward_matches_regular_on_two_calls(cuda_device):
    fn = _noalloc_fn()
    # Two different problems back to back: different grids, shot counts and
    # point sets, so stale lists from call 1 would corrupt call 2.
    for seed, ny, nx, shots, n_rec in ((301, 61, 97, 3, 9), (302, 140, 75, 2, 30)):
        pb = random_problem(seed, ny, nx, shots, 80, n_rec=n_rec)
        ref = clone_problem(pb, cuda_device)
        new = clone_problem(pb, cuda_device)
        r_ref = torch.zeros((ref.nt, ref.n_shots, ref.n_rec), device=cuda_device)
        r_new = torch.zeros_like(r_ref)
        tm2d.native_forward(ref, ref.ca, ref.cb, ref.f, r_ref, 0, ref.nt)
        _call(fn, new, r_new, 0, new.nt)
        torch.cuda.synchronize()
        assert rel_l2(r_new, r_ref) <= TOL
        assert torch.equal(r_new.cpu(), r_ref.cpu())
        for a, b in zip(new.fields, ref.fields):
            assert rel_l2(a, b) <= TOL
            assert torch.equal(a.cpu(), b.cpu())


def test_noalloc_forward_rejects_oversize(cuda_device):
    fn = _noalloc_fn()
    lib = nat.load()
    lib.tide_b200_clear_error()
    pb = random_problem(303, 20, 24, 1, 4)
    g = clone_problem(pb, cuda_device)
    # Claim a huge shot count: the size check refuses the call before any GPU
    # work touches the (much smaller) buffers.
    ey, hx, hz, mex, mez, mhx, mhz = g.fields
    prof = [nat.ptr(g.profiles[n]) for n in tm2d._PROFILE_ORDER]
    r = torch.zeros((g.nt, 1, g.n_rec), device=cuda_device)
    fn(
        nat.ptr(g.ca), nat.ptr(g.cb), nat.ptr(g.cq), nat.ptr(g.f),
        nat.ptr(ey), nat.ptr(hx), nat.ptr(hz), nat.ptr(mex), nat.ptr(mez), nat.ptr(mhx), nat.ptr(mhz),
        0, 0, 0, 0, 0, nat.ptr(r), 0, *prof, nat.ptr(g.sources_i), nat.ptr(g.receivers_i),
        g.rdy, g.rdx, g.dt, g.nt, 60000, 4096, 4096, g.n_src, g.n_rec, 1, False,
        False, False, False, 0, g.pml_y0, g.pml_x0, g.pml_y1, g.pml_x1,
        0, 0, int(torch.cuda.current_stream(cuda_device).cuda_stream),
    )
    assert lib.tide_b200_last_status() != 0
    assert b"scratch words" in lib.tide_b200_last_error()
    lib.tide_b200_clear_error()
    torch.cuda.synchronize()
