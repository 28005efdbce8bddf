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
    """A problem needing more scratch than the fixed array is refused.  The
    buffers match the arguments (one shot, a small grid, 2.2 M source entries
    per shot, all with index -1, one step), so even if the size check ever
    stopped refusing the call every access would stay in bounds."""
    fn = _noalloc_fn()
    lib = nat.load()
    lib.tide_b200_clear_error()
    pb = random_problem(303, 20, 24, 1, 1)
    g = clone_problem(pb, cuda_device)
    n_src = 2_200_000  # 2 (tiles + 1) + 2 n_src words > 4 Mi words
    src_i = torch.full((1, n_src), -1, dtype=torch.int64, device=cuda_device)
    f = torch.zeros((1, 1, n_src), device=cuda_device)
    ey, hx, hz, mex, mez, mhx, mhz = g.fields
    prof = [nat.ptr(g.profiles[n]) for n in tm2d._PROFILE_ORDER]
    r = torch.zeros((1, 1, g.n_rec), device=cuda_device)
    fn(
        nat.ptr(g.ca), nat.ptr(g.cb), nat.ptr(g.cq), nat.ptr(f),
        nat.ptr(ey), nat.ptr(hx), nat.ptr(hz), nat.ptr(mex), nat.ptr(mez), nat.ptr(mhx), nat.ptr(mhz),
        0, 0, 0, 0, 0, nat.ptr(r), 0, *prof, nat.ptr(src_i), nat.ptr(g.receivers_i),
        g.rdy, g.rdx, g.dt, 1, 1, g.ny, g.nx, n_src, g.n_rec, 1, False,
        False, False, False, 0, g.pml_y0, g.pml_x0, g.pml_y1, g.pml_x1,
        0, cuda_device.index or 0, int(torch.cuda.current_stream(cuda_device).cuda_stream),
    )
    assert lib.tide_b200_last_status() != 0
    assert b"scratch words" in lib.tide_b200_last_error()
    lib.tide_b200_clear_error()
    torch.cuda.synchronize()


def _driver():
    import ctypes

    cu = ctypes.CDLL("libcuda.so.1")
    cu.cuDeviceGetDefaultMemPool.argtypes = [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int]
    cu.cuMemPoolGetAttribute.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    cu.cuMemPoolSetAttribute.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
    return cu


def test_noalloc_forward_allocates_nothing(cuda_device):
    """The call's promise: no allocation of any kind.  The regular forward
    takes its point lists from the device's default stream-ordered pool, so
    the pool's high-water mark of used memory (reset just before the call)
    would grow with it; here it must not, and the device's free memory must
    not change either."""
    import ctypes

    used_current, used_high = 7, 8  # CU_MEMPOOL_ATTR_USED_MEM_CURRENT / _HIGH
    fn = _noalloc_fn()
    pb = random_problem(304, 90, 130, 4, 60, n_rec=25)
    g = clone_problem(pb, cuda_device)
    r = torch.zeros((g.nt, g.n_shots, g.n_rec), device=cuda_device)
    _call(fn, g, r, 0, g.nt)  # first call on the device: may load the module
    torch.cuda.synchronize()
    cu = _driver()
    pool = ctypes.c_void_p()
    assert cu.cuDeviceGetDefaultMemPool(ctypes.byref(pool), cuda_device.index or 0) == 0
    zero = ctypes.c_uint64(0)
    assert cu.cuMemPoolSetAttribute(pool, used_high, ctypes.byref(zero)) == 0
    cur = ctypes.c_uint64(0)
    assert cu.cuMemPoolGetAttribute(pool, used_current, ctypes.byref(cur)) == 0
    free0, _ = torch.cuda.mem_get_info(cuda_device)
    _call(fn, g, r, 0, g.nt)
    torch.cuda.synchronize()
    high = ctypes.c_uint64(0)
    assert cu.cuMemPoolGetAttribute(pool, used_high, ctypes.byref(high)) == 0
    free1, _ = torch.cuda.mem_get_info(cuda_device)
    assert high.value <= cur.value, (high.value, cur.value)
    assert free1 == free0
