"""Host-side policy and helpers of the TM2D / 3-D paths (CPU only)."""

from __future__ import annotations

import pytest
import torch

from tide_b200 import physics as ph
from tide_b200 import storage as stg
from tide_b200 import tm2d


@pytest.mark.parametrize("shape,pad", [((5, 7), [2, 3, 1, 4]), ((3, 5, 7), [0, 2, 3, 0]),
                                       ((4, 5, 6), [1, 2, 0, 3, 2, 1]),
                                       ((2, 4, 5, 6), [3, 1, 2, 2, 1, 0])])
def test_replicate_pad_matches_torch_and_is_deterministic(shape, pad):
    t = torch.randn(shape, dtype=torch.float64, requires_grad=True)
    nd = len(pad) // 2
    order = []
    for i in range(nd - 1, -1, -1):
        order += [pad[2 * i], pad[2 * i + 1]]
    x = t.reshape(1, -1, *t.shape[t.ndim - nd:])  # (batch 1, channels, *padded dims)
    ref = torch.nn.functional.pad(x, order, mode="replicate")
    ref = ref.reshape(*t.shape[: t.ndim - nd], *ref.shape[-nd:])
    out = ph.replicate_pad(t, pad)
    assert torch.equal(out, ref)
    w = torch.randn(out.shape, dtype=torch.float64)
    (g,) = torch.autograd.grad((out * w).sum(), t)
    (g_ref,) = torch.autograd.grad((ref * w).sum(), t)
    assert torch.allclose(g, g_ref, rtol=1e-13, atol=1e-13)


def test_checkpoint_segment_length():
    assert tm2d.checkpoint_steps(400, 1, 0) == 20  # about sqrt(nt)
    assert tm2d.checkpoint_steps(400, 3, 10) == 12  # rounded up to the sampling interval
    assert tm2d.checkpoint_steps(7, 2, 1) == 2
    assert tm2d.checkpoint_steps(5, 1, 50) == 50


def test_storage_modes():
    assert stg.StorageMode("checkpoint") is stg.StorageMode.CHECKPOINT
    assert stg.mode_code("cpu") == stg.STORAGE_CPU
    with pytest.raises(ValueError):
        stg.mode_code("tape")
    assert stg.resolve_mode("disk", device=torch.device("cpu"), n_store=1, n_shots=1, ny=4,
                            nx=4, itemsize=4, n_arrays=2, bytes_limit_device=None,
                            bytes_limit_host=None) == stg.STORAGE_DISK
    # auto: device when the history fits the device budget, else pinned host
    kw = dict(device=torch.device("cpu"), n_store=10, n_shots=2, ny=8, nx=8, itemsize=4, n_arrays=2)
    total = stg.history_bytes(10, 2, 8, 8, 4, 2)
    assert stg.resolve_mode("auto", bytes_limit_device=total, bytes_limit_host=None, **kw) == stg.STORAGE_DEVICE
    assert stg.resolve_mode("auto", bytes_limit_device=total - 1, bytes_limit_host=None, **kw) == stg.STORAGE_CPU
    with pytest.raises(MemoryError, match="checkpoint"):
        stg.resolve_mode("auto", bytes_limit_device=0, bytes_limit_host=0, **kw)


def test_history_pool_reuses_released_device_history():
    """A released device history is handed to the next request of the same
    shape (both snapshot kinds); another shape releases it."""
    import gc

    from tide_b200 import storage as stg

    stg.release_history_pool()
    dev = torch.device("cpu")  # the pool logic is device-agnostic
    a = stg.allocate(stg.STORAGE_DEVICE, torch.float32, 0, 3, 2, 4, 5, dev, True, True)
    ptrs = {a.ey_dev.data_ptr(), a.curl_dev.data_ptr()}
    del a
    gc.collect()
    b = stg.allocate(stg.STORAGE_DEVICE, torch.float32, 0, 3, 2, 4, 5, dev, True, True)
    assert {b.ey_dev.data_ptr(), b.curl_dev.data_ptr()} == ptrs
    c = stg.allocate(stg.STORAGE_DEVICE, torch.float32, 0, 4, 2, 4, 5, dev, True, False)
    assert c.ey_dev.data_ptr() not in ptrs
    del b, c
    gc.collect()
    stg.release_history_pool()


def test_disk_files_per_kind(tmp_path):
    """One temporary file per wanted snapshot kind (the 2-D pair or the six
    3-D components), a char** array per file for the native calls, and the
    files removed with the history."""
    import ctypes
    import gc

    from tide_b200 import storage as stg

    f = stg.DiskFiles(str(tmp_path), True, False, True, tags=("ex", "ey", "ez"))
    assert f.pointer(1) == 0 and f.pointer(0) != 0 and f.pointer(2) != 0
    names = sorted(p.name for p in tmp_path.iterdir())
    assert len(names) == 2 and names[0].startswith("tide_b200_ex_")
    first = ctypes.cast(f.pointer(0), ctypes.POINTER(ctypes.c_char_p))[0].decode()
    assert first == f.paths[0]
    two = stg.DiskFiles(str(tmp_path), True, True)  # the 2-D default kinds
    assert two.paths[0].split("/")[-1].startswith("tide_b200_ey_")
    del f, two
    gc.collect()
    assert list(tmp_path.iterdir()) == []
