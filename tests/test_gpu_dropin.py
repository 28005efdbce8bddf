"""The literal drop-in: the unmodified reference package running on CUDA
tensors with its native handle pointed at libtide_b200.so.

The reference's loader keeps the native library in
``tide.backend_utils._runtime.dll`` (src/tide/backend_utils.py:64-99) and
resolves every entry point there by name with its own argtypes
(:823-877); pointing that handle at this library is the whole integration.
The reference's own operator, ``tide.MaxwellTM``, then runs its CUDA code
path (src/tide/maxwell/tm2d_autograd.py: zero-initialised adjoint state,
adjoint_memory_scratch layout, per-shot gradient buffers) against these
kernels.  Receivers and eps / sigma gradients of the heterogeneous golden
case must match the reference's exact autograd gradients
(tests/golden/hetero_grad.npz, made by running the reference): relative L2
<= 1e-10 in FP64 and <= 1e-5 in FP32.

The reference package comes from `python -m pip install --no-index
--no-build-isolation --no-deps --find-links /opt/wheelhouse --target
baseline/_ref <copy of the reference tree>` (--no-deps: the reference pins a
newer torch than the image's; its Python code runs on this one); without it
the test is skipped.  Its own native library, if the install built one, is
never loaded: the handle is set before the first call.
"""

from __future__ import annotations

import ctypes
import sys

import numpy as np
import pytest
import torch

from cases import hetero_inputs
from conftest import GOLDEN, REPO
from oracle_harness import rel_l2
from tide_b200 import _native as nat

pytestmark = pytest.mark.gpu
REF_PKG = REPO / "baseline" / "_ref"


@pytest.fixture(scope="module")
def ref_tide():
    if not (REF_PKG / "tide" / "__init__.py").is_file():
        pytest.skip("reference package not installed under baseline/_ref")
    sys.path.insert(0, str(REF_PKG))
    try:
        import tide
        from tide import backend_utils as bu
    finally:
        sys.path.remove(str(REF_PKG))
    bu._runtime.dll = ctypes.CDLL(str(nat.library_path()))
    bu._runtime.lib_path = nat.library_path()
    bu._runtime.probed = True
    bu._runtime.use_openmp = False
    assert bu.is_backend_available()
    return tide


def _run(tide, stencil, dtype, dev):
    c = hetero_inputs(dtype)
    eps = c["eps"].to(dev).requires_grad_(True)
    sig = c["sig"].to(dev).requires_grad_(True)
    op = tide.MaxwellTM(
        tide.Discretization(tuple(c["dx"]), c["dt"], stencil=stencil,
                            boundary=tide.CPML(c["pml"])),
        tide.Experiment(tide.Acquisition(c["src"].to(dev), c["rec"].to(dev)),
                        c["amp"].to(dev)),
    )
    res = op(tide.EMModel(eps, sig, c["mu"].to(dev)))
    r = res.receiver_data
    (r * c["w"].to(dev)).sum().backward()
    torch.cuda.synchronize()
    return r.detach().cpu(), eps.grad.cpu(), sig.grad.cpu()


@pytest.mark.parametrize("stencil", [2, 4])
@pytest.mark.parametrize("dtype,tol", [(torch.float64, 1e-10), (torch.float32, 1e-5)])
def test_reference_operator_on_this_library(ref_tide, cuda_device, stencil, dtype, tol):
    z = np.load(GOLDEN / "hetero_grad.npz")
    lib = nat.load()
    launches0 = lib.tide_b200_launch_count()
    r, ge, gs = _run(ref_tide, stencil, dtype, cuda_device)
    lib.tide_b200_launch_count.restype = ctypes.c_int64
    assert lib.tide_b200_launch_count() > launches0  # the kernels ran here
    assert rel_l2(r, torch.from_numpy(z[f"r_f64_s{stencil}"])) <= tol
    assert rel_l2(ge, torch.from_numpy(z[f"geps_f64_s{stencil}"])) <= tol
    assert rel_l2(gs, torch.from_numpy(z[f"gsig_f64_s{stencil}"])) <= tol
    assert lib.tide_b200_last_status() == 0
