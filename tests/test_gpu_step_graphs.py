"""Step blocks replayed from CUDA graphs give the results of per-step launches.

A TM2D call of at least three step blocks (64 steps, or the next multiple of
the even snapshot interval) captures one block into a graph and replays it,
the step-indexed pointers moving with a device-side block counter.  These
tests run the same calls with the graphs off and on and require bit-identical
receivers, snapshots, fields and gradients, plus the oracle on one case; the
step counts leave a tail after the last whole block so both the replayed
blocks and the tail are covered.
"""

from __future__ import annotations

import pytest
import torch

from cases import clone_problem, random_problem
from oracle_harness import set_grad_order
from tide_b200 import _native as nat
from tide_b200 import storage as stg
from tide_b200 import tm2d

pytestmark = pytest.mark.gpu


def _zeros_r(pb, device="cpu"):
    return torch.zeros((pb.nt, pb.n_shots, pb.n_rec), dtype=pb.dtype, device=device)


class _Graphs:
    """Sets the step-graph switch for a block and restores it afterwards."""

    def __init__(self, on: bool):
        self.on = on

    def __enter__(self):
        self.prev = nat.set_step_graphs(self.on)

    def __exit__(self, *exc):
        nat.set_step_graphs(self.prev)


def _forward(pb, dev, on):
    g = clone_problem(pb, dev)
    r = _zeros_r(g, dev)
    n0 = nat.graph_replays()
    with _Graphs(on):
        tm2d.native_forward(g, g.ca, g.cb, g.f, r, 0, g.nt)
        torch.cuda.synchronize()
    return [r] + [f.detach().clone() for f in g.fields], nat.graph_replays() - n0


def _gradients(pb, dev, grad_r, on, fmt=0, k=1):
    g = clone_problem(pb, dev)
    g.grad_interval = k
    S, ny, nx, nt = g.n_shots, g.ny, g.nx, g.nt
    sdt = torch.bfloat16 if fmt else g.dtype
    n_store = (nt + k - 1) // k
    snaps = stg.allocate(stg.STORAGE_DEVICE, sdt, fmt, n_store, S, ny, nx, dev, True, True)
    snaps.ey_dev.zero_()
    snaps.curl_dev.zero_()
    r = _zeros_r(g, dev)
    n0 = nat.graph_replays()
    with _Graphs(on):
        tm2d._run_forward_storage(g, g.ca, g.cb, g.f, r, snaps, True, True, None, 0)
        gca, gcb, gf = tm2d._run_backward(g, g.ca, g.cb, grad_r.to(dev), snaps, True, True,
                                          True, {})
        torch.cuda.synchronize()
    out = [r, snaps.ey_dev.clone(), snaps.curl_dev.clone(), gca, gcb, gf]
    return out, nat.graph_replays() - n0


def _same(a, b, names):
    for x, y, n in zip(a, b, names):
        assert torch.equal(x.detach().cpu(), y.detach().cpu()), f"{n}: graph replay differs"


@pytest.mark.parametrize("stencil", [2, 4])
@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_forward_graphs_bitwise(cuda_device, stencil, dtype):
    pb = random_problem(300 + stencil, 41, 57, 3, 229, stencil=stencil, dtype=dtype)
    eager, n_eager = _forward(pb, cuda_device, False)
    graph, n_graph = _forward(pb, cuda_device, True)
    assert n_eager == 0 and n_graph == 229 // 64 - 1  # blocks 1.. replayed, block 0 eager
    _same(eager, graph, ("r", "Ey", "Hx", "Hz", "mEyx", "mEyz", "mHxz", "mHzx"))


@pytest.mark.parametrize("fmt,k", [(0, 1), (1, 1), (0, 3), (1, 4)])
def test_storage_and_backward_graphs_bitwise(cuda_device, fmt, k):
    nt = 241
    pb = random_problem(77 + k, 39, 51, 2, nt)
    gen = torch.Generator().manual_seed(11)
    grad_r = torch.randn((nt, pb.n_shots, pb.n_rec), generator=gen)
    eager, n_eager = _gradients(pb, cuda_device, grad_r, False, fmt, k)
    graph, n_graph = _gradients(pb, cuda_device, grad_r, True, fmt, k)
    blk = {1: 64, 3: 66, 4: 64}[k]  # 64 rounded up to a multiple of lcm(2, k)
    assert n_eager == 0 and n_graph == 2 * (nt // blk - 1)
    _same(eager, graph, ("r", "Ey snapshots", "curl snapshots", "grad_ca", "grad_cb", "grad_f"))


def test_backward_graphs_double_stencil8(cuda_device):
    nt = 200
    pb = random_problem(91, 40, 48, 2, nt, stencil=8, dtype=torch.float64)
    grad_r = torch.randn((nt, pb.n_shots, pb.n_rec), generator=torch.Generator().manual_seed(4),
                         dtype=torch.float64)
    eager, _ = _gradients(pb, cuda_device, grad_r, False)
    graph, n_graph = _gradients(pb, cuda_device, grad_r, True)
    assert n_graph == 2 * (nt // 64 - 1)
    _same(eager, graph, ("r", "Ey snapshots", "curl snapshots", "grad_ca", "grad_cb", "grad_f"))


def test_graphs_vs_oracle(oracle, cuda_device):
    """The replayed blocks against the CPU oracle (step-major gradient order)."""
    nt = 200
    pb = random_problem(93, 33, 45, 2, nt)
    grad_r = torch.randn((nt, pb.n_shots, pb.n_rec), generator=torch.Generator().manual_seed(6))
    graph, n_graph = _gradients(pb, cuda_device, grad_r, True)
    assert n_graph > 0
    qb = clone_problem(pb)
    store = (torch.zeros((nt, 2, pb.ny, pb.nx)), torch.zeros((nt, 2, pb.ny, pb.nx)))
    r_o = _zeros_r(qb)
    oracle.forward(qb, qb.ca, qb.cb, qb.f, r_o, store=store, need_ca=True, need_cb=True)
    set_grad_order(oracle, 1)
    try:
        oca, ocb, ogf, _ = oracle.backward(qb, qb.ca, qb.cb, grad_r, store)
    finally:
        set_grad_order(oracle, 0)
    r, ey_s, cu_s, gca, gcb, gf = graph
    _same([r, ey_s, cu_s, gca[0], gcb[0], gf.reshape(ogf.shape)],
          [r_o, store[0], store[1], oca, ocb, ogf],
          ("r", "Ey snapshots", "curl snapshots", "grad_ca", "grad_cb", "grad_f"))


def _read_profile(lib):
    import ctypes

    ms = (ctypes.c_double * 16)()
    n = (ctypes.c_int64 * 16)()
    lib.tide_b200_profile_read.restype = ctypes.c_int
    k = lib.tide_b200_profile_read(ms, n, 16)
    lib.tide_b200_profile_kind_name.restype = ctypes.c_char_p
    return {lib.tide_b200_profile_kind_name(i).decode(): (ms[i], n[i]) for i in range(k)}


def test_profiled_blocks_replay_a_timed_graph(cuda_device):
    """Blocks holding a profiled step replay a second graph whose event-record
    nodes time the kernels of its first step; results are unchanged."""
    nt = 260
    pb = random_problem(95, 36, 44, 2, nt)
    lib = nat.load()
    base, _ = _forward(pb, cuda_device, True)
    lib.tide_b200_profile_enable(1, 128)
    _read_profile(lib)
    try:
        prof, n_graph = _forward(pb, cuda_device, True)
    finally:
        lib.tide_b200_profile_enable(0, 1)
    times = _read_profile(lib)
    # blocks 1..3 of 64 steps replay (block 2, steps 128.., through the timed
    # graph); the profiled steps 0 (block 0) and 256 (tail) run as ordinary
    # launches and are not timed on this path
    assert n_graph == 3
    for kind in ("fwd_h", "fwd_e"):
        ms, n = times[kind]
        assert n == 1 and ms > 0, (kind, times[kind])
    # a call too short for graphs times its profiled steps as launches
    short = random_problem(96, 36, 44, 2, 150)
    lib.tide_b200_profile_enable(1, 128)
    try:
        _, n_short = _forward(short, cuda_device, True)
    finally:
        lib.tide_b200_profile_enable(0, 1)
    times = _read_profile(lib)
    assert n_short == 0 and times["fwd_h"][1] == 2 and times["fwd_e"][1] == 2
    _same(base, prof, ("r", "Ey", "Hx", "Hz", "mEyx", "mEyz", "mHxz", "mHzx"))


# ---------------------------------------------------------------- Born passes


def _born_case(dev, nt=230, dtype=torch.float64, seed=21):
    import tide_b200 as tide

    g = torch.Generator().manual_seed(seed)
    ny, nx, S = 32, 46, 2
    eps = (2.0 + 4.0 * torch.rand((ny, nx), generator=g, dtype=torch.float64)).to(dtype).to(dev)
    sig = (0.005 * torch.rand((ny, nx), generator=g, dtype=torch.float64)).to(dtype).to(dev)
    dx = 0.02
    dt = 0.9 * dx / (tide.C0 / float(eps.min().sqrt()) * 2 ** 0.5)
    return dict(
        eps=eps, sig=sig, mu=torch.ones((ny, nx), device=dev, dtype=dtype), dx=dx, dt=dt,
        amp=tide.ricker(500e6, nt, dt, dtype=dtype).view(1, 1, nt).repeat(S, 1, 1).to(dev),
        src=torch.tensor([[[10, 12]], [[15, 30]]], device=dev),
        rec=torch.tensor([[[5, 5 + 3 * j] for j in range(10)]] * S, device=dev),
        deps=(0.3 * torch.randn((ny, nx), generator=g, dtype=torch.float64)).to(dtype).to(dev),
        dsig=(1e-3 * torch.randn((ny, nx), generator=g, dtype=torch.float64)).to(dtype).to(dev),
        w=torch.randn((nt, S, 10), generator=g, dtype=torch.float64).to(dtype).to(dev))


def _borntm(c, deps, dsig, eps=None, sig=None):
    import tide_b200 as tide

    return tide.borntm(c["eps"] if eps is None else eps, c["sig"] if sig is None else sig,
                       c["mu"], c["dx"], c["dt"], c["amp"], c["src"], c["rec"], c["rec"],
                       depsilon=deps, dsigma=dsig, stencil=2, pml_width=8)


def _with_graphs(on, fn):
    n0 = nat.graph_replays()
    with _Graphs(on):
        out = fn()
        torch.cuda.synchronize()
    return out, nat.graph_replays() - n0


def test_born_forward_graphs_bitwise(cuda_device):
    c = _born_case(cuda_device)

    def run():
        with torch.no_grad():
            return [t.clone() for t in _borntm(c, c["deps"], c["dsig"]) if t.numel()]

    eager, n_eager = _with_graphs(False, run)
    graph, n_graph = _with_graphs(True, run)
    assert n_eager == 0 and n_graph == 230 // 64 - 1
    _same(eager, graph, [f"born output {i}" for i in range(len(eager))])


def test_born_storage_and_second_order_graphs_bitwise(cuda_device):
    """Born forward with background and scattered histories (graph replay)
    feeding the second-order adjoint: gradients in eps, sigma, deps, dsigma."""
    c = _born_case(cuda_device)

    def run():
        leaves = [t.clone().requires_grad_() for t in (c["eps"], c["sig"], c["deps"], c["dsig"])]
        r = _borntm(c, leaves[2], leaves[3], eps=leaves[0], sig=leaves[1])[-1]
        (r * c["w"]).sum().backward()
        return [r.detach()] + [t.grad for t in leaves]

    eager, _ = _with_graphs(False, run)
    graph, n_graph = _with_graphs(True, run)
    assert n_graph >= 230 // 64 - 1  # the storing forward replays; adjoints as their paths allow
    _same(eager, graph, ("r", "grad eps", "grad sigma", "grad deps", "grad dsigma"))


def test_tangent_from_history_graphs_bitwise(cuda_device):
    """MaxwellTM.linearize(...).jvp from the kept device history
    (born_tangent_forward_with_storage) with and without graph replay."""
    import tide_b200 as tide

    c = _born_case(cuda_device)
    op = tide.MaxwellTM(tide.Discretization(c["dx"], c["dt"], stencil=2, boundary=tide.CPML(8)),
                        tide.Experiment(tide.Acquisition(c["src"], c["rec"]), c["amp"]))
    v = tide.EMDirection(c["deps"], c["dsig"])

    def run():
        lin = op.linearize(tide.EMModel(c["eps"], c["sig"], c["mu"]))
        out = lin._jvp_from_history(v)
        assert out is not None
        return [out.receiver_data.clone(), out.final_state.Ey.clone()]

    eager, _ = _with_graphs(False, run)
    graph, n_graph = _with_graphs(True, run)
    assert n_graph >= 2 * (230 // 64 - 1)  # primal storing forward + tangent pass
    _same(eager, graph, ("jvp receivers", "jvp final Ey"))
