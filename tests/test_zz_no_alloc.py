"""The adjoint entry point without caller scratch (jxb_sim_backward_noalloc).

It serves callers that cannot allocate device memory while they simulate (buffers
that come from a host-owned pool, or a plugin whose framework allocator must not be
re-entered from inside a step): its trajectory scratch is a fixed array inside the
library. This test calls it through the C ABI and checks it against
jxb_sim_backward on the same inputs, twice in a row (the array keeps the previous
call's contents, which must not leak into the next result). Tolerance: identical
state adjoints (the same kernel on the same data); parameter gradients to 1e-12
relative, because the float64 column sums are accumulated with atomics whose order
varies between launches. Float64 and float32; blocks whose work areas live in the
caller's global scratch (the kernel then reads the trajectory straight from the fixed
array); and a segment just under the array's size, next to one just over it.
"""
import ctypes as C

import pytest
import torch

from conftest import load_fixture
from jaxley_pytorch_b200 import _lib, synth
from jaxley_pytorch_b200.lower import lower
from jaxley_pytorch_b200.sim import Simulation

ARRAY_BYTES = 32 << 20  # size of the library's fixed array


def _need_bytes(low, K, item):
    """Scratch bytes of a K-step segment: states, then pivots at a 256-byte boundary."""
    traj = K * low.batch * low.n_slots * item
    return (traj + 255) // 256 * 256 + K * low.batch * low.n_nodes * item

pytestmark = pytest.mark.gpu


def _adjoint(sim, ckpt, rec_grad, T, noalloc):
    m, low, K = sim.model, sim.low, sim.checkpoint
    adj = torch.zeros((low.batch, low.n_slots), dtype=m.dtype, device=m.device)
    pgrad = torch.zeros((low.batch, low.n_cols), dtype=torch.float64, device=m.device)
    traj = piv = None
    if not noalloc:
        traj = torch.empty((K, low.batch, low.n_slots), dtype=m.dtype, device=m.device)
        piv = torch.empty((K, low.batch, low.n_nodes), dtype=m.dtype, device=m.device)
    lib = _lib.load()
    fn = lib.jxb_sim_backward_noalloc if noalloc else lib.jxb_sim_backward
    stream = torch.cuda.current_stream(m.device).cuda_stream
    for seg in range((T + K - 1) // K - 1, -1, -1):
        t0 = seg * K
        base = m.args(ckpt[seg], min(K, T - t0), t0, None, traj=traj, adj=adj,
                      rec_grad=rec_grad, pgrad=pgrad)
        for group in m.groups["backward"]:  # in turn on one stream: they never overlap
            a = m.group_args(base, "backward", group)
            a.ckpt = ckpt[seg].data_ptr()
            a.traj_piv = piv.data_ptr() if piv is not None else None
            _lib.check(fn(C.byref(a), C.c_void_p(stream)), fn.__name__)
    torch.cuda.synchronize()
    return adj, pgrad


def _compare(sim, T, dtype, device):
    """Forward with a checkpoint per segment, then the adjoint through both entry
    points: the no-allocation one twice in a row."""
    low = sim.low
    K = sim.checkpoint
    ckpt = torch.empty(((T + K - 1) // K, low.batch, low.n_slots), dtype=dtype, device=device)
    rec, _ = sim.forward_raw(sim.model.pscale, T, ckpt=ckpt)
    g = torch.Generator(device="cpu").manual_seed(0)
    rec_grad = torch.randn(rec.shape, generator=g, dtype=torch.float64).to(device, dtype)
    ref_adj, ref_pg = _adjoint(sim, ckpt, rec_grad, T, noalloc=False)
    for _ in range(2):
        adj, pg = _adjoint(sim, ckpt, rec_grad, T, noalloc=True)
        assert torch.equal(adj, ref_adj)
        assert (pg - ref_pg).abs().max().item() <= 1e-12 * ref_pg.abs().max().item()
    assert ref_pg.abs().max() > 0


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_noalloc_adjoint_matches_scratch_adjoint(cuda_device, dtype):
    prob, extra = load_fixture("l5pc_7x4_batch3")
    T = 120
    prob.n_steps = T
    sim = Simulation(prob, dtype=dtype, device=cuda_device, checkpoint=40)
    _compare(sim, T, dtype, cuda_device)


def test_noalloc_adjoint_with_global_work_areas(cuda_device):
    prob = synth.config_uneven(n_cells=12, n_steps=60, max_comp=300, seed=5)
    low = lower(prob, max_block_nodes=128, keep_currents=False)
    sim = Simulation(prob, low=low, dtype=torch.float64, device=cuda_device, checkpoint=25, segment=30)
    sim.model.smem_limit = 1  # every block keeps its work areas in global scratch
    sim.model.set_rows_per_item(1)
    assert {g["gm"] for g in sim.model.groups["backward"]} == {True}
    assert _need_bytes(low, 25, 8) <= ARRAY_BYTES
    _compare(sim, 60, torch.float64, cuda_device)


def test_noalloc_segment_at_the_size_limit(cuda_device):
    prob, extra = load_fixture("l5pc_7x4_batch3")
    probe = Simulation(prob, dtype=torch.float64, device=cuda_device)
    low = probe.low
    K = 1
    while _need_bytes(low, K + 1, 8) <= ARRAY_BYTES:
        K += 1
    assert _need_bytes(low, K, 8) > ARRAY_BYTES - 2 * low.batch * (low.n_slots + low.n_nodes) * 8
    prob.n_steps = K
    sim = Simulation(prob, dtype=torch.float64, device=cuda_device, checkpoint=K)
    _compare(sim, K, torch.float64, cuda_device)
    # one step more no longer fits: refused on the host before any launch
    m = sim.model
    state = m.initial_state()
    adj = torch.zeros_like(state)
    pgrad = torch.zeros((low.batch, low.n_cols), dtype=torch.float64, device=cuda_device)
    a = m.group_args(m.args(state, K + 1, 0, None, adj=adj, pgrad=pgrad), "backward",
                     m.groups["backward"][0])
    a.ckpt = state.data_ptr()
    rc = _lib.load().jxb_sim_backward_noalloc(C.byref(a), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 5  # JXB_ERR_TOO_LARGE


def test_noalloc_rejects_oversized_segments(cuda_device):
    prob, extra = load_fixture("l5pc_7x4_batch3")
    sim = Simulation(prob, dtype=torch.float64, device=cuda_device, checkpoint=40)
    low = sim.low
    m = sim.model
    state = m.initial_state()
    adj = torch.zeros_like(state)
    pgrad = torch.zeros((low.batch, low.n_cols), dtype=torch.float64, device=cuda_device)
    a = m.group_args(m.args(state, 10**6, 0, None, adj=adj, pgrad=pgrad), "backward",
                     m.groups["backward"][0])
    a.ckpt = state.data_ptr()
    rc = _lib.load().jxb_sim_backward_noalloc(C.byref(a), C.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 5  # JXB_ERR_TOO_LARGE
    assert b"fixed array" in _lib.load().jxb_last_error()
