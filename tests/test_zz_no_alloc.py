"""The adjoint entry point without caller scratch (jxb_sim_backward_noalloc).

It serves callers that cannot allocate device memory while they simulate (buffers
that come from a host-owned pool, or a plugin whose framework allocator must not be
re-entered from inside a step): its trajectory scratch is a fixed array inside the
library. This test calls it through the C ABI and checks it against
jxb_sim_backward on the same inputs, twice in a row (the array keeps the previous
call's contents, which must not leak into the next result). Tolerance: identical
state adjoints (the same kernel on the same data); parameter gradients to 1e-12
relative, because the float64 column sums are accumulated with atomics whose order
varies between launches. Float64 and float32.
"""
import ctypes as C

import pytest
import torch

from conftest import load_fixture
from jaxley_pytorch_b200 import _lib
from jaxley_pytorch_b200.sim import Simulation

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
        a = m.args(ckpt[seg], min(K, T - t0), t0, None, traj=traj, adj=adj,
                   rec_grad=rec_grad, pgrad=pgrad)
        (group,) = m.groups["backward"]  # every block of the fixture fits shared memory
        a = m.group_args(a, "backward", group)
        a.ckpt = ckpt[seg].data_ptr()
        a.traj_piv = piv.data_ptr() if piv is not None else None
        _lib.check(fn(C.byref(a), C.c_void_p(stream)), fn.__name__)
    torch.cuda.synchronize()
    return adj, pgrad


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_noalloc_adjoint_matches_scratch_adjoint(cuda_device, dtype):
    prob, extra = load_fixture("l5pc_7x4_batch3")
    T = 120
    prob.n_steps = T
    sim = Simulation(prob, dtype=dtype, device=cuda_device, checkpoint=40)
    low = sim.low
    K = sim.checkpoint
    ckpt = torch.empty(((T + K - 1) // K, low.batch, low.n_slots), dtype=dtype, device=cuda_device)
    rec, _ = sim.forward_raw(sim.model.pscale, T, ckpt=ckpt)
    g = torch.Generator(device="cpu").manual_seed(0)
    rec_grad = torch.randn(rec.shape, generator=g, dtype=torch.float64).to(cuda_device, dtype)
    ref_adj, ref_pg = _adjoint(sim, ckpt, rec_grad, T, noalloc=False)
    for _ in range(2):
        adj, pg = _adjoint(sim, ckpt, rec_grad, T, noalloc=True)
        assert torch.equal(adj, ref_adj)
        assert (pg - ref_pg).abs().max().item() <= 1e-12 * ref_pg.abs().max().item()
    assert ref_pg.abs().max() > 0


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
