"""Blocks routed to the global-scratch kernels (working set over the shared-memory
limit) compute the same forward and adjoint as the shared-memory kernels: the
arithmetic is identical, only where the work areas live differs. Recordings must be
identical; parameter gradients agree to 1e-12 relative (float64 column sums are
accumulated with atomics whose order varies)."""
import numpy as np
import pytest
import torch

from jaxley_pytorch_b200 import synth
from jaxley_pytorch_b200.lower import lower
from jaxley_pytorch_b200.sim import Simulation

pytestmark = pytest.mark.gpu


def _grad_run(sim, T):
    ps = sim.model.pscale.clone().requires_grad_(True)
    rec = sim.run(n_steps=T, pscale=ps)
    loss = ((rec - rec.detach().mean()) ** 2).mean()
    (g,) = torch.autograd.grad(loss, ps)
    return rec.detach(), g


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("mode", ["all", "mixed"])
def test_global_scratch_matches_shared_memory(cuda_device, dtype, mode):
    prob = synth.config_uneven(n_cells=24, n_steps=60, max_comp=300, seed=5)
    low = lower(prob, max_block_nodes=128, keep_currents=False)
    ref = Simulation(prob, low=low, dtype=dtype, device=cuda_device, checkpoint=25, segment=30)
    if mode == "all":
        limit = 1
    else:  # the larger half of the blocks goes to global scratch
        m = ref.model
        need = [m._layout_bytes(m._block_maxima(np.asarray([b])), True) for b in range(len(low.blocks))]
        limit = int(np.median(need))
    gm = Simulation(prob, low=low, dtype=dtype, device=cuda_device, checkpoint=25, segment=30)
    gm.model.smem_limit = limit
    gm.model.set_rows_per_item(1)
    kinds = {g["gm"] for g in gm.model.groups["backward"]}
    assert (kinds == {True}) if mode == "all" else (kinds == {True, False})
    r0, g0 = _grad_run(ref, 60)
    r1, g1 = _grad_run(gm, 60)
    torch.cuda.synchronize()
    assert torch.equal(r0, r1)
    scale = g0.abs().max().item()
    assert scale > 0
    assert (g0 - g1).abs().max().item() <= 1e-12 * scale


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("threads", [64, 256])
def test_node_schedule_does_not_change_results(cuda_device, dtype, threads):
    """The per-warp node schedule only reorders which thread handles which node."""
    prob = synth.config_uneven(n_cells=16, n_steps=60, max_comp=400, seed=9)
    low = lower(prob, max_block_nodes=512, keep_currents=False)
    kw = dict(low=low, dtype=dtype, device=cuda_device, checkpoint=25, threads=threads)
    a = Simulation(prob, schedule=False, **kw)
    b = Simulation(prob, schedule=True, **kw)
    assert b.model.sched_warps == threads // 32 and a.model.sched_warps == 0
    r0, g0 = _grad_run(a, 60)
    r1, g1 = _grad_run(b, 60)
    torch.cuda.synchronize()
    assert torch.equal(r0, r1)
    assert (g0 - g1).abs().max().item() <= 1e-12 * g0.abs().max().item()


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
@pytest.mark.parametrize("gm", [False, True])
def test_stored_trajectory_equals_recompute(cuda_device, dtype, gm):
    """The adjoint over the trajectory the forward stored and the adjoint that
    recomputes every segment from its checkpoint see the same states and pivots:
    identical recordings, gradients equal up to the order of the float64 atomics.
    70 steps in segments of 25 (two full, one ragged); shared-memory and
    global-scratch kernels."""
    prob = synth.config_uneven(n_cells=24, n_steps=70, max_comp=300, seed=5)
    low = lower(prob, max_block_nodes=128, keep_currents=False)
    out = []
    for store in (True, False):
        sim = Simulation(prob, low=low, dtype=dtype, device=cuda_device, checkpoint=25,
                         store_trajectory=store)
        if gm:
            sim.model.smem_limit = 1
            sim.model.set_rows_per_item(1)
        assert sim.stores_trajectory(70) == store
        out.append(_grad_run(sim, 70))
    torch.cuda.synchronize()
    (r0, g0), (r1, g1) = out
    assert torch.equal(r0, r1)
    scale = g0.abs().max().item()
    assert scale > 0
    assert (g0 - g1).abs().max().item() <= 1e-12 * scale


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_forward_launch_shape_does_not_change_results(cuda_device, dtype):
    """Forward launches of another CTA size (own node schedule) and the wide register
    budget run the same per-node arithmetic: identical recordings, and gradients
    equal up to the order of the float64 atomics."""
    prob = synth.config_uneven(n_cells=24, n_steps=60, max_comp=300, seed=5)
    low = lower(prob, max_block_nodes=256, keep_currents=False)
    kw = dict(low=low, dtype=dtype, device=cuda_device, checkpoint=25, threads=512)
    a = Simulation(prob, **kw)
    b = Simulation(prob, forward_threads=256, forward_wide=True, **kw)
    assert b.model.kind_threads == {"forward": 256, "backward": 512}
    r0, g0 = _grad_run(a, 60)
    r1, g1 = _grad_run(b, 60)
    torch.cuda.synchronize()
    assert torch.equal(r0, r1)
    scale = g0.abs().max().item()
    assert (g0 - g1).abs().max().item() <= 1e-12 * scale


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_adjoint_cta_sizes_agree(cuda_device, dtype):
    """The adjoint at 384 threads (float: the kernels bounded for two 12-warp CTAs per
    SM with up to 80 registers) gives the 512-thread launch's gradients: the CTA size
    only changes which thread handles which node."""
    prob = synth.config_uneven(n_cells=16, n_steps=60, max_comp=400, seed=9)
    low = lower(prob, max_block_nodes=512, keep_currents=False)
    runs = []
    for th in (512, 384):
        sim = Simulation(prob, low=low, dtype=dtype, device=cuda_device, checkpoint=25, threads=th,
                         forward_threads=256)
        assert sim.model.kind_threads["backward"] == th
        runs.append(_grad_run(sim, 60))
    torch.cuda.synchronize()
    (r0, g0), (r1, g1) = runs
    assert torch.equal(r0, r1)
    assert (g0 - g1).abs().max().item() <= 1e-12 * g0.abs().max().item()
