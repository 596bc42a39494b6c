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
