"""A captured training iteration replays the eager one; the autotuner picks a
candidate that runs and whose results equal the default launch's."""
import pytest
import torch

from conftest import load_fixture
from jaxley_pytorch_b200 import synth
from jaxley_pytorch_b200.graphs import GraphedIteration
from jaxley_pytorch_b200.sim import Simulation
from jaxley_pytorch_b200.tune import autotune

pytestmark = pytest.mark.gpu


def _problem():
    return synth.config_uneven(n_cells=12, n_steps=80, max_comp=200, seed=7)


@pytest.mark.parametrize("dtype", [torch.float64, torch.float32])
def test_graphed_gradient_matches_eager(cuda_device, dtype):
    prob = _problem()
    sim = Simulation(prob, dtype=dtype, device=cuda_device, checkpoint=30, keep_currents=False)
    with torch.no_grad():
        target = sim.run(pscale=sim.model.pscale * 1.1).detach()

    def loss_fn(rec):
        return ((rec - target) ** 2).mean()

    ps = sim.model.pscale.clone().requires_grad_(True)
    loss_e = loss_fn(sim.run(pscale=ps))
    (g_e,) = torch.autograd.grad(loss_e, ps)
    it = GraphedIteration(sim, loss_fn, sim.model.pscale.clone().requires_grad_(True))
    assert it.launches_per_replay >= 2
    tol = 1e-12 if dtype == torch.float64 else 1e-6
    for _ in range(2):
        loss, g = it.replay()
        torch.cuda.synchronize()
        assert abs(loss.item() - loss_e.item()) <= tol * abs(loss_e.item())
        assert (g - g_e).abs().max().item() <= tol * g_e.abs().max().item()


def test_graphed_adam_step_matches_eager(cuda_device):
    prob = _problem()
    sim = Simulation(prob, dtype=torch.float64, device=cuda_device, checkpoint=40, keep_currents=False)
    with torch.no_grad():
        target = sim.run(pscale=sim.model.pscale * 1.1).detach()

    def loss_fn(rec):
        return ((rec - target) ** 2).mean()

    p_e = sim.model.pscale.clone().requires_grad_(True)
    # capturable=True in both: its step counter is a float32 device tensor, so its bias
    # corrections differ from the default Adam's at the 1e-5 level.
    opt_e = torch.optim.Adam([p_e], lr=1e-3, capturable=True)
    for _ in range(5):  # eager: 2 warm-up steps + 3 replays of the captured one
        opt_e.zero_grad()
        (g,) = torch.autograd.grad(loss_fn(sim.run(pscale=p_e)), p_e)
        p_e.grad = g
        opt_e.step()
    p_g = sim.model.pscale.clone().requires_grad_(True)
    opt_g = torch.optim.Adam([p_g], lr=1e-3, capturable=True)
    it = GraphedIteration(sim, loss_fn, p_g, optimizer=opt_g, warmup=2)
    for _ in range(3):
        it.replay()
    torch.cuda.synchronize()
    assert (p_g.detach() - p_e.detach()).abs().max().item() <= 1e-12


def test_autotune_picks_a_running_candidate(cuda_device):
    prob = _problem()
    choice, low, table = autotune(prob, dtype=torch.float64, device=cuda_device, probe_steps=20,
                                  block_nodes=(64, 512), threads=(128, 256), rows=(1,),
                                  checkpoints=(20, 40), horizon=80)
    ran = [r for r in table if "ms_per_step" in r and "threads" in r]
    assert ran and choice.max_block_nodes in (64, 512) and choice.threads in (128, 256)
    assert choice.checkpoint in (20, 40)
    assert choice.ms_per_step == min(r["ms_per_step"] for r in table if "checkpoint" in r)
    a = Simulation(prob, dtype=torch.float64, device=cuda_device).run()
    b = Simulation(prob, low=low, dtype=torch.float64, device=cuda_device, threads=choice.threads,
                   rows_per_item=choice.rows_per_item, checkpoint=choice.checkpoint).run()
    assert (a - b).abs().max().item() <= 1e-12 * max(1.0, a.abs().max().item())
