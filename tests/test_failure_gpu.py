"""Failure detection without a GPU fault: a NaN injected on the host into one
parameter of a run makes the kernels flag the non-finite result on the device
(JxbSimArgs.status), and the host raises `FloatingPointError` (the reference's
trainer raises it for a non-finite loss, training/engine.py:229-230). The kernels keep
running to the end of the launch; afterwards the same model and context give finite
results again."""
import math

import numpy as np
import pytest
import torch

from conftest import load_fixture
from jaxley_pytorch_b200.network import NetworkSimulation
from jaxley_pytorch_b200.sim import Simulation

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("segment", [None, 1])
def test_nan_parameter_raises_and_context_stays_usable(cuda_device, segment):
    prob, extra = load_fixture("l5pc_7x4_batch3")
    sim = Simulation(prob, dtype=torch.float32, device=cuda_device, segment=segment)
    ps = sim.model.pscale.clone()
    col = int(np.nonzero(np.asarray(sim.low.pcol) > 0)[0][0])  # a column that some parameter reads
    ps[1, int(sim.low.pcol[col])] = math.nan  # one row's scale of one parameter
    with pytest.raises(FloatingPointError):
        sim.run(pscale=ps)
    clean = sim.run()
    assert torch.isfinite(clean).all()


def test_nan_gradient_raises_in_the_adjoint(cuda_device):
    prob, extra = load_fixture("hh_tree_15x3")
    sim = Simulation(prob, dtype=torch.float64, device=cuda_device, checkpoint=50)
    ps = sim.model.pscale.clone().requires_grad_(True)
    rec = sim.run(pscale=ps)
    w = torch.ones_like(rec)
    w[0, 0, 5] = math.nan  # a non-finite loss weight, as from a non-finite loss
    with pytest.raises(FloatingPointError):
        (rec * w).sum().backward()
    ps2 = sim.model.pscale.clone().requires_grad_(True)
    sim.run(pscale=ps2).sum().backward()
    assert torch.isfinite(ps2.grad).all()


def test_nan_synapse_weight_raises_in_a_network(cuda_device):
    prob, extra = load_fixture("synapse_net_8")
    net = NetworkSimulation(prob, dtype=torch.float32, device=cuda_device)
    params = [[p.clone() for p in ty.params] for ty in net.types]
    params[0][0][3] = math.nan
    with pytest.raises(FloatingPointError):
        net.run(net.model.pscale, params)
    assert torch.isfinite(net.run()).all()


def test_flag_is_not_read_while_capturing(cuda_device):
    """Inside a CUDA-graph capture the check is skipped (reading the flag would
    synchronise); the flag stays set for the next check outside the capture."""
    prob, extra = load_fixture("hh_tree_15x3")
    sim = Simulation(prob, dtype=torch.float32, device=cuda_device)
    sim.model.status.fill_(1)
    x = torch.zeros(4, device=cuda_device)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        x.add_(1.0)
        sim.model.check_finite("capture")  # no raise, no read
    g.replay()
    torch.cuda.synchronize()
    with pytest.raises(FloatingPointError):
        sim.model.check_finite("after the capture")
    sim.model.check_finite("cleared")
