"""Parity of the fused CUDA simulation against the reference (fixtures) and the
oracle. FP64 runs must agree to <= 1e-9 relative; FP32 runs to <= 1e-3 mV over
non-chaotic stretches (here: the whole trace of the small fixtures, tolerance
stated per test)."""
import numpy as np
import pytest
import torch

import oracle
from conftest import fixture_names, load_fixture
from jaxley_pytorch_b200.sim import Simulation

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", fixture_names())
@pytest.mark.parametrize("segment", [1, None])
def test_fp64_matches_reference(cuda_device, name, segment):
    prob, extra = load_fixture(name)
    if prob.synapses:
        pytest.skip("synapse problems run through the network path")
    steady = bool(extra.get("init_steady", 0))
    sim = Simulation(prob, dtype=torch.float64, device=cuda_device, segment=segment, init_steady=steady)
    out = sim.run().cpu().numpy()
    ref = extra["ref"].reshape(out.shape)
    scale = max(1.0, np.abs(ref).max())
    err = np.abs(out - ref).max() / scale
    assert err <= 1e-9, err


@pytest.mark.parametrize("name", ["cell_8comp_hh", "hh_tree_15x3", "l5pc_7x4_batch3", "hh_forest_6"])
def test_fp32_close_to_fp64_oracle(cuda_device, name):
    prob, extra = load_fixture(name)
    sim = Simulation(prob, dtype=torch.float32, device=cuda_device)
    out = sim.run().cpu().numpy().astype(np.float64)
    ref = extra["ref"].reshape(out.shape)
    # Voltage recordings only; tolerance in mV.
    vcols = [c for c, (nm, _) in enumerate(prob.recordings) if nm == "v"]
    err = np.abs(out[:, vcols] - ref[:, vcols]).max()
    assert err <= 5e-2, err


@pytest.mark.parametrize("rows", [1, 2, 3])
@pytest.mark.parametrize("max_block", [16, 4096])
def test_blocking_and_rows_do_not_change_results(cuda_device, rows, max_block):
    prob, extra = load_fixture("l5pc_7x4_batch3")
    a = Simulation(prob, dtype=torch.float64, device=cuda_device).run()
    b = Simulation(prob, dtype=torch.float64, device=cuda_device, rows_per_item=rows,
                   max_block_nodes=max_block, segment=7).run()
    assert torch.equal(a, b) or (a - b).abs().max().item() <= 1e-12
