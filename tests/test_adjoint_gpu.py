"""The hand-written adjoint against central finite differences of the float64
oracle and against the reference's autograd gradient (fixtures). Tolerances:
float64 1e-6 relative against finite differences (the FD error dominates), float32
1e-3 relative against the float64 adjoint."""
import numpy as np
import pytest
import torch

import oracle
from conftest import load_fixture
from jaxley_pytorch_b200.sim import Simulation

pytestmark = pytest.mark.gpu


def _loss_weights(shape, seed=0):
    rng = np.random.default_rng(seed)
    return rng.normal(size=shape)


def _oracle_loss(prob, W, steady):
    out = oracle.integrate(prob, init_steady=steady)
    return float(np.sum(W * out))


def _fd_grad(prob, low, W, b, col, h, steady):
    base_params = {k: np.array(v, copy=True) for k, v in prob.params.items()}
    vals = []
    for sgn in (1, -1):
        for k in base_params:
            prob.params[k] = np.array(base_params[k], copy=True)
        for name, r, base in low.col_members[col]:
            arr = prob.params[name]
            if arr.ndim == 1:
                arr = np.broadcast_to(arr, (prob.batch, arr.shape[0])).copy()
            arr[b, r] += sgn * h * base
            prob.params[name] = arr
        vals.append(_oracle_loss(prob, W, steady))
    for k in base_params:
        prob.params[k] = base_params[k]
    return (vals[0] - vals[1]) / (2 * h)


@pytest.mark.parametrize("name,steps,ckpt", [("l5pc_7x4_batch3", 160, 50), ("synth_l5pc_15x4", 120, 40)])
def test_adjoint_matches_central_differences(cuda_device, name, steps, ckpt):
    """Against central differences of the float64 CUDA forward (h = 1e-4 on the column
    scale; tolerance 1e-6 of the largest gradient) and of the float64 oracle
    (h = 1e-3: the oracle's finite-difference current slope makes its loss noisy at
    the 1e-10 level, so its tolerance is 1e-3 of the largest gradient)."""
    prob, extra = load_fixture(name)
    steady = bool(extra.get("init_steady", 0))
    prob.n_steps = steps
    sim = Simulation(prob, dtype=torch.float64, device=cuda_device, checkpoint=ckpt, init_steady=steady)
    low = sim.low
    W = _loss_weights((prob.batch, low.n_rec, steps + 1))
    W[:, [c for c, (nm, _) in enumerate(prob.recordings) if nm != "v"]] = 0.0
    Wt = torch.as_tensor(W, device=cuda_device)
    pscale = sim.model.pscale.clone().requires_grad_(True)
    loss = (sim.run(pscale=pscale) * Wt).sum()
    loss.backward()
    g = pscale.grad.cpu().numpy()
    assert low.n_cols > 1
    gmax = np.abs(g[:, 1:]).max()
    h = 1e-4
    for col in range(1, low.n_cols):
        for b in range(prob.batch):
            vals = []
            for sgn in (1, -1):
                ps = sim.model.pscale.clone()
                ps[b, col] += sgn * h
                vals.append(float((sim.run(pscale=ps) * Wt).sum()))
            fd = (vals[0] - vals[1]) / (2 * h)
            assert abs(g[b, col] - fd) <= 1e-6 * gmax, (col, b, g[b, col], fd)
            fd_or = _fd_grad(prob, low, W, b, col, 1e-3, steady)
            assert abs(g[b, col] - fd_or) <= 1e-3 * gmax, (col, b, g[b, col], fd_or)


def test_adjoint_segments_and_plain_agree(cuda_device):
    prob, extra = load_fixture("l5pc_7x4_batch3")
    prob.n_steps = 200
    grads = []
    for ckpt, seg in [(200, None), (1, 1), (37, None), (50, 7)]:
        sim = Simulation(prob, dtype=torch.float64, device=cuda_device, checkpoint=ckpt, segment=seg)
        W = torch.as_tensor(_loss_weights((prob.batch, sim.low.n_rec, 201), 3), device=cuda_device)
        ps = sim.model.pscale.clone().requires_grad_(True)
        (sim.run(pscale=ps) * W).sum().backward()
        grads.append(ps.grad.clone())
    for g in grads[1:]:
        torch.testing.assert_close(g, grads[0], rtol=1e-10, atol=1e-12)


def _fp32_vs_fp64(prob, steps, seed=5):
    prob.n_steps = steps
    out = {}
    for dt in (torch.float64, torch.float32):
        sim = Simulation(prob, dtype=dt, device="cuda", checkpoint=50, init_steady=True)
        W = torch.as_tensor(_loss_weights((prob.batch, sim.low.n_rec, steps + 1), seed),
                            device="cuda", dtype=dt)
        ps = sim.model.pscale.clone().requires_grad_(True)
        v = sim.run(pscale=ps)
        (v * W).sum().backward()
        out[dt] = (v.detach().double(), ps.grad.double())
    (v64, g64), (v32, g32) = out[torch.float64], out[torch.float32]
    dv = (v32 - v64).abs().max().item()
    rel = ((g32 - g64).abs().max() / g64.abs().max()).item()
    return dv, rel, v64.max().item()


def test_fp32_subthreshold_within_stated_tolerance(cuda_device):
    """Non-chaotic (subthreshold) trace: max|dV| <= 1e-3 mV and gradient error
    <= 1e-3 relative, float32 against float64."""
    prob, extra = load_fixture("synth_l5pc_15x4")
    for k in ("somatic_NaTs2T_gNaTs2T", "apical_NaTs2T_gNaTs2T"):
        prob.params[k] = np.asarray(prob.params[k]) * 0.02
    prob.stim = prob.stim * 0.2
    dv, rel, vmax = _fp32_vs_fp64(prob, 400)
    assert vmax < -30.0  # no spike
    assert dv <= 1e-3, dv
    assert rel <= 1e-3, rel


def test_fp32_spiking_error_is_bounded(cuda_device):
    """Spiking trace: float32 spike times drift by rounding; stated bound 2 mV and 5e-2
    relative gradient error over 200 steps with two spikes."""
    prob, extra = load_fixture("synth_l5pc_15x4")
    dv, rel, vmax = _fp32_vs_fp64(prob, 200)
    assert vmax > 0.0
    assert dv <= 2.0, dv
    assert rel <= 5e-2, rel


@pytest.mark.parametrize("name", ["cell_8comp_hh", "hh_tree_15x3", "hh_forest_6", "synth_l5pc_15x4",
                                  "l5pc_7x4_batch3"])
def test_compile_time_programs_match_interpreter(cuda_device, name):
    """Node classes that run a compile-time channel program (csrc/jxb_prog.cuh) give
    the interpreter's results, forward and adjoint (float64)."""
    prob, extra = load_fixture(name)
    prob.n_steps = min(prob.n_steps, 150)
    steady = bool(extra.get("init_steady", 0))
    res = []
    for programs in (True, False):
        sim = Simulation(prob, dtype=torch.float64, device=cuda_device, checkpoint=40,
                         init_steady=steady, keep_currents=False, programs=programs)
        W = torch.as_tensor(_loss_weights((prob.batch, sim.low.n_rec, prob.n_steps + 1), 2),
                            device=cuda_device)
        ps = sim.model.pscale.clone().requires_grad_(True)
        out = sim.run(pscale=ps)
        (out * W).sum().backward()
        res.append((out.detach(), ps.grad))
        if programs and name != "l5pc_7x4_batch3":
            assert int(sim.low.cls_prog.max()) > 0  # the program path is exercised
    torch.testing.assert_close(res[0][0], res[1][0], rtol=1e-12, atol=1e-10)
    torch.testing.assert_close(res[0][1], res[1][1], rtol=1e-10, atol=1e-12)
