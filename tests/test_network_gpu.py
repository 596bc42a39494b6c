"""Networks: the synapse step fused into the simulation loop and its adjoint.
Forward parity: float64 within 1e-9 relative of the reference's run (fixture) and of
the oracle (synthetic network). Gradients: central differences of the float64 CUDA
forward, within 1e-6 of the largest gradient. float32: within 2e-3 mV of float64
over a non-spiking-to-spiking network trace of 200 steps (stated per test)."""
import numpy as np
import pytest
import torch

import oracle
from conftest import load_fixture
from jaxley_pytorch_b200.graphs import GraphedIteration
from jaxley_pytorch_b200.network import NetworkSimulation, config_network

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["synapse_net_8", "c4_network_72"])
def test_fixture_matches_reference_fp64(cuda_device, name):
    """Reference runs: 8 cells with k = 3, and the fixed in-degree network at 72 cells,
    k = 64 of each synapse type, 4 rows of Poisson input."""
    prob, extra = load_fixture(name)
    net = NetworkSimulation(prob, dtype=torch.float64, device=cuda_device, checkpoint=40)
    out = net.run().cpu().numpy()
    ref = extra["ref"].reshape(out.shape)
    err = np.abs(out - ref).max() / max(1.0, np.abs(ref).max())
    assert err <= 1e-9, err


def _small(n_steps=120, batch=3, seed=1):
    p = config_network(n_cells=24, ncomp=3, k=5, batch=batch, n_steps=n_steps, seed=seed, rate_hz=400.0, amp=0.3)
    p.trainable = [("HH_gNa", np.arange(p.n_nodes))]
    return p


def test_synthetic_network_matches_oracle_fp64(cuda_device):
    prob = _small()
    net = NetworkSimulation(prob, dtype=torch.float64, device=cuda_device, checkpoint=25, max_block_nodes=16)
    out = net.run().cpu().numpy()
    ref = oracle.integrate(prob)
    err = np.abs(out - ref).max() / max(1.0, np.abs(ref).max())
    assert err <= 1e-9, err


def test_fp32_close_to_fp64(cuda_device):
    prob = _small(n_steps=200)
    a = NetworkSimulation(prob, dtype=torch.float64, device=cuda_device).run().cpu().numpy()
    b = NetworkSimulation(prob, dtype=torch.float32, device=cuda_device).run().cpu().numpy()
    assert np.abs(a - b).max() <= 2e-3


def test_gradients_match_central_differences(cuda_device):
    prob = _small(n_steps=80, batch=2)
    net = NetworkSimulation(prob, dtype=torch.float64, device=cuda_device, checkpoint=30, max_block_nodes=16)
    rng = np.random.default_rng(0)
    w = torch.as_tensor(rng.normal(size=(2, len(prob.recordings), 81)), device=cuda_device)
    params = [[p.clone().requires_grad_(True) for p in ty.params] for ty in net.types]
    ps = net.model.pscale.clone().requires_grad_(True)
    loss = (net.run(ps, params) * w).sum()
    flat = [p for ty in params for p in ty]
    grads = torch.autograd.grad(loss, [ps] + flat)
    g_ps, g_par = grads[0], grads[1:]

    def f(ps_, params_):
        with torch.no_grad():
            return float((net.run(ps_, params_) * w).sum())

    base = [[p.detach().clone() for p in ty] for ty in params]
    checks = []
    for t, ty in enumerate(net.types):
        for i in [0, 1]:  # gS and the first kinetic / sigmoid constant
            for e in [0, 7]:
                h = 1e-6 * max(1.0, abs(float(base[t][i][e])))
                plus = [[p.clone() for p in x] for x in base]
                minus = [[p.clone() for p in x] for x in base]
                plus[t][i][e] += h
                minus[t][i][e] -= h
                fd = (f(ps.detach(), plus) - f(ps.detach(), minus)) / (2 * h)
                q = sum(len(x) for x in base[:t]) + i
                checks.append((fd, float(g_par[q][e])))
    for col in range(1, ps.shape[1]):
        for b in range(2):
            h = 1e-6
            p1, p2 = ps.detach().clone(), ps.detach().clone()
            p1[b, col] += h
            p2[b, col] -= h
            checks.append(((f(p1, base) - f(p2, base)) / (2 * h), float(g_ps[b, col])))
    scale = max(abs(c[0]) for c in checks)
    assert scale > 0
    for fd, g in checks:
        assert abs(fd - g) <= 1e-6 * scale, (fd, g)


def test_graphed_adam_training_step_matches_eager(cuda_device):
    """The training step (simulation, MSE loss, adjoint, capturable Adam on the
    synaptic weights of both types) replayed from a CUDA graph equals eager steps."""
    prob = _small(n_steps=60, batch=2)
    net = NetworkSimulation(prob, dtype=torch.float64, device=cuda_device, checkpoint=20, max_block_nodes=16)
    with torch.no_grad():
        target = net.run().detach() + 0.5
    sizes = [ty.E for ty in net.types]

    def run(w):  # w: the gS of both types, concatenated
        parts = torch.split(w, sizes)
        return net.run(net.model.pscale, [[parts[t]] + ty.params[1:] for t, ty in enumerate(net.types)])

    def loss_fn(rec):
        return ((rec - target) ** 2).mean()

    w0 = torch.cat([ty.params[0] for ty in net.types])
    we = w0.clone().requires_grad_(True)
    opt = torch.optim.Adam([we], lr=1e-5, capturable=True)
    for _ in range(4):  # as many steps as the graph below: 2 warm-up + 2 replays
        (g,) = torch.autograd.grad(loss_fn(run(we)), we)
        we.grad = g
        opt.step()
    wg = w0.clone().requires_grad_(True)
    it = GraphedIteration(net, loss_fn, wg, optimizer=torch.optim.Adam([wg], lr=1e-5, capturable=True),
                          warmup=2, run=run)
    assert it.launches_per_replay > 60
    for _ in range(2):
        it.replay()
    torch.cuda.synchronize()
    assert (wg.detach() - we.detach()).abs().max().item() <= 1e-12


def _net_grads(prob, w, device, k, store):
    net = NetworkSimulation(prob, dtype=torch.float64, device=device, checkpoint=k, max_block_nodes=16,
                            store_trajectory=store)
    params = [[p.clone().requires_grad_(True) for p in ty.params] for ty in net.types]
    ps = net.model.pscale.clone().requires_grad_(True)
    loss = (net.run(ps, params) * w).sum()
    return [g.cpu().numpy() for g in torch.autograd.grad(loss, [ps] + [p for ty in params for p in ty])]


@pytest.mark.parametrize("K", [1, 7])
def test_gradients_independent_of_checkpoint_interval(cuda_device, K):
    """Without a stored trajectory the adjoint recomputes each segment's kinetic
    synapse states from its checkpoint; every checkpoint interval must give the
    gradients of a single segment."""
    prob = _small(n_steps=40, batch=2)
    w = torch.as_tensor(np.random.default_rng(3).normal(size=(2, len(prob.recordings), 41)), device=cuda_device)
    ref, got = _net_grads(prob, w, cuda_device, 40, False), _net_grads(prob, w, cuda_device, K, False)
    for a, b in zip(ref, got):
        assert np.abs(a - b).max() <= 1e-10 * max(1.0, np.abs(a).max()), np.abs(a - b).max()


def test_stored_synapse_trajectory_equals_recompute(cuda_device):
    """The adjoint over the stored kinetic states and synaptic terms gives the
    gradients of the recompute form (the same arithmetic on the same values)."""
    prob = _small(n_steps=40, batch=2)
    w = torch.as_tensor(np.random.default_rng(4).normal(size=(2, len(prob.recordings), 41)), device=cuda_device)
    ref, got = _net_grads(prob, w, cuda_device, 7, False), _net_grads(prob, w, cuda_device, 7, True)
    for a, b in zip(ref, got):
        assert np.abs(a - b).max() <= 1e-12 * max(1.0, np.abs(a).max()), np.abs(a - b).max()
