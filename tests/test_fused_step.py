"""`fused_step`, the entry `Network._step_regular_synapses` calls
(reference `modules/network.py:402-407`, `kernels/synapse_step.py:451-498`), and the
plan helpers it relies on.

CPU: the presynaptic lists of the backward pass hold every synapse exactly once,
grouped by presynaptic node; `kernel_scalars` holds the exact values; `fused_step`
declines (returns `None`) where the reference's does. GPU: the node-space slope and
offset and the new states equal an autograd-free restatement of the synapse step
(float64, 1e-9 relative), for both models, targets that are nodes or a subset, and
voltages with two leading batch dimensions.
"""
import numpy as np
import pytest
import torch

from jaxley_pytorch_b200.kernels import synapse_step as ss
from jaxley_pytorch_b200.lower import presynaptic_lists


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_presynaptic_lists_cover_every_synapse_once(seed):
    rng = np.random.default_rng(seed)
    E = int(rng.integers(1, 400))
    pre = rng.integers(0, 37, E)
    nodes, lists = presynaptic_lists(pre)
    assert np.all(np.diff(nodes) > 0)
    assert set(nodes.tolist()) == set(pre.tolist())
    assert lists.shape == (len(nodes), np.bincount(pre).max())
    flat = lists[lists >= 0]
    assert sorted(flat.tolist()) == list(range(E))
    for r, node in enumerate(nodes):
        row = lists[r][lists[r] >= 0]
        assert np.all(pre[row] == node)
        assert np.all(np.diff(row) > 0)  # synapses of a node in index order
        assert np.all(lists[r][len(row):] == -1)  # padding only at the end


def test_presynaptic_lists_empty():
    nodes, lists = presynaptic_lists(np.zeros(0, dtype=np.int64))
    assert nodes.shape == (0,) and lists.shape == (0, 1)


def test_kernel_scalars_are_exact():
    s = ss.kernel_scalars(0.025, 1e-3, torch.float64, "cpu")
    assert s.dtype == torch.float64 and s.tolist() == [0.025, 1e-3]


class _Syn:
    def __init__(self, name):
        self._name = name


def _plan(model, n, targets, k, pre, dev, name):
    nodes, inv = presynaptic_lists(pre)
    sp = {
        "kernel_model": model,
        "kernel_params": [f"{name}_{p}" for p in ss._NAMES[model]],
        "kernel_pre": torch.as_tensor(pre, dtype=torch.int32, device=dev),
        "kernel_targets": torch.as_tensor(targets, dtype=torch.int32, device=dev),
        "kernel_pre_nodes": torch.as_tensor(nodes, device=dev),
        "kernel_inv": torch.as_tensor(inv, device=dev),
        "pre_per_target": torch.zeros(len(targets), k),
        "targets": torch.as_tensor(targets, dtype=torch.long, device=dev),
        "targets_are_nodes": len(targets) == n and np.array_equal(targets, np.arange(n)),
        "synapse": _Syn(name),
    }
    return sp


def test_fused_step_declines_where_the_reference_does():
    sp = _plan(0, 4, np.arange(4), 2, np.arange(8) % 4, "cpu", "KineticSynapse")
    v = torch.zeros(3, 4, dtype=torch.float64)
    gp = {"params": {}, "area_post": torch.ones(8, dtype=torch.float64),
          "kernel_scalars": ss.kernel_scalars(0.025, 1e-3, torch.float64, "cpu")}
    assert ss.fused_step({"v": v}, 0.025, sp, gp) is None  # not on a CUDA device
    assert ss.fused_step({"v": v}, 0.025, {}, gp) is None  # no kernel entries
    assert ss.fused_step({"v": v}, 0.025, sp, {}) is None  # no kernel scalars


def _restated(model, v, s, pre, targets, k, params, area, dt, diff):
    """The synapse step of one type in numpy (modules/network.py:434-478): new states,
    current and the node-space slope and offset (offset with the caller's sign)."""
    vpre = v[:, pre]
    vp = np.repeat(v[:, targets], k, axis=1)
    gs = params[0]
    if model == 0:
        e_syn, alpha, beta, v_th, delta = params[1:6]
        a = alpha / (1 + np.exp(-(vpre - v_th) / delta))
        rate = a + beta
        s_inf = a / rate
        s_new = s_inf + (s - s_inf) * np.exp(-dt * rate)
        i0 = gs * s_new * (vp - e_syn)
        i1 = gs * s_new * ((vp + diff) - e_syn)
    else:
        x_off, slope = params[1:3]
        s_new = None
        sig = lambda x: 1 / (1 + np.exp(-x))  # noqa: E731
        i0 = -gs * sig((vpre - x_off) * slope)
        i1 = -gs * sig(((vpre + diff) - x_off) * slope)
    d0 = i0 / area * 1e5
    d1 = i1 / area * 1e5
    lin = (d1 - d0) / diff
    cst = d0 - lin * vp
    B, n = v.shape
    node_lin, node_cst = np.zeros((B, n)), np.zeros((B, n))
    np.add.at(node_lin.T, targets, lin.reshape(B, -1, k).sum(-1).T)
    np.add.at(node_cst.T, targets, cst.reshape(B, -1, k).sum(-1).T)
    return s_new, i0, node_lin, -node_cst


@pytest.mark.gpu
@pytest.mark.parametrize("model", [0, 1])
@pytest.mark.parametrize("all_nodes", [False, True])
def test_fused_step_matches_restatement(cuda_device, model, all_nodes):
    rng = np.random.default_rng(3 + model)
    n, k = 24, 5
    targets = np.arange(n) if all_nodes else np.sort(rng.choice(n, 9, replace=False))
    E = len(targets) * k
    pre = rng.integers(0, n, E)
    lead = (2, 3)
    name = "KineticSynapse" if model == 0 else "SigmoidRateSynapse"
    ranges = {0: [(1e-4, 1e-3), (-80.0, 0.0), (0.5, 2.0), (0.05, 0.5), (-40.0, 0.0), (1.0, 4.0)],
              1: [(-1e-3, 1e-3), (-70.0, -40.0), (0.05, 0.5)]}[model]
    params = [rng.uniform(lo, hi, E) for lo, hi in ranges]
    area = rng.uniform(100.0, 500.0, E)
    v = rng.uniform(-80, 20, lead + (n,))
    t = lambda x: torch.as_tensor(x, dtype=torch.float64, device=cuda_device)  # noqa: E731
    sp = _plan(model, n, targets, k, pre, cuda_device, name)
    gp = {"params": {f"{name}_{p}": t(x) for p, x in zip(ss._NAMES[model], params)},
          "area_post": t(area), "store_current": True,
          "kernel_scalars": ss.kernel_scalars(0.025, 1e-3, torch.float64, cuda_device)}
    states = {"v": t(v)}
    s = None
    if model == 0:
        s = rng.uniform(0, 1, lead + (E,))
        states[f"{name}_s"] = t(s)
    out = ss.fused_step(states, 0.025, sp, gp)
    assert out is not None
    new_states, (lin, cst) = out
    r_s, r_i, r_lin, r_cst = _restated(model, v.reshape(-1, n), None if s is None else s.reshape(-1, E),
                                       pre, targets, k, params, area, 0.025, 1e-3)
    assert tuple(lin.shape) == lead + (n,) and tuple(cst.shape) == lead + (n,)

    def rel(a, b):
        a = a.detach().cpu().numpy().reshape(b.shape)
        return np.abs(a - b).max() / max(np.abs(b).max(), 1e-300)

    assert rel(lin, r_lin) <= 1e-9
    assert rel(cst, r_cst) <= 1e-9
    assert rel(new_states[f"i_{name}"], r_i) <= 1e-9
    if model == 0:
        assert rel(new_states[f"{name}_s"], r_s) <= 1e-12
    assert states.keys() <= new_states.keys()  # the input dict itself is left as it was
    assert f"i_{name}" not in states
