"""The hand-written adjoint against the reference's own autograd gradients.

The fixtures hold gradients that the reference computed with `loss.backward()` through
its `jx.integrate` (autograd of the step, `_DHSSolve.backward` at
`solver_voltage.py:143-187`), for the linear loss `sum(loss_w * recordings)`, in
float64 (written by `tests/golden/make_fixtures.py`). The CUDA adjoint in float64 must
agree to 1e-6 relative (of the largest gradient of each array); the trainables cover
`make_trainable` groups (one value per cell, branch or view, shared over the batch),
per-row `data_set` conductances of the benchmarked L5PC tree, every cell's own
conductances of the uneven batch, a clamped cell, and every synapse's gS of two
networks.
"""
import numpy as np
import pytest
import torch

from conftest import load_fixture
from jaxley_pytorch_b200.lower import lower
from jaxley_pytorch_b200.network import NetworkSimulation
from jaxley_pytorch_b200.sim import Simulation

pytestmark = pytest.mark.gpu

REL = 1e-6


def _close(got, ref, what):
    got, ref = np.asarray(got, dtype=np.float64), np.asarray(ref, dtype=np.float64)
    scale = np.abs(ref).max()
    assert scale > 0, what
    err = np.abs(got - ref).max() / scale
    assert err <= REL, (what, err)
    return err


def _pgrad(prob, extra, dtype=torch.float64, device="cuda"):
    low = lower(prob)
    sim = Simulation(prob, low=low, dtype=dtype, device=device, checkpoint=50,
                     init_steady=bool(extra.get("init_steady", 0)))
    ps = sim.model.pscale.clone().requires_grad_(True)
    rec = sim.run(pscale=ps)
    w = torch.as_tensor(extra["loss_w"], device=device).reshape(rec.shape).to(rec.dtype)
    (rec * w).sum().backward()
    return low, ps.grad.double().cpu().numpy(), rec.detach().double().cpu().numpy()


@pytest.mark.parametrize("name", ["l5pc_7x4_batch3", "hh_clamp_7x3", "pospischil_7x3", "cn_hh_7x3"])
def test_make_trainable_groups(cuda_device, name):
    """Every group of every trainable (one per row of indices_set_by_trainables)."""
    prob, extra = load_fixture(name)
    low, pg, _ = _pgrad(prob, extra, device=cuda_device)
    cols, base = low.group_scale()
    src = extra["trainable_source"]
    n_entries = int(src[:, 0].max()) + 1
    for q in range(n_entries):
        ref = extra[f"grad_{q}"].reshape(-1)  # one value per group, summed over the batch
        groups = np.nonzero(src[:, 0] == q)[0]
        got = np.zeros(len(ref))
        for g in groups:
            assert cols[g] > 0, (q, g)
            got[src[g, 1]] = pg[:, cols[g]].sum() / base[g]
        _close(got, ref, (name, q))


def test_c2_tree_per_row_conductances(cuda_device):
    """The 300 x 4 L5PC tree: gradients with respect to every scaled conductance of
    every parameter set (data_set with a batch dimension, one column per profile)."""
    prob, extra = load_fixture("c2_l5pc_tree_b2")
    low, pg, _ = _pgrad(prob, extra, device=cuda_device)
    names = bytes(extra["grad_names"]).decode().split(",")
    for q, nm in enumerate(names):
        cols = [c for c in range(1, low.n_cols) if low.col_info[c][0] == nm]
        assert len(cols) == 1, (nm, cols)
        bases = {round(b, 15) for _, _, b in low.col_members[cols[0]]}
        assert len(bases) == 1
        got = pg[:, cols[0]] / bases.pop()
        _close(got, extra[f"grad_{q}"].reshape(-1), nm)


def test_c3_uneven_cells_own_conductances(cuda_device):
    """Eight cells of the uneven batch (HH and L5PC, up to 3000 compartments): every
    cell's trainable conductances."""
    prob, extra = load_fixture("c3_uneven_8")
    low, pg, _ = _pgrad(prob, extra, device=cuda_device)
    cols, base = low.group_scale()
    got = np.asarray([pg[:, cols[g]].sum() / base[g] for g in range(len(prob.trainable))])
    ref = np.asarray([extra[f"grad_{g}"].reshape(-1)[0] for g in range(len(prob.trainable))])
    _close(got, ref, "c3")


@pytest.mark.parametrize("name,ntypes", [("synapse_net_8", 2), ("c4_network_72", 2)])
def test_network_synapse_weights(cuda_device, name, ntypes):
    """Every synapse's gS of both synapse types and the shared HH_gNa."""
    prob, extra = load_fixture(name)
    if not prob.trainable:
        prob.trainable = [("HH_gNa", np.arange(prob.n_nodes))]
    net = NetworkSimulation(prob, dtype=torch.float64, device=cuda_device, checkpoint=40)
    params = [[p.clone().requires_grad_(True) for p in ty.params] for ty in net.types]
    ps = net.model.pscale.clone().requires_grad_(True)
    rec = net.run(ps, params)
    w = torch.as_tensor(extra["loss_w"], device=cuda_device).reshape(rec.shape)
    (rec * w).sum().backward()
    for t in range(ntypes):
        _close(params[t][0].grad.cpu().numpy(), extra[f"grad_{t}"], (name, t))
    cols, base = net.low.group_scale()
    g_na = ps.grad[:, cols[0]].sum().item() / base[0]
    _close([g_na], extra[f"grad_{ntypes}"].reshape(-1), (name, "HH_gNa"))
