"""Host-side assembly of a reference module into a `Problem` and its lowering (no GPU):
trainable groups from `make_trainable` and from `data_set` values that require
gradients, clamps from `Module.clamp` / `data_clamp`, one batch shape for all inputs,
and the lowered clamp and gradient-column tables. Runs the reference on the CPU."""
import numpy as np
import pytest
import torch

import reference_models as rm
from conftest import import_reference
from jaxley_pytorch_b200.lower import V_SOLVE, lower
from jaxley_pytorch_b200.problem import problem_from_module


def test_trainable_groups_follow_make_trainable():
    jx = import_reference()
    cell, kw = rm.hh_tree(jx)
    params = cell.get_parameters()
    prob = problem_from_module(cell, params=params, delta_t=0.025)
    names = [k for k, _ in prob.trainable]
    assert names == ["HH_gNa"] + ["HH_gK"] * 15  # one value, then one per branch
    assert len(prob.trainable[0][1]) == 45
    assert [len(nodes) for _, nodes in prob.trainable[1:]] == [3] * 15
    assert prob.trainable_source == [(0, 0)] + [(1, g) for g in range(15)]
    low = lower(prob)
    cols, base = low.group_scale()
    assert np.all(cols > 0) and len(set(cols.tolist())) == 16
    assert np.allclose(base[0], 0.12) and np.allclose(base[1:], 0.036)


def test_data_set_gradient_groups_and_batch_shape():
    jx = import_reference()
    cell, kw = rm.hh_tree(jx)
    val = torch.tensor([[0.10], [0.12], [0.14]], dtype=torch.float64, requires_grad=True)
    ps = cell.branch(2).data_set("HH_gNa", val, None)
    ps = cell.data_set("HH_gLeak", torch.tensor(3e-4, dtype=torch.float64), ps)  # no gradient
    prob = problem_from_module(cell, param_state=ps, delta_t=0.025)
    assert prob.batch == 3 and tuple(prob.batch_shape) == (3,)
    assert [k for k, _ in prob.trainable] == ["HH_gNa"]  # one group: the broadcast value
    assert len(prob.trainable[0][1]) == 3
    low = lower(prob)
    cols, base = low.group_scale()
    assert cols[0] > 0 and np.allclose(low.pscale[:, cols[0]] * base[0], [0.10, 0.12, 0.14])


def test_clamps_are_assembled_and_lowered():
    jx = import_reference()
    cell, kw = rm.clamped_cell(jx, torch)
    prob = problem_from_module(cell, data_clamps=kw["data_clamps"], delta_t=0.025)
    assert [c[0] for c in prob.clamps] == ["v", "HH_m"]
    for _, nodes, vals in prob.clamps:
        assert len(nodes) == 1 and vals.shape == (1, 1, prob.n_steps)
    assert prob.n_steps == 241
    low = lower(prob)
    vnode = int(low.node2int[prob.clamps[0][1][0]])
    mnode = int(low.node2int[prob.clamps[1][1][0]])
    assert low.slot_names[vnode][-1] == V_SOLVE
    assert V_SOLVE not in low.slot_names[mnode]
    assert low.clamp_ptr[vnode + 1] - low.clamp_ptr[vnode] == 1
    assert low.clamp_slot[low.clamp_ptr[vnode]] == 0
    assert low.slot_names[mnode][low.clamp_slot[low.clamp_ptr[mnode]]] == "HH_m"
    assert low.clamp.shape == (241, 1, 2)
    np.testing.assert_allclose(low.clamp[:, 0, 1], 0.3, rtol=1e-7)


def test_short_clamp_is_refused():
    jx = import_reference()
    cell, kw = rm.clamped_cell(jx, torch)
    with pytest.raises(NotImplementedError):
        problem_from_module(cell, data_clamps=kw["data_clamps"], t_max=20.0, delta_t=0.025)


def test_differentiable_and_unwrap():
    """Inputs that ask for derivatives are recognised in reverse mode, inside a
    forward-AD level and under `torch.func.jvp`, whose wrapped tensors are read
    through `unwrap` in `host_mode`."""
    import torch
    import torch.autograd.forward_ad as fwAD

    from jaxley_pytorch_b200.problem import _cpu64, differentiable, host_mode, unwrap

    x = torch.tensor([1.0, 2.0], dtype=torch.float64)
    assert not differentiable(x) and not differentiable(3.0)
    assert differentiable(x.clone().requires_grad_(True))
    with fwAD.dual_level():
        d = fwAD.make_dual(x, torch.ones_like(x))
        assert differentiable(d)
        assert not differentiable(x)
        assert torch.equal(_cpu64(d), x)
    seen = {}

    def f(y):
        seen["diff"] = differentiable(y)
        with host_mode():
            seen["val"] = _cpu64(y).numpy().copy()
        seen["plain"] = unwrap(y) is not y
        return y * 2

    torch.func.jvp(f, (x,), (torch.ones_like(x),))
    assert seen["diff"] and seen["plain"]
    np.testing.assert_array_equal(seen["val"], [1.0, 2.0])
