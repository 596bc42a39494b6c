"""`jx.integrate` on the sm_100a kernels.

`integrate(module, params, *, param_state, data_stimuli, data_clamps, t_max, delta_t,
solver, voltage_solver, checkpoint_lengths, all_states, return_states, compile)` has
the signature and the return values of jaxley-pytorch's `integrate`
(`integrate.py:396-666`): recordings of shape `(..., num_recordings, time)` with the
inputs' batch dimensions, and with `return_states=True` also the final states as a
dict of `(..., num_nodes)` arrays. It assembles the module's problem on the host with
the reference's own module API (`problem_from_module`), lowers it, and runs the fused
forward kernel; the result is differentiable with respect to the trainable `params`
and to `param_state` values that require gradients, through the hand-written adjoint
kernel (channel parameters; geometry has no gradient here).

The simulation runs on the CUDA device of the inputs, or on the current CUDA device
when the inputs are on the CPU (there is no CPU path); the recordings are returned on
the inputs' device, in the inputs' dtype (float32 or float64). `solver` is
`bwd_euler` or `crank_nicolson` (`fwd_euler` and `exp_euler` are not covered).
`voltage_solver`
accepts the reference's names: every one of them solves the same tree system, here
with the chain-ordered DHS solve. `checkpoint_lengths` sets the adjoint's segment
length (its innermost entry), `compile` is accepted and has no effect (the kernels
are compiled ahead of time).
"""
from __future__ import annotations

from typing import Dict, List, Optional

import numpy as np
import torch

from .lower import lower
from .problem import differentiable, host_mode, problem_from_module
from .sim import Simulation

VOLTAGE_SOLVERS = ("jaxley.dhs", "jaxley.dhs.cpu", "jaxley.dhs.gpu", "jaxley.stone",
                   "jax.sparse", "torch.dense")


def _first_float_tensor(*trees):
    """The first floating-point tensor in the given (nested) inputs, as the reference
    infers the simulation's device and dtype (integrate.py:480-490)."""
    for tree in trees:
        stack = [tree]
        while stack:
            x = stack.pop(0)
            if isinstance(x, torch.Tensor):
                if x.is_floating_point():
                    return x
            elif isinstance(x, dict):
                stack.extend(x.values())
            elif isinstance(x, (list, tuple)):
                stack.extend(x)
    return None


def _has_tangent(x) -> bool:
    """Whether a tensor carries a forward-mode tangent."""
    import torch.autograd.forward_ad as fwAD

    if torch._C._functorch.is_functorch_wrapped_tensor(x):
        return True
    return fwAD._current_level >= 0 and fwAD.unpack_dual(x).tangent is not None


def _group_values(t: torch.Tensor, g: int, batch_shape, device, dtype) -> torch.Tensor:
    """Per-row values of group g of a trainable tensor `(..., n_groups)`."""
    v = t[..., g] if t.dim() > 0 and t.shape[-1] > g else (t[..., 0] if t.dim() > 0 else t)
    v = v.to(device=device, dtype=dtype)
    if len(batch_shape):
        v = torch.broadcast_to(v, tuple(batch_shape)).reshape(-1)
    return v.reshape(-1)


def named_states(sim: Simulation, problem, state: torch.Tensor) -> Dict[str, torch.Tensor]:
    """The states of a `(B, n_slots)` state vector as `{name: (B, n_nodes)}` in the
    reference's node order: simulated values where a node has the state, the initial
    value elsewhere."""
    low = sim.low
    B, n = state.shape[0], low.n_nodes
    names = low.slot_names
    out = {}
    for name, init in problem.states.items():
        arr = torch.as_tensor(np.asarray(init, dtype=np.float64), dtype=state.dtype, device=state.device)
        arr = torch.broadcast_to(arr, (B, n)).clone()
        nodes, slots = [], []
        for g, gnames in enumerate(names.grp_names):
            if name in gnames:
                idx = np.nonzero(np.asarray(names.grp_int) == g)[0]
                nodes.append(low.int2node[idx])
                slots.append(np.asarray(low.soff)[idx] + gnames.index(name))
        if nodes:
            nd = torch.as_tensor(np.concatenate(nodes), device=state.device)
            sl = torch.as_tensor(np.concatenate(slots), device=state.device)
            arr[:, nd] = state[:, sl]
        out[name] = arr
    return out


def integrate(module, params: list = [], *, param_state: Optional[list] = None, data_stimuli=None,
              data_clamps=None, t_max: Optional[float] = None, delta_t: float = 0.025,
              solver: str = "bwd_euler", voltage_solver: str = "jaxley.dhs",
              checkpoint_lengths: Optional[List[int]] = None, all_states: Optional[dict] = None,
              return_states: bool = False, compile: bool = False):
    """Simulates `module` with the fused CUDA kernels (see the module docstring)."""
    if solver not in ("bwd_euler", "crank_nicolson"):
        raise NotImplementedError(f"solver={solver!r}: the CUDA step covers bwd_euler and crank_nicolson")
    if voltage_solver not in VOLTAGE_SOLVERS:
        raise ValueError(f"Unknown voltage_solver: {voltage_solver}.")
    assert module.initialized, "Module is not initialized, run `._initialize()`."
    if module.recordings.empty:
        raise ValueError("No recordings are set. Please set them.")
    ref = _first_float_tensor(params, param_state, data_stimuli[1] if data_stimuli is not None else None,
                              data_clamps[1] if data_clamps is not None else None, all_states)
    dtype = ref.dtype if ref is not None else torch.get_default_dtype()
    if dtype not in (torch.float32, torch.float64):
        raise TypeError(f"unsupported dtype {dtype}")
    out_device = ref.device if ref is not None else torch.device("cpu")
    if out_device.type == "cuda":
        sim_device = out_device
    elif torch.cuda.is_available():
        sim_device = torch.device("cuda", torch.cuda.current_device())
    else:
        raise RuntimeError("jaxley_pytorch_b200.integrate runs on a CUDA device; none is available")

    with host_mode():  # the host-side assembly reads tensors, also under torch.func transforms
        prob = problem_from_module(module, params=params, param_state=param_state, data_stimuli=data_stimuli,
                                   t_max=t_max, delta_t=delta_t, data_clamps=data_clamps,
                                   all_states=all_states, solver=solver)
        if prob.synapses:
            raise NotImplementedError("networks with synapses: use jaxley_pytorch_b200.network.NetworkSimulation "
                                      "or the reference's integrate with the drop-in kernels installed")
        K = int(checkpoint_lengths[-1]) if checkpoint_lengths else 100
        low = lower(prob)
        sim = Simulation(prob, low=low, dtype=dtype, device=sim_device, checkpoint=K)
    pscale = sim.model.pscale
    sources = [list(e.values())[0] for e in params] + [e["val"] for e in (param_state or [])]
    for tree in (data_stimuli[1] if data_stimuli is not None else [],
                 data_clamps[1] if data_clamps is not None else [], list((all_states or {}).values())):
        if any(isinstance(x, torch.Tensor) and _has_tangent(x) for x in tree):
            raise NotImplementedError("forward-mode derivatives with respect to stimuli, clamps or states "
                                      "are not covered")
    wants = any(differentiable(t) for t in sources) and (
        torch.is_grad_enabled() or torch.autograd.forward_ad._current_level >= 0)
    if wants and prob.trainable:
        cols, base = low.group_scale()
        columns = list(pscale.unbind(1))
        B = pscale.shape[0]
        for q, (src, g) in enumerate(prob.trainable_source):
            t = sources[src]
            if not differentiable(t):
                continue
            if cols[q] <= 0:
                raise NotImplementedError(f"trainable {prob.trainable[q][0]}: its nodes do not share one value")
            v = _group_values(t, g, prob.batch_shape, sim_device, dtype)
            columns[cols[q]] = torch.broadcast_to(v / float(base[q]), (B,))
        pscale = torch.stack(columns, 1)
    rec = sim.run(pscale=pscale)  # (B, n_rec, T + 1)
    shape = tuple(prob.batch_shape) + tuple(rec.shape[1:])
    rec = rec.reshape(shape).to(out_device)
    if not return_states:
        return rec
    with host_mode():
        states = named_states(sim, prob, sim.last_state)
        n = prob.n_nodes
        states = {k: v.reshape(tuple(prob.batch_shape) + (n,)).to(out_device) for k, v in states.items()}
    return rec, states
