"""The problem format: everything one simulation of the hot path consumes.

A `Problem` holds, in the reference's node order, what `jx.integrate` assembles
before its step loop (`integrate.py:481-622` in jaxley-pytorch):

* the tree system of the implicit-Euler voltage step, as the reference stores it:
  axial conductances per compartment edge (`utils/morph_attributes.py:315-436`), the
  edge sinks (`modules/base.py:3080-3084`) and the DHS solve order with its lower /
  upper maps and parent lookup (`modules/base.py:1142-1266`,
  `modules/network.py:192-293`);
* the inserted channels in insertion order with their node indices
  (`modules/base.py:3050-3068`);
* all parameters and initial states as `(B, n_nodes)` or `(n_nodes,)` arrays,
  including the initial channel currents (`modules/base.py:2375-2383`);
* the step-current stimuli (`integrate.py:495-568`) and the recordings
  (`integrate.py:53-84`);
* regular-layout synapse types (`modules/network.py:295-348`).

A `Problem` comes either from a reference `Module` (`problem_from_module`, for users
of jaxley-pytorch and for the parity fixtures) or from the seeded generators in
`synth.py`. Both the CUDA path (`lower.py`) and the CPU restatement consume it.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

from .channels import ChannelInstance, spec_for_reference_channel, current_name


@dataclass
class SynapseType:
    """A synapse type in the regular layout: synapses ordered by postsynaptic node,
    `k` per node (`utils/syn_utils.py:13-27`). `model` is 0 for `KineticSynapse`,
    1 for `SigmoidRateSynapse` (`kernels/synapse_step.py:43`)."""

    model: int
    name: str
    pre: np.ndarray  # (E,) presynaptic node index (reference node order)
    post: np.ndarray  # (E,) postsynaptic node index
    k: int
    targets: np.ndarray  # (E // k,) postsynaptic nodes, increasing
    params: List[np.ndarray]  # one (E,) array per parameter, in the reference order
    param_names: List[str]
    state: Optional[np.ndarray]  # (B or 1, E) initial `s` (kinetic), else None
    current: Optional[np.ndarray] = None  # (B or 1, E) initial current (recording)


@dataclass
class Problem:
    n_nodes: int
    comp_inds: np.ndarray  # compartments (nodes that are not branchpoints)
    # Tree system (reference layout).
    sinks: np.ndarray  # (E_ax,) sink node of every compartment edge
    axial: np.ndarray  # (E_ax,) or (B, E_ax) axial conductances (divided by cm)
    parent_lookup: np.ndarray  # (n_nodes,) parent in solve order, -1 for roots
    to_solve: np.ndarray  # (n_nodes,) node index of solve position j
    map_lower: np.ndarray  # (n_nodes,) axial edge of the lower of solve position j
    map_upper: np.ndarray  # (n_nodes,) axial edge of the upper of solve position j
    channels: List[ChannelInstance]
    params: Dict[str, np.ndarray]
    states: Dict[str, np.ndarray]
    dt: float
    n_steps: int  # number of steps simulated (recordings have n_steps + 1 samples)
    stim_inds: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int64))
    stim: Optional[np.ndarray] = None  # (B or 1, n_stim, >= n_steps) in nA
    recordings: List[Tuple[str, int]] = field(default_factory=list)
    synapses: List[SynapseType] = field(default_factory=list)
    batch: int = 1
    current_names: List[str] = field(default_factory=list)
    # Trainable parameter groups `(parameter name, reference nodes)`: the nodes of a
    # group share one scale column and so one gradient, like one `make_trainable`
    # call on a view in the reference (`modules/base.py:1625`).
    trainable: List[Tuple[str, np.ndarray]] = field(default_factory=list)
    # Clamps `(state name, reference nodes (n_c,), values (B or 1, n_c, >= n_steps))`:
    # after step t the state of node q is set to values[..., q, t]; a voltage clamp
    # after the voltage solve, any other state after the channel update of the step
    # (`modules/base.py:3305-3308, 3396-3398`). For a node clamped twice the later
    # entry wins.
    clamps: List[Tuple[str, np.ndarray, np.ndarray]] = field(default_factory=list)
    # Step scheme of the voltage: "bwd_euler" or "crank_nicolson" (modules/base.py:3327-3365).
    solver: str = "bwd_euler"

    def solve_order_system(self):
        """Per solve position `j`: parent, `g_low[j]` (coupling of row `j` to its
        parent) and `g_up[j]` (coupling of the parent's row to `j`), both as axial
        conductances before the `-dt` factor (`solver_voltage.py:330-348`)."""
        parent = np.asarray(self.parent_lookup, dtype=np.int64)
        ax = np.asarray(self.axial, dtype=np.float64)
        if ax.shape[-1] == 0:
            z = np.zeros(ax.shape[:-1] + (self.n_nodes,))
            return parent, z, z
        g_low = ax[..., self.map_lower]
        g_up = ax[..., self.map_upper]
        has = parent >= 0
        g_low = np.where(has, g_low, 0.0)
        g_up = np.where(has, g_up, 0.0)
        return parent, g_low, g_up

    def gsum(self):
        """Sum of the axial conductances of the edges that sink into every node."""
        ax = np.asarray(self.axial, dtype=np.float64)
        if ax.shape[-1] == 0:
            return np.zeros(ax.shape[:-1] + (self.n_nodes,))
        rows = ax.reshape(-1, ax.shape[-1])
        out = np.zeros((rows.shape[0], self.n_nodes))
        for b in range(rows.shape[0]):
            np.add.at(out[b], np.asarray(self.sinks, dtype=np.int64), rows[b])
        return out if ax.ndim == 2 else out[0]


def _np(x, dtype=np.float64):
    import torch

    if isinstance(x, torch.Tensor):
        return x.detach().cpu().numpy().astype(dtype)
    return np.asarray(x, dtype=dtype)


def _flatten_batch(a: np.ndarray) -> np.ndarray:
    """`(..., n)` -> `(n,)` without batch dims, else `(B, n)`."""
    if a.ndim <= 1:
        return a
    return a.reshape(-1, a.shape[-1])


def _flatten_to(a: np.ndarray, batch_shape: tuple, core: int = 1) -> np.ndarray:
    """An array with `core` trailing dimensions and optional leading batch dimensions:
    unchanged without batch dimensions, else broadcast to `batch_shape` and flattened
    to one leading dimension."""
    if a.ndim <= core:
        return a
    tail = a.shape[a.ndim - core:]
    return np.broadcast_to(a, tuple(batch_shape) + tail).reshape((-1,) + tail)


def unwrap(x):
    """The plain tensor under the wrappers of `torch.func` transforms (`jvp`, `grad`),
    whose data cannot be read directly (other values unchanged)."""
    import torch

    ft = torch._C._functorch
    while isinstance(x, torch.Tensor) and ft.is_functorch_wrapped_tensor(x):
        x = ft.get_unwrapped(x)
    return x


def host_mode():
    """A context in which tensors can be read on the host (`.numpy()`, `data_ptr()`)
    also inside `torch.func` transforms: their functorch layers are switched off, and
    tensors made inside are plain."""
    import torch

    return torch._C._DisableFuncTorch()


def differentiable(x) -> bool:
    """Whether a tensor asks for derivatives: it requires grad (reverse mode) or
    carries a forward-mode tangent (`torch.autograd.forward_ad`, `torch.func.jvp`)."""
    import torch
    import torch.autograd.forward_ad as fwAD

    if not isinstance(x, torch.Tensor):
        return False
    if x.requires_grad or torch._C._functorch.is_functorch_wrapped_tensor(x):
        return True
    return fwAD._current_level >= 0 and fwAD.unpack_dual(x).tangent is not None


def _cpu64(x):
    """A detached CPU float64 copy of a tensor (other values unchanged)."""
    import torch

    x = unwrap(x)
    if isinstance(x, torch.Tensor):
        return x.detach().to(device="cpu", dtype=torch.float64)
    return x


def _broadcast_last(x) -> bool:
    """Whether the last dimension of a tensor is a broadcast (stride 0) of one value."""
    import torch

    x = unwrap(x)
    return isinstance(x, torch.Tensor) and x.dim() > 0 and x.shape[-1] > 1 and x.stride(-1) == 0


# Parameters that enter the axial conductances (`utils/morph_attributes.py:315-436`)
# or the membrane area rather than a channel: the CUDA adjoint has no gradient for them.
GEOMETRY_PARAMS = ("radius", "length", "axial_resistivity", "capacitance", "area")


def problem_from_module(
    module,
    params: list = [],
    param_state: Optional[list] = None,
    data_stimuli=None,
    t_max: Optional[float] = None,
    delta_t: float = 0.025,
    data_clamps=None,
    all_states: Optional[dict] = None,
    solver: str = "bwd_euler",
) -> Problem:
    """Lower a reference `jx.Module` (jaxley-pytorch) into a `Problem`.

    Follows `jx.integrate` (`integrate.py:476-622`): the stimulus is padded or
    truncated to `int(t_max // delta_t + 1)` samples, clamps truncated (they must be
    at least that long, `integrate.py:528-545`), parameters come from
    `get_all_parameters`, initial states from `get_all_states` plus the initial
    currents (`_append_currents_with_plan`), or from `all_states` (a previous run's
    final states). Every group of the trainable `params` (one per row of
    `module.indices_set_by_trainables`) that sets a channel parameter of nodes
    becomes a `Problem.trainable` group; `problem.trainable_source[q] = (entry, group)`
    names where group q came from. `solver` is the step scheme, `bwd_euler` or
    `crank_nicolson`, both with the DHS solve.
    """
    if solver not in ("bwd_euler", "crank_nicolson"):
        raise NotImplementedError(f"solver={solver!r}: the CUDA step covers bwd_euler and crank_nicolson")
    import torch

    from jaxley_pytorch.integrate import _batch_shape, _expand_states  # noqa: F401
    from jaxley_pytorch.utils.cell_utils import params_to_pstate
    from jaxley_pytorch.utils.torch_utils import tree_tensors

    base = module.base
    device = torch.device("cpu")
    dtype = torch.float64
    module.to_torch(device=device, dtype=dtype)
    # Inputs may live on any device and dtype: the problem is assembled from detached
    # float64 copies on the CPU (which entries ask for gradients is noted first).
    ps_grad = [(differentiable(e["val"]), _broadcast_last(e["val"]))
               for e in (param_state or [])]
    params = [{k: _cpu64(v) for k, v in e.items()} for e in params]
    if param_state is not None:
        param_state = [dict(e, val=_cpu64(e["val"])) for e in param_state]
    if data_stimuli is not None:
        data_stimuli = (data_stimuli[0], [_cpu64(v) for v in data_stimuli[1]], data_stimuli[2])
    if data_clamps is not None:
        data_clamps = (data_clamps[0], [_cpu64(v) for v in data_clamps[1]], data_clamps[2])
    if all_states is not None:
        all_states = {k: _cpu64(v) for k, v in all_states.items()}

    externals = {k: torch.as_tensor(v, dtype=dtype) for k, v in module.externals.items()}
    external_inds = dict(module.external_inds)
    from jaxley_pytorch.integrate import add_clamps, add_stimuli

    externals, external_inds = add_stimuli(externals, external_inds, data_stimuli)
    externals, external_inds = add_clamps(externals, external_inds, data_clamps)
    clamp_keys = [k for k in externals if k != "i"]
    if "i" in externals:
        stim = externals["i"]
        n_samples = stim.shape[-1]
        if t_max is not None:
            want = int(t_max // delta_t + 1)
            if want > n_samples:
                pad = torch.zeros((*stim.shape[:-1], want - n_samples), dtype=dtype)
                stim = torch.cat([stim, pad], dim=-1)
            else:
                stim = stim[..., :want]
        n_steps = stim.shape[-1]
        stim_np = _np(stim)
        stim_inds = np.asarray(external_inds["i"], dtype=np.int64)
    else:
        stim_np, stim_inds = None, np.zeros(0, np.int64)
        if clamp_keys and t_max is None:
            n_steps = int(torch.as_tensor(externals[clamp_keys[0]]).shape[-1])
        else:
            if t_max is None:
                raise ValueError("without a stimulus or clamp, t_max is required")
            n_steps = int(t_max // delta_t + 1)
    clamps = []
    for key in clamp_keys:
        vals = _np(externals[key])
        if vals.shape[-1] < n_steps:
            raise NotImplementedError("clamp must be at least as long as simulation.")
        vals = vals[..., :n_steps]
        if vals.ndim == 1:
            vals = vals.reshape(1, -1)
        clamps.append((str(key), np.asarray(external_inds[key], dtype=np.int64).reshape(-1), vals))

    pstate = params_to_pstate(params, module.indices_set_by_trainables)
    if param_state is not None:
        pstate = pstate + list(param_state)
    all_params = module.get_all_parameters(pstate)
    if all_states is None:
        init_states = module.get_all_states(pstate)
        batch = _batch_shape(list(tree_tensors(all_params)) + list(tree_tensors(init_states)))
        init_states = _expand_states(init_states, batch)
    else:
        batch = _batch_shape(list(tree_tensors(all_params)) + list(tree_tensors(all_states)))
        init_states = _expand_states(all_states, batch)
    # One batch shape for everything (integrate.py:570-585): the inputs' batch
    # dimensions broadcast against each other, then flatten to rows.
    batch_shape = tuple(batch)
    if stim_np is not None:
        batch_shape = tuple(np.broadcast_shapes(batch_shape, stim_np.shape[:-2]))
    for _, _, vals in clamps:
        batch_shape = tuple(np.broadcast_shapes(batch_shape, vals.shape[:-2]))
    if stim_np is not None:
        stim_np = _flatten_to(stim_np, batch_shape, core=2)
        if stim_np.ndim == 2:
            stim_np = stim_np[None]
    clamps = [(k, i, _flatten_to(v, batch_shape, core=2) if v.ndim > 2 else v[None]) for k, i, v in clamps]
    plan = module._get_step_plan(device, "jaxley.dhs.gpu", "bwd_euler")
    gathered = module._gather_step_params(plan, all_params)
    if all_states is None:
        init_states = module._append_currents_with_plan(init_states, delta_t, plan, gathered)

    n = int(base._n_nodes)
    indexer = base._dhs_solve_indexer
    channels = []
    for cp in plan["channels"]:
        ch = cp["channel"]
        type_name, spec = spec_for_reference_channel(ch)
        pnames = list(ch.channel_params.keys())
        snames = list(ch.channel_states.keys())
        consts = [float(ch.channel_constants[k]) for k, _ in spec.constants]
        channels.append(
            ChannelInstance(
                type_name=type_name,
                name=ch._name,
                inds=_np(cp["inds"], np.int64),
                params=pnames,
                states=snames,
                current=ch.current_name,
                constants=consts,
            )
        )

    def flat(d):
        out = {}
        for k, v in d.items():
            if isinstance(v, dict):
                continue
            if isinstance(v, torch.Tensor) and v.ndim >= 1 and v.shape[-1] == n:
                out[k] = _flatten_to(_np(v), batch_shape)
        return out

    params_np = flat(all_params)
    states_np = flat(init_states)
    axial = _flatten_to(_np(all_params["axial_conductances"]["v"]), batch_shape)

    synapses = []
    for sp, gp in zip(plan["synapses"], gathered["synapses"]):
        synapses.append(_synapse_from_plan(sp, gp, init_states))

    rec = []
    for idx, name in zip(
        module.recordings.rec_index.to_numpy().astype(int), module.recordings.state.to_numpy()
    ):
        rec.append((str(name), int(idx)))

    batches = [a.shape[0] for a in list(params_np.values()) + list(states_np.values()) if a.ndim == 2]
    if stim_np is not None:
        batches.append(stim_np.shape[0])
    if axial.ndim == 2:
        batches.append(axial.shape[0])
    batches += [c[2].shape[0] for c in clamps]
    B = max(batches) if batches else 1

    # Trainable groups of node parameters, in the order of `params` and its groups,
    # then those of the `param_state` entries whose value requires a gradient (the
    # source index of the latter is len(params) + their position in param_state).
    trainable, source = [], []
    node_keys = set(base.nodes.columns)
    entries = [(list(e.keys())[0], np.asarray(module.indices_set_by_trainables[q]), True, False)
               for q, e in enumerate(params)]
    for ps, (grad, bcast) in zip(param_state or [], ps_grad):
        entries.append((ps["key"], np.asarray(ps["indices"]), grad, bcast))
    for q, (key, inds, grad, bcast) in enumerate(entries):
        if not grad or key not in node_keys or key in GEOMETRY_PARAMS or key not in params_np:
            continue
        inds = inds.reshape(inds.shape[0], -1)
        if bcast and inds.shape[0] > 1:
            # one value broadcast over the view (data_set of a `(..., 1)` value)
            inds = inds.reshape(1, -1)
        for g in range(inds.shape[0]):
            nodes = inds[g][inds[g] >= 0].astype(np.int64)
            trainable.append((key, nodes))
            source.append((q, g))

    prob = Problem(
        n_nodes=n,
        comp_inds=np.asarray(base._internal_node_inds, dtype=np.int64),
        sinks=_np(plan["sinks"], np.int64),
        axial=axial,
        parent_lookup=np.asarray(indexer["parent_lookup"], dtype=np.int64)[:n],
        to_solve=np.asarray(indexer["map_to_solve_order"], dtype=np.int64),
        map_lower=np.asarray(indexer["map_to_solve_order_lower"], dtype=np.int64),
        map_upper=np.asarray(indexer["map_to_solve_order_upper"], dtype=np.int64),
        channels=channels,
        params=params_np,
        states=states_np,
        dt=float(delta_t),
        n_steps=int(n_steps),
        stim_inds=stim_inds,
        stim=stim_np,
        recordings=rec,
        synapses=synapses,
        batch=int(B),
        current_names=list(base.membrane_current_names),
        trainable=trainable,
        clamps=clamps,
        solver=solver,
    )
    prob.trainable_source = source
    prob.batch_shape = batch_shape
    return prob


def _synapse_from_plan(sp, gp, states) -> SynapseType:
    if "k" not in sp:
        raise NotImplementedError("only synapse types in the regular layout are covered")
    syn = sp["synapse"]
    cls = type(syn).__name__
    if cls == "KineticSynapse":
        model = 0
    elif cls == "SigmoidRateSynapse":
        model = 1
    else:
        raise NotImplementedError(f"synapse {cls} has no sm_100a implementation")
    names = list(syn.synapse_params.keys())
    E = int(sp["pre"].shape[0])
    prm = []
    for nm in names:
        v = _np(gp["params"][nm])
        if v.ndim != 1:
            raise NotImplementedError("batched synapse parameters are not covered")
        prm.append(np.broadcast_to(v, (E,)).copy())
    state = None
    if model == 0:
        s = _np(states[f"{syn._name}_s"])
        state = s.reshape(-1, E)
    cur_name = f"i_{syn._name}"
    current = _np(states[cur_name]).reshape(-1, E) if cur_name in states else None
    return SynapseType(
        model=model,
        name=syn._name,
        pre=_np(sp["pre"], np.int64),
        post=_np(sp["post"], np.int64),
        k=int(sp["k"]),
        targets=_np(sp["targets"], np.int64),
        params=prm,
        param_names=names,
        state=state,
        current=current,
    )


# --------------------------------------------------------------------------------------
# Serialization (npz, no pickle): fixtures travel to machines without the reference.
# --------------------------------------------------------------------------------------
def save_problem(problem: Problem, path: str, **extra) -> None:
    import json

    arrays = {
        "comp_inds": problem.comp_inds, "sinks": problem.sinks, "axial": problem.axial,
        "parent_lookup": problem.parent_lookup, "to_solve": problem.to_solve,
        "map_lower": problem.map_lower, "map_upper": problem.map_upper,
        "stim_inds": problem.stim_inds,
    }
    if problem.stim is not None:
        arrays["stim"] = problem.stim
    meta = {
        "n_nodes": problem.n_nodes, "dt": problem.dt, "n_steps": problem.n_steps,
        "batch": problem.batch, "current_names": problem.current_names,
        "recordings": [[n, int(i)] for n, i in problem.recordings],
        "params": list(problem.params), "states": list(problem.states),
        "channels": [], "synapses": [],
        "trainable": [name for name, _ in problem.trainable],
        "solver": problem.solver,
    }
    for q, (_, nodes) in enumerate(problem.trainable):
        arrays[f"trainable/{q}"] = np.asarray(nodes, dtype=np.int64)
    meta["clamps"] = [name for name, _, _ in problem.clamps]
    for q, (_, nodes, vals) in enumerate(problem.clamps):
        arrays[f"clamp/{q}/nodes"] = np.asarray(nodes, dtype=np.int64)
        arrays[f"clamp/{q}/values"] = np.asarray(vals, dtype=np.float64)
    for k, v in problem.params.items():
        arrays[f"param/{k}"] = v
    for k, v in problem.states.items():
        arrays[f"state/{k}"] = v
    for q, ch in enumerate(problem.channels):
        meta["channels"].append({"type": ch.type_name, "name": ch.name, "params": ch.params,
                                 "states": ch.states, "current": ch.current,
                                 "constants": list(ch.constants)})
        arrays[f"channel/{q}"] = np.asarray(ch.inds)
    for q, syn in enumerate(problem.synapses):
        meta["synapses"].append({"model": syn.model, "name": syn.name, "k": syn.k,
                                 "param_names": syn.param_names,
                                 "has_state": syn.state is not None,
                                 "has_current": syn.current is not None})
        arrays[f"syn/{q}/pre"] = syn.pre
        arrays[f"syn/{q}/post"] = syn.post
        arrays[f"syn/{q}/targets"] = syn.targets
        arrays[f"syn/{q}/params"] = np.stack(syn.params)
        if syn.state is not None:
            arrays[f"syn/{q}/state"] = syn.state
        if syn.current is not None:
            arrays[f"syn/{q}/current"] = syn.current
    for k, v in extra.items():
        arrays[f"extra/{k}"] = np.asarray(v)
    arrays["meta"] = np.frombuffer(json.dumps(meta).encode(), dtype=np.uint8)
    np.savez_compressed(path, **arrays)


def load_problem(path: str):
    """Returns `(problem, extra)` where `extra` holds the additional arrays."""
    import json

    from .channels import ChannelInstance

    z = np.load(path, allow_pickle=False)
    meta = json.loads(bytes(z["meta"]).decode())
    channels = [
        ChannelInstance(type_name=c["type"], name=c["name"], inds=z[f"channel/{q}"],
                        params=c["params"], states=c["states"], current=c["current"],
                        constants=c["constants"])
        for q, c in enumerate(meta["channels"])
    ]
    synapses = []
    for q, s in enumerate(meta["synapses"]):
        synapses.append(SynapseType(
            model=s["model"], name=s["name"], pre=z[f"syn/{q}/pre"], post=z[f"syn/{q}/post"],
            k=s["k"], targets=z[f"syn/{q}/targets"], params=list(z[f"syn/{q}/params"]),
            param_names=s["param_names"],
            state=z[f"syn/{q}/state"] if s["has_state"] else None,
            current=z[f"syn/{q}/current"] if s["has_current"] else None,
        ))
    prob = Problem(
        n_nodes=meta["n_nodes"], comp_inds=z["comp_inds"], sinks=z["sinks"], axial=z["axial"],
        parent_lookup=z["parent_lookup"], to_solve=z["to_solve"], map_lower=z["map_lower"],
        map_upper=z["map_upper"], channels=channels,
        params={k: z[f"param/{k}"] for k in meta["params"]},
        states={k: z[f"state/{k}"] for k in meta["states"]},
        dt=meta["dt"], n_steps=meta["n_steps"], stim_inds=z["stim_inds"],
        stim=z["stim"] if "stim" in z else None,
        recordings=[(n, i) for n, i in meta["recordings"]], synapses=synapses,
        batch=meta["batch"], current_names=meta["current_names"],
        trainable=[(n, z[f"trainable/{q}"]) for q, n in enumerate(meta.get("trainable", []))],
        clamps=[(n, z[f"clamp/{q}/nodes"], z[f"clamp/{q}/values"]) for q, n in enumerate(meta.get("clamps", []))],
        solver=meta.get("solver", "bwd_euler"),
    )
    extra = {k[len("extra/"):]: z[k] for k in z.files if k.startswith("extra/")}
    return prob, extra
