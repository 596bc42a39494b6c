"""Fixed in-degree synapse step on sm_100a: the drop-in for jaxley-pytorch's
`kernels/synapse_step.py`.

Same public surface as the reference module (`synapse_step.py:43-498`): `KINETIC`,
`SIGMOID_RATE`, `kernel_plan(synapse_type, pre, targets, n_nodes, device)`,
`kernel_scalars(delta_t, diff, dtype, device)`, the custom ops `synapse_step` and
`synapse_step_backward` with the reference's argument lists and autograd, and
`fused_step(states, delta_t, sp, gp)`. The kernels are `jxb_synapse_forward` /
`jxb_synapse_backward` of libjxb: warp reductions over the k synapses of a target
(forward), batch-sliced warps with a fixed-order reduction of the parameter
gradients and the transposed index for the presynaptic voltages (backward) — no
atomics at any width. `JAXLEY_PYTORCH_SYNAPSE_KERNEL=off` disables the plan (then
the caller runs its own code, as in the reference).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, Optional

import numpy as np
import torch

from .. import _lib

KINETIC, SIGMOID_RATE = 0, 1
_NAMES = {
    KINETIC: ("gS", "e_syn", "alpha", "beta", "v_th", "delta"),
    SIGMOID_RATE: ("gS", "x_offset", "slope"),
}


def _model_of(synapse_type) -> Optional[int]:
    m = getattr(synapse_type, "model", None)
    if isinstance(m, int):
        return m
    cls = type(synapse_type).__name__
    return {"KineticSynapse": KINETIC, "SigmoidRateSynapse": SIGMOID_RATE}.get(cls)


def _transposed_index(pre: np.ndarray):
    """`(nodes, inv)`: the presynaptic nodes (sorted) and, as `(len(nodes), width)`
    int32, the synapses of every presynaptic node padded with -1
    (`synapse_step.py:66-76`)."""
    nodes, local = np.unique(pre, return_inverse=True)
    counts = np.bincount(local, minlength=len(nodes))
    order = np.argsort(local, kind="stable")
    starts = np.r_[0, np.cumsum(counts)[:-1]]
    rows = local[order]
    inv = np.full((len(nodes), max(int(counts.max()), 1)), -1, dtype=np.int32)
    inv[rows, np.arange(len(pre)) - starts[rows]] = order
    return nodes.astype(np.int32), inv


def kernel_plan(synapse_type, pre: np.ndarray, targets: np.ndarray, n_nodes: int, device) -> Dict:
    """Plan entries of the kernels (empty when they do not apply, `synapse_step.py:79-103`)."""
    if torch.device(device).type != "cuda" or os.environ.get("JAXLEY_PYTORCH_SYNAPSE_KERNEL", "auto") == "off":
        return {}
    model = _model_of(synapse_type)
    if model is None:
        return {}
    name = getattr(synapse_type, "_name", None) or getattr(synapse_type, "name")
    pre = np.asarray(pre)
    nodes, inv = _transposed_index(pre)
    return {
        "kernel_model": model,
        "kernel_params": [f"{name}_{p}" for p in _NAMES[model]],
        "kernel_pre": torch.as_tensor(pre.astype(np.int32), device=device),
        "kernel_targets": torch.as_tensor(np.asarray(targets).astype(np.int32), device=device),
        "kernel_pre_nodes": torch.as_tensor(nodes, device=device),
        "kernel_inv": torch.as_tensor(inv, device=device),
    }


def kernel_scalars(delta_t: float, diff: float, dtype, device) -> torch.Tensor:
    """`[delta_t, diff]` filled on the device (no host-to-device copy, capturable)."""
    scalars = torch.full((2,), diff, dtype=dtype, device=device)
    scalars[:1].fill_(delta_t)
    return scalars


def _code(t):
    return _lib.F32 if t.dtype == torch.float32 else _lib.F64


def _args(v, s, pre, targets, params, area, scalars, k, model, targets_are_nodes):
    a = _lib.JxbSynArgs()
    a.dtype = _code(v)
    a.model = model
    a.batch, a.n_nodes = v.shape
    a.n_syn = pre.shape[0]
    a.k = k
    a.targets_are_nodes = int(targets_are_nodes)
    a.v = v.data_ptr()
    a.s = s.data_ptr() if (model == KINETIC and s.numel()) else None
    a.pre = pre.data_ptr()
    a.targets = targets.data_ptr()
    for q, p in enumerate(params):
        a.p[q] = p.data_ptr()
    a.area = area.data_ptr()
    a.scalars = scalars.data_ptr()
    return a


def _stream(t):
    return C.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def _forward(v, s, pre, targets, p0, p1, p2, p3, p4, p5, area, scalars, inv, pre_nodes, k, model,
             targets_are_nodes, store_current):
    B, n = v.shape
    E = pre.shape[0]
    T = E // k
    v = v.contiguous()
    params = [p.to(v.dtype).contiguous() for p in (p0, p1, p2, p3, p4, p5)]
    area = area.to(v.dtype).contiguous()
    kinetic = model == KINETIC
    s = s.to(v.dtype).contiguous() if kinetic else v.new_empty(0)
    s_new = torch.empty_like(s) if kinetic else v.new_empty(0)
    current = v.new_empty(B, E) if store_current else v.new_empty(0)
    lin = v.new_empty(B, T)
    const = v.new_empty(B, T)
    a = _args(v, s, pre, targets, params, area, scalars.to(v.dtype), k, model, targets_are_nodes)
    a.store_current = int(store_current)
    a.s_new = s_new.data_ptr() if kinetic else None
    a.current = current.data_ptr() if store_current else None
    a.lin = lin.data_ptr()
    a.cst = const.data_ptr()
    _lib.check(_lib.load().jxb_synapse_forward(C.byref(a), _stream(v)), "jxb_synapse_forward")
    return s_new, current, lin, const


def _backward(v, s, pre, targets, p0, p1, p2, p3, p4, p5, area, scalars, inv, pre_nodes, g_s_new,
              g_current, g_lin, g_const, k, model, targets_are_nodes, has_g_s_new, has_g_current, need):
    B, n = v.shape
    E = pre.shape[0]
    T = E // k
    v = v.contiguous()
    params = [p.to(v.dtype).contiguous() for p in (p0, p1, p2, p3, p4, p5)]
    area = area.to(v.dtype).contiguous()
    kinetic = model == KINETIC
    s = s.to(v.dtype).contiguous() if kinetic else v.new_empty(0)
    g_s = torch.empty_like(s) if kinetic else v.new_empty(0)
    n_need = bin(need).count("1")
    g_params = v.new_empty(n_need, E)
    g_v = torch.empty_like(v)
    g_pre = v.new_empty(E, B)
    g_post = v.new_empty(B, T)
    a = _args(v, s, pre, targets, params, area, scalars.to(v.dtype), k, model, targets_are_nodes)
    gsn = g_s_new.to(v.dtype).contiguous() if has_g_s_new else None
    gcu = g_current.to(v.dtype).contiguous() if has_g_current else None
    gl = g_lin.to(v.dtype).contiguous()
    gc = g_const.to(v.dtype).contiguous()
    a.g_s_new = gsn.data_ptr() if gsn is not None else None
    a.g_current = gcu.data_ptr() if gcu is not None else None
    a.g_lin = gl.data_ptr()
    a.g_const = gc.data_ptr()
    a.g_s = g_s.data_ptr() if kinetic else None
    a.g_v = g_v.data_ptr()
    a.g_params = g_params.data_ptr() if n_need else None
    a.g_pre = g_pre.data_ptr()
    a.g_post = g_post.data_ptr()
    a.need = need
    a.inv_width = inv.shape[1]
    a.n_pre_nodes = pre_nodes.shape[0]
    a.inv = inv.data_ptr()
    a.pre_nodes = pre_nodes.data_ptr()
    _lib.check(_lib.load().jxb_synapse_backward(C.byref(a), _stream(v)), "jxb_synapse_backward")
    return g_v, g_s, g_params


synapse_step_op = None
synapse_step_backward_op = None


def _define_in(ns: str):
    global synapse_step_op, synapse_step_backward_op

    @torch.library.custom_op(f"{ns}::synapse_step", mutates_args=())
    def _op(v: torch.Tensor, s: torch.Tensor, pre: torch.Tensor, targets: torch.Tensor,
            p0: torch.Tensor, p1: torch.Tensor, p2: torch.Tensor, p3: torch.Tensor,
            p4: torch.Tensor, p5: torch.Tensor, area: torch.Tensor, scalars: torch.Tensor,
            inv: torch.Tensor, pre_nodes: torch.Tensor, k: int, model: int,
            targets_are_nodes: bool, store_current: bool
            ) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor, torch.Tensor]:
        """`(states, current, slope, offset)` of one synapse type
        (reference `synapse_step.py:336-363`)."""
        return _forward(v, s, pre, targets, p0, p1, p2, p3, p4, p5, area, scalars, inv,
                        pre_nodes, k, model, targets_are_nodes, store_current)

    @_op.register_fake
    def _(v, s, pre, targets, p0, p1, p2, p3, p4, p5, area, scalars, inv, pre_nodes, k, model,
          targets_are_nodes, store_current):
        B, E = v.shape[0], pre.shape[0]
        s_new = torch.empty_like(s) if model == KINETIC else v.new_empty(0)
        cur = v.new_empty(B, E) if store_current else v.new_empty(0)
        return s_new, cur, v.new_empty(B, E // k), v.new_empty(B, E // k)

    @torch.library.custom_op(f"{ns}::synapse_step_backward", mutates_args=())
    def _bop(v: torch.Tensor, s: torch.Tensor, pre: torch.Tensor, targets: torch.Tensor,
             p0: torch.Tensor, p1: torch.Tensor, p2: torch.Tensor, p3: torch.Tensor,
             p4: torch.Tensor, p5: torch.Tensor, area: torch.Tensor, scalars: torch.Tensor,
             inv: torch.Tensor, pre_nodes: torch.Tensor, g_s_new: torch.Tensor,
             g_current: torch.Tensor, g_lin: torch.Tensor, g_const: torch.Tensor, k: int,
             model: int, targets_are_nodes: bool, has_g_s_new: bool, has_g_current: bool,
             need: int) -> tuple[torch.Tensor, torch.Tensor, torch.Tensor]:
        """Gradients of `v`, of the states and of the parameters in `need`
        (reference `synapse_step.py:372-416`)."""
        return _backward(v, s, pre, targets, p0, p1, p2, p3, p4, p5, area, scalars, inv,
                         pre_nodes, g_s_new, g_current, g_lin, g_const, k, model,
                         targets_are_nodes, has_g_s_new, has_g_current, need)

    @_bop.register_fake
    def _(v, s, pre, targets, p0, p1, p2, p3, p4, p5, area, scalars, inv, pre_nodes, g_s_new,
          g_current, g_lin, g_const, k, model, targets_are_nodes, has_g_s_new, has_g_current, need):
        g_s = torch.empty_like(s) if model == KINETIC else v.new_empty(0)
        return torch.empty_like(v), g_s, v.new_empty(bin(need).count("1"), pre.shape[0])

    def _setup(ctx, inputs, output):
        (v, s, pre, targets, p0, p1, p2, p3, p4, p5, area, scalars, inv, nodes, k, model, tan,
         store) = inputs
        ctx.save_for_backward(v, s, pre, targets, p0, p1, p2, p3, p4, p5, area, scalars, inv, nodes)
        ctx.k, ctx.model, ctx.tan = k, model, tan

    def _bw(ctx, g_s_new, g_current, g_lin, g_const):
        v, s, pre, targets, p0, p1, p2, p3, p4, p5, area, scalars, inv, nodes = ctx.saved_tensors
        n_params = 6 if ctx.model == KINETIC else 3
        need = sum(1 << i for i in range(n_params) if ctx.needs_input_grad[4 + i])
        B, T = v.shape[0], pre.shape[0] // ctx.k
        empty = v.new_empty(0)
        has_gs = ctx.model == KINETIC and g_s_new is not None
        has_gc = g_current is not None and g_current.numel() > 0
        g_lin = g_lin.contiguous() if g_lin is not None else v.new_zeros(B, T)
        g_const = g_const.contiguous() if g_const is not None else v.new_zeros(B, T)
        g_v, g_s, g_params = _bop(v, s, pre, targets, p0, p1, p2, p3, p4, p5, area, scalars, inv,
                                  nodes, g_s_new.contiguous() if has_gs else empty,
                                  g_current.contiguous() if has_gc else empty, g_lin, g_const,
                                  ctx.k, ctx.model, ctx.tan, has_gs, has_gc, need)
        rows = [bin(need & ((1 << i) - 1)).count("1") for i in range(6)]
        g_p = [g_params[rows[i]] if need & (1 << i) else None for i in range(6)]
        return (g_v, g_s if ctx.model == KINETIC else None, None, None, *g_p) + (None,) * 8

    _op.register_autograd(_bw, setup_context=_setup)
    synapse_step_op = _op
    synapse_step_backward_op = _bop


def _ensure_ops():
    if synapse_step_op is not None:
        return
    for ns in ("jaxley_pytorch", "jaxley_pytorch_b200"):
        try:
            _define_in(ns)
            return
        except RuntimeError:
            continue
    raise RuntimeError("could not register the synapse ops")


def fused_step(states: Dict, delta_t: float, sp: Dict, gp: Dict) -> Optional[tuple]:
    """`Network._step_regular_synapses` with the fused kernels
    (reference `synapse_step.py:451-498`): returns `(states, (lin, -const))` on the
    nodes, or `None` when the plan has no kernel entries."""
    if "kernel_model" not in sp or "kernel_scalars" not in gp:
        return None
    _ensure_ops()
    v = states["v"]
    model = sp["kernel_model"]
    num_targets, k = sp["pre_per_target"].shape
    num_syn = num_targets * k
    params = [gp["params"][name] for name in sp["kernel_params"]]
    area = gp["area_post"]
    params = [torch.broadcast_to(torch.as_tensor(p, dtype=v.dtype, device=v.device), (num_syn,))
              for p in params]
    params += [params[0]] * (6 - len(params))
    batch, n = v.shape[:-1], v.shape[-1]
    name = sp["synapse_name"] if "synapse_name" in sp else sp["synapse"]._name
    state = f"{name}_s"
    if model == KINETIC:
        s = states[state].reshape(-1, num_syn).contiguous()
    else:
        s = v.new_empty(0)
    store = gp.get("store_current", True)
    s_new, current, lin, const = synapse_step_op(
        v.reshape(-1, n).contiguous(), s, sp["kernel_pre"], sp["kernel_targets"], *params,
        torch.broadcast_to(area, (num_syn,)).to(v.dtype).contiguous(), gp["kernel_scalars"],
        sp["kernel_inv"], sp["kernel_pre_nodes"], k, model, sp["targets_are_nodes"], store,
    )
    states = dict(states)
    if model == KINETIC:
        states[state] = s_new.reshape(*batch, num_syn)
    if store:
        states[f"i_{name}"] = current.reshape(*batch, num_syn)
    lin = lin.reshape(*batch, lin.shape[-1])
    const = const.reshape(*batch, const.shape[-1])
    if sp["targets_are_nodes"]:
        return states, (lin, -const)
    zeros = torch.zeros_like(v)
    targets = sp["targets"]
    return states, (zeros.index_add(-1, targets, lin), zeros.index_add(-1, targets, -const))
