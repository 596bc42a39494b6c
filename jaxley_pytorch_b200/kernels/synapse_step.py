"""Fixed in-degree synapse step on sm_100a: the drop-in for jaxley-pytorch's
`kernels/synapse_step.py`.

Same public surface as the reference module (`synapse_step.py:43-498`): `KINETIC`,
`SIGMOID_RATE`, `kernel_plan(synapse_type, pre, targets, n_nodes, device)`,
`kernel_scalars(delta_t, diff, dtype, device)`, the custom ops `synapse_step` and
`synapse_step_backward` with the reference's argument lists and autograd
(registered as `jaxley_pytorch_b200::synapse_step[_backward]`, beside the
reference's own ops), and `fused_step(states, delta_t, sp, gp)`. The kernels are
`jxb_synapse_forward` / `jxb_synapse_backward` of libjxb: lane groups per (row,
target) with shuffle sums over the target's synapses, a fixed-order reduction of
the parameter gradients over the batch and the transposed index for the
presynaptic voltages — no atomics at any width. `JAXLEY_PYTORCH_SYNAPSE_KERNEL=off`
disables the plan (then the caller runs its own code, as in the reference).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Dict, Optional

import numpy as np
import torch

from .. import _lib
from ..lower import presynaptic_lists
from . import OP_NAMESPACE

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


def kernel_plan(synapse_type, pre: np.ndarray, targets: np.ndarray, n_nodes: int, device) -> Dict:
    """Plan entries of the kernels (empty when they do not apply, `synapse_step.py:79-103`)."""
    if torch.device(device).type != "cuda" or os.environ.get("JAXLEY_PYTORCH_SYNAPSE_KERNEL", "auto") == "off":
        return {}
    model = _model_of(synapse_type)
    if model is None:
        return {}
    name = getattr(synapse_type, "_name", None) or getattr(synapse_type, "name")
    pre = np.asarray(pre)
    nodes, inv = presynaptic_lists(pre)
    return {
        "kernel_model": model,
        "kernel_params": [f"{name}_{p}" for p in _NAMES[model]],
        "kernel_pre": torch.as_tensor(pre.astype(np.int32), device=device),
        "kernel_targets": torch.as_tensor(np.asarray(targets).astype(np.int32), device=device),
        "kernel_pre_nodes": torch.as_tensor(nodes, device=device),
        "kernel_inv": torch.as_tensor(inv, device=device),
    }


def kernel_scalars(delta_t: float, diff: float, dtype, device) -> torch.Tensor:
    """`[delta_t, diff]` as a device tensor. Each value is written by a fill on the
    device and the two are stacked there, so no host-to-device copy is issued and
    the call can run inside a CUDA-graph capture."""
    dt_t = torch.full((), float(delta_t), dtype=dtype, device=device)
    diff_t = torch.full((), float(diff), dtype=dtype, device=device)
    return torch.stack((dt_t, diff_t))


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

    # Autograd of the forward op: the 18 inputs are (v, s, pre, targets, p0..p5,
    # area, scalars, inv, pre_nodes, k, model, targets_are_nodes, store_current);
    # gradients flow to v, to the kinetic state and to the parameters that ask for
    # them, whose rows the backward op returns in parameter order.
    n_inputs = 18

    def _save(ctx, inputs, output):
        ctx.save_for_backward(*inputs[:14])
        ctx.k, ctx.model, ctx.tan = inputs[14], inputs[15], inputs[16]

    def _grad(ctx, g_s_new, g_current, g_lin, g_const):
        saved = ctx.saved_tensors
        v, pre = saved[0], saved[2]
        kinetic = ctx.model == KINETIC
        wanted = [q for q in range(len(_NAMES[ctx.model])) if ctx.needs_input_grad[4 + q]]
        need = 0
        for q in wanted:
            need |= 1 << q
        shape_post = (v.shape[0], pre.shape[0] // ctx.k)
        none = v.new_empty(0)
        use_s = kinetic and g_s_new is not None
        use_cur = g_current is not None and g_current.numel() > 0
        g_v, g_s, g_rows = _bop(
            *saved,
            g_s_new.contiguous() if use_s else none,
            g_current.contiguous() if use_cur else none,
            v.new_zeros(shape_post) if g_lin is None else g_lin.contiguous(),
            v.new_zeros(shape_post) if g_const is None else g_const.contiguous(),
            ctx.k, ctx.model, ctx.tan, use_s, use_cur, need)
        grads = [None] * n_inputs
        grads[0] = g_v
        if kinetic:
            grads[1] = g_s
        for row, q in enumerate(wanted):
            grads[4 + q] = g_rows[row]
        return tuple(grads)

    _op.register_autograd(_grad, setup_context=_save)
    synapse_step_op = _op
    synapse_step_backward_op = _bop


def _ensure_ops():
    if synapse_step_op is not None:
        return
    _define_in(OP_NAMESPACE)


def _scatter_to_nodes(per_target: torch.Tensor, targets: torch.Tensor, n: int) -> torch.Tensor:
    """`(rows, n)` node array holding `per_target (rows, T)` at the target nodes and
    zero elsewhere (the regular layout has distinct targets)."""
    out = per_target.new_zeros(per_target.shape[0], n)
    idx = targets.to(torch.long).reshape(1, -1).expand(per_target.shape[0], -1)
    return out.scatter_add_(1, idx, per_target)


def fused_step(states: Dict, delta_t: float, sp: Dict, gp: Dict) -> Optional[tuple]:
    """`Network._step_regular_synapses` on the CUDA kernels (the reference's entry,
    `kernels/synapse_step.py:451-498`, called at `modules/network.py:402-407`).

    Returns `(states, (slope, offset))` with node arrays of the synapse type's
    summed slope and offset (the offset with the sign the caller adds), or `None`
    when the kernels do not apply: no kernel entries in the plan, voltages not on a
    CUDA device or not float32/float64, parameters or areas that are not one value
    per synapse on that device, a trainable area, or a kinetic state of another
    shape. The caller then runs its own code, as with the reference."""
    if "kernel_model" not in sp or "kernel_scalars" not in gp:
        return None
    v = states["v"]
    if not v.is_cuda or v.dtype not in (torch.float32, torch.float64) or v.dim() == 0:
        return None
    model = sp["kernel_model"]
    n_targets, k = sp["pre_per_target"].shape
    E = n_targets * k
    per_syn = [gp["params"][name] for name in sp["kernel_params"]] + [gp["area_post"]]
    for p in per_syn:
        if not isinstance(p, torch.Tensor) or tuple(p.shape) != (E,) or p.device != v.device:
            return None
    if gp["area_post"].requires_grad:
        return None
    lead, n = tuple(v.shape[:-1]), v.shape[-1]
    name = sp["synapse"]._name if "synapse" in sp else sp["synapse_name"]
    state_key, current_key = f"{name}_s", f"i_{name}"
    if model == KINETIC:
        s = states[state_key]
        if tuple(s.shape) != lead + (E,):
            return None
        s = s.reshape(-1, E).contiguous()
    else:
        s = v.new_empty(0)
    _ensure_ops()
    cast = [p.to(v.dtype).contiguous() for p in per_syn]
    area = cast.pop()
    six = cast + [cast[0]] * (6 - len(cast))  # unused slots of SigmoidRateSynapse
    keep_current = bool(gp.get("store_current", True))
    s_new, current, slope, offset = synapse_step_op(
        v.reshape(-1, n).contiguous(), s, sp["kernel_pre"], sp["kernel_targets"], *six, area,
        gp["kernel_scalars"], sp["kernel_inv"], sp["kernel_pre_nodes"], k, model,
        sp["targets_are_nodes"], keep_current)
    new_states = {**states}
    if model == KINETIC:
        new_states[state_key] = s_new.view(lead + (E,))
    if keep_current:
        new_states[current_key] = current.view(lead + (E,))
    if not sp["targets_are_nodes"]:
        slope = _scatter_to_nodes(slope, sp["targets"], n)
        offset = _scatter_to_nodes(offset, sp["targets"], n)
    return new_states, (slope.view(lead + (slope.shape[-1],)), -offset.view(lead + (offset.shape[-1],)))
