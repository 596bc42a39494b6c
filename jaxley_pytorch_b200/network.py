"""Networks: the synapse step fused into the simulation loop, with its adjoint.

Every step of `jx.integrate` on a network (`modules/network.py:350-478`) runs the
synapse pass of every synapse type on the voltages before the step (kinetic states
advance), adds each target's summed slope and offset to its linear and constant
terms, and then takes the cell step. Here a step is one `jxb_synapse_forward` launch
per synapse type, reading the voltages straight from the simulation's state vector
(the presynaptic and postsynaptic indices are state-slot offsets), and one
one-step `jxb_sim_forward` launch that adds the synaptic terms by target
(`JxbSimArgs.syn_ptr`). The whole loop is graph-capturable.

The adjoint runs segments of `checkpoint` steps in reverse. The forward stores the
cell state before every step and the kinetic states every `checkpoint` steps; a
segment first recomputes its kinetic states and synaptic terms, then, step by step
in reverse: the one-step cell adjoint (`jxb_sim_backward`, which also returns the
gradient of the step's synaptic slopes and offsets), the synapse adjoint of every
type (`jxb_synapse_backward`: voltage gradient in the state layout, kinetic-state
gradient, parameter gradients summed over the batch), and the voltage gradient added
to the state adjoint.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from .kernels.synapse_step import KINETIC
from .lower import presynaptic_lists
from .problem import Problem, SynapseType
from .sim import Simulation

DIFF = 1e-3  # finite-difference step of the synaptic current slope (modules/network.py:434-478)


class _SynType:
    """Device plan of one synapse type in the regular layout."""

    def __init__(self, syn: SynapseType, low, area: np.ndarray, B: int, dtype, device, dt: float):
        self.model = int(syn.model)
        self.k = int(syn.k)
        self.E = len(syn.pre)
        self.T = self.E // self.k
        soff = np.asarray(low.soff, dtype=np.int64)
        n2i = np.asarray(low.node2int, dtype=np.int64)
        pre_slot = soff[n2i[np.asarray(syn.pre, dtype=np.int64)]].astype(np.int32)
        tgt_slot = soff[n2i[np.asarray(syn.targets, dtype=np.int64)]].astype(np.int32)
        nodes, inv = presynaptic_lists(pre_slot)
        i32 = lambda x: torch.as_tensor(np.ascontiguousarray(x), dtype=torch.int32, device=device)  # noqa: E731
        self.pre = i32(pre_slot)
        self.targets = i32(tgt_slot)
        self.pre_nodes = i32(nodes)
        self.inv = i32(inv)
        self.target_int = n2i[np.asarray(syn.targets, dtype=np.int64)]  # internal node of every target
        self.params = [torch.as_tensor(np.asarray(p, dtype=np.float64), dtype=dtype, device=device).contiguous()
                       for p in syn.params]
        self.param_names = list(syn.param_names)
        self.area = torch.as_tensor(np.asarray(area, dtype=np.float64)[np.asarray(syn.post)], dtype=dtype,
                                    device=device).contiguous()
        self.scalars = torch.tensor([dt, DIFF], dtype=dtype, device=device)
        self.kinetic = self.model == KINETIC
        if self.kinetic:
            # row-major (B, E): np.array of a broadcast view would keep its axis order
            s0 = np.broadcast_to(np.asarray(syn.state, dtype=np.float64), (B, self.E)).copy(order="C")
            self.s0 = torch.as_tensor(s0, dtype=dtype, device=device).contiguous()
        self.dtype = dtype

    def args(self, state: torch.Tensor, n_slots: int, B: int, params: Sequence[torch.Tensor]):
        a = _lib.JxbSynArgs()
        a.dtype = _lib.F32 if self.dtype == torch.float32 else _lib.F64
        a.model = self.model
        a.batch, a.n_nodes = B, n_slots
        a.n_syn = self.E
        a.k = self.k
        a.targets_are_nodes = 0
        a.v = _ptr(state, self.dtype, B * n_slots, "state")
        a.pre = self.pre.data_ptr()
        a.targets = self.targets.data_ptr()
        for q, p in enumerate(params):
            a.p[q] = _ptr(p, self.dtype, self.E, self.param_names[q] if q < len(self.param_names) else "param")
        a.area = self.area.data_ptr()
        a.scalars = self.scalars.data_ptr()
        a.inv_width = self.inv.shape[1]
        a.n_pre_nodes = self.pre_nodes.shape[0]
        a.inv = self.inv.data_ptr()
        a.pre_nodes = self.pre_nodes.data_ptr()
        return a


def _ptr(t: torch.Tensor, dtype, numel: int, what: str) -> int:
    """Device address of a row-major tensor the kernels index flat; anything else
    (another dtype, a transposed or strided view, a wrong size) is refused."""
    if t.dtype != dtype or not t.is_contiguous() or t.numel() != numel:
        raise ValueError(f"{what}: expected a contiguous {dtype} tensor of {numel} elements, got "
                         f"{t.dtype} {tuple(t.shape)} with strides {t.stride()}")
    return t.data_ptr()


def _stream():
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


class NetworkSimulation:
    """`jx.integrate` for a `Problem` with synapses (regular layout) on the CUDA
    kernels. `run(pscale, syn_params)` returns the recordings `(B, n_rec, T + 1)`,
    differentiable with respect to the cell parameter scales and the synapse
    parameters (lists of `(E,)` tensors per synapse type, in the reference order)."""

    def __init__(self, problem: Problem, dtype=torch.float32, device="cuda", checkpoint: int = 50,
                 threads: int = 256, max_block_nodes: int = 256, rows_per_item: int = 1,
                 init_steady: bool = False, store_trajectory="auto", store_fraction: float = 0.5):
        if not problem.synapses:
            raise ValueError("the problem has no synapses (use Simulation)")
        self.problem = problem
        self.sim = Simulation(problem, dtype=dtype, device=device, threads=threads, segment=1,
                              checkpoint=1, keep_currents=False, max_block_nodes=max_block_nodes,
                              rows_per_item=rows_per_item)
        self.low = low = self.sim.low
        self.model = self.sim.model
        # A float32 cell step of up to 256 threads whose work items fit in one wave at
        # two CTAs per SM runs on the kernels of two CTAs per SM with up to 128
        # registers, forward and adjoint (measured on B200: point-neuron networks of
        # 2048 cells x 32 rows, 256 items, 0.7 % faster each; 2048 four-compartment
        # cells, 1024 items, 6 % slower with the forward on them).
        dev = torch.device(device)
        if dtype == torch.float32 and threads <= 256 and dev.type == "cuda" and torch.cuda.is_available():
            sms = torch.cuda.get_device_properties(dev).multi_processor_count
            one_wave = self.model.n_items <= 2 * sms
            self.model.forward_wide = self.model.backward_wide = one_wave
        self.init_steady = bool(init_steady)  # channel gates start at their steady state
        self.dtype, self.device = dtype, torch.device(device)
        self.B = low.batch
        self.checkpoint = int(checkpoint)
        area = np.asarray(problem.params["area"], dtype=np.float64)
        if area.ndim == 2:
            area = area[0]
        self.types = [_SynType(s, low, area, self.B, dtype, device, low.dt) for s in problem.synapses]
        # per-target CSR over internal nodes into the concatenated per-type outputs
        offs, entries = 0, []
        self.region = []
        for ty in self.types:
            self.region.append((offs, self.B * ty.T))
            for t in range(ty.T):
                entries.append((int(ty.target_int[t]), offs + t, ty.T))
            offs += self.B * ty.T
        self.syn_size = offs
        entries.sort(key=lambda e: e[0])
        n = low.n_nodes
        ptr = np.zeros(n + 1, dtype=np.int32)
        ptr[1:] = np.cumsum(np.bincount([e[0] for e in entries], minlength=n))
        i32 = lambda x: torch.as_tensor(np.asarray(x, dtype=np.int32), device=device).contiguous()  # noqa: E731
        self.syn_ptr = i32(ptr)
        self.syn_off = i32([e[1] for e in entries] or [0])
        self.syn_rs = i32([e[2] for e in entries] or [1])
        self.syn_launches = 0  # synapse kernel launches issued (forward and adjoint)
        # With a stored trajectory the differentiable forward keeps every step's
        # kinetic states and synaptic slopes and offsets, and the adjoint reads them
        # instead of recomputing each checkpoint segment ("auto": when they take at
        # most `store_fraction` of the free device memory).
        if store_trajectory not in (True, False, "auto"):
            raise ValueError("store_trajectory must be True, False or 'auto'")
        self.store_trajectory = store_trajectory
        self.store_fraction = float(store_fraction)
        self._store_free: Optional[int] = None

    def trajectory_bytes(self, T: int) -> int:
        """Device bytes of the synapse trajectory of T steps (states and slopes)."""
        item = torch.empty((), dtype=self.dtype).element_size()
        states = sum((T + 1) * self.B * ty.E for ty in self.types if ty.kinetic)
        return (states + 2 * T * self.syn_size) * item

    def stores_trajectory(self, T: int) -> bool:
        if self.store_trajectory != "auto":
            return bool(self.store_trajectory)
        if self._store_free is None:  # sampled once, outside any graph capture
            if torch.cuda.is_current_stream_capturing():
                return False
            self._store_free = torch.cuda.mem_get_info(self.device)[0]
        return self.trajectory_bytes(T) <= self.store_fraction * self._store_free

    def _zeros(self, *shape, dtype=None):
        return torch.zeros(shape, dtype=dtype or self.dtype, device=self.device)

    def _set_syn(self, a, lin, cst):
        a.syn_lin = lin.data_ptr()
        a.syn_const = cst.data_ptr()
        a.syn_ptr = self.syn_ptr.data_ptr()
        a.syn_off = self.syn_off.data_ptr()
        a.syn_rs = self.syn_rs.data_ptr()

    def _syn_forward(self, ty: _SynType, k: int, state, s, s_new, lin, cst, params):
        a = ty.args(state, self.low.n_slots, self.B, params)
        a.s = _ptr(s, self.dtype, self.B * ty.E, "s") if ty.kinetic else None
        a.s_new = _ptr(s_new, self.dtype, self.B * ty.E, "s_new") if ty.kinetic else None
        a.store_current = 0
        off, size = self.region[k]
        a.lin = lin.data_ptr() + off * lin.element_size()
        a.cst = cst.data_ptr() + off * cst.element_size()
        _lib.check(_lib.load().jxb_synapse_forward(C.byref(a), _stream()), "jxb_synapse_forward")
        self.syn_launches += 1

    def forward_raw(self, pscale: torch.Tensor, syn_params: List[List[torch.Tensor]], T: int,
                    keep: bool = False):
        """Runs T steps; with `keep` also stores what the adjoint needs. Returns
        `(rec (T + 1, B, n_rec), saved)`."""
        m, low, B = self.model, self.low, self.B
        state = m.initial_state()
        rec = self._zeros(T + 1, B, low.n_rec)
        m.launch_forward(m.args(state, 0, 0, rec, mode=2 if self.init_steady else 1, pscale=pscale))
        K = self.checkpoint
        stored = keep and self.stores_trajectory(T)
        saved = None
        if keep:
            # every step's state (before it, and after the last) and the reciprocal
            # pivots of its solve: the one-step adjoint launches read them instead of
            # recomputing the step
            saved = {"states": self._zeros(T + 1, B, low.n_slots), "piv": self._zeros(T, B, low.n_nodes),
                     "stored": stored}
            if stored:  # every step's kinetic states, slopes and offsets
                saved["s_traj"] = [self._zeros(T + 1, B, ty.E) if ty.kinetic else None for ty in self.types]
                saved["lin"] = self._zeros(T, self.syn_size)
                saved["cst"] = self._zeros(T, self.syn_size)
                for q, ty in enumerate(self.types):
                    if ty.kinetic:
                        saved["s_traj"][q][0].copy_(ty.s0)
            else:
                saved["s_ckpt"] = [self._zeros((T + K - 1) // K, B, ty.E) if ty.kinetic else None
                                   for ty in self.types]
        if not stored:
            lin = self._zeros(self.syn_size)
            cst = self._zeros(self.syn_size)
            s_cur = [ty.s0.clone() if ty.kinetic else None for ty in self.types]
            s_nxt = [torch.empty_like(s) if s is not None else None for s in s_cur]
        for t in range(T):
            if stored:
                lin, cst = saved["lin"][t], saved["cst"][t]
                s_cur = [st[t] if st is not None else None for st in saved["s_traj"]]
                s_nxt = [st[t + 1] if st is not None else None for st in saved["s_traj"]]
            elif keep and t % K == 0:
                for q, ty in enumerate(self.types):
                    if ty.kinetic:
                        saved["s_ckpt"][q][t // K].copy_(s_cur[q])
            for q, ty in enumerate(self.types):
                self._syn_forward(ty, q, state, s_cur[q], s_nxt[q], lin, cst, syn_params[q])
            a = m.args(state, 1, t, rec, pscale=pscale, traj=saved["states"][t] if keep else None)
            if keep:
                a.traj_piv = saved["piv"][t].data_ptr()
            self._set_syn(a, lin, cst)
            m.launch_forward(a)
            if not stored:
                s_cur, s_nxt = s_nxt, s_cur
        return rec, saved

    def backward_raw(self, pscale, syn_params, T: int, saved, rec_grad: torch.Tensor,
                     need: Optional[List[int]] = None):
        """Returns `(d loss / d pscale (B, n_cols) float64, [per type: (n_params, E)])`.
        `need` (per type, a bit mask of its parameters; default all) selects the
        parameter gradients the synapse adjoint computes; the others are zero."""
        m, low, B = self.model, self.low, self.B
        K = self.checkpoint
        adj = self._zeros(B, low.n_slots)
        pgrad = self._zeros(B, low.n_cols, dtype=torch.float64)
        if not saved["stored"]:
            LC_lin = self._zeros(K, self.syn_size)
            LC_cst = self._zeros(K, self.syn_size)
            s_seg = [self._zeros(K + 1, B, ty.E) if ty.kinetic else None for ty in self.types]
        g_lin = self._zeros(self.syn_size)
        g_cst = self._zeros(self.syn_size)
        g_s = [self._zeros(B, ty.E) if ty.kinetic else None for ty in self.types]
        g_s2 = [self._zeros(B, ty.E) if ty.kinetic else None for ty in self.types]
        g_pre = [self._zeros(ty.E, B) for ty in self.types]
        n_par = [len(p) for p in syn_params]
        # the synapse adjoint adds every step's parameter gradients here and its
        # voltage gradients straight into the state adjoint (accumulate mode)
        if need is None:
            need = [(1 << n) - 1 for n in n_par]
        g_rows = [self._zeros(bin(need[q]).count("1"), ty.E) for q, ty in enumerate(self.types)]
        states = saved["states"]
        rec_grad = rec_grad.contiguous()
        stored = saved["stored"]
        for seg in range((T + K - 1) // K - 1, -1, -1):
            t0 = seg * K
            k = min(K, T - t0)
            if stored:  # the forward kept the segment's kinetic states and synaptic terms
                s_seg = [st[t0:t0 + k + 1] if st is not None else None for st in saved["s_traj"]]
                LC_lin, LC_cst = saved["lin"][t0:t0 + k], saved["cst"][t0:t0 + k]
            else:  # recompute them from the segment's checkpoint
                for q, ty in enumerate(self.types):
                    if ty.kinetic:
                        s_seg[q][0].copy_(saved["s_ckpt"][q][seg])
                for i in range(k):
                    for q, ty in enumerate(self.types):
                        self._syn_forward(ty, q, states[t0 + i], s_seg[q][i] if ty.kinetic else None,
                                          s_seg[q][i + 1] if ty.kinetic else None, LC_lin[i], LC_cst[i],
                                          syn_params[q])
            for i in range(k - 1, -1, -1):
                t = t0 + i
                a = m.args(states[t], 1, t, None, pscale=pscale, traj=states[t], adj=adj, rec_grad=rec_grad,
                           pgrad=pgrad)
                a.ckpt = states[t].data_ptr()
                a.traj_piv = saved["piv"][t].data_ptr()
                a.traj_stored = 1
                self._set_syn(a, LC_lin[i], LC_cst[i])
                a.g_syn_lin = g_lin.data_ptr()
                a.g_syn_const = g_cst.data_ptr()
                m.launch_backward(a)
                for q, ty in enumerate(self.types):
                    b = ty.args(states[t], low.n_slots, B, syn_params[q])
                    b.s = s_seg[q][i].data_ptr() if ty.kinetic else None
                    b.g_s_new = g_s[q].data_ptr() if ty.kinetic else None
                    b.g_current = None
                    off, size = self.region[q]
                    b.g_lin = g_lin.data_ptr() + off * g_lin.element_size()
                    b.g_const = g_cst.data_ptr() + off * g_cst.element_size()
                    b.g_s = g_s2[q].data_ptr() if ty.kinetic else None
                    b.g_v = adj.data_ptr()
                    b.accumulate = 1
                    b.need = need[q]
                    b.g_params = g_rows[q].data_ptr() if need[q] else None
                    b.g_pre = g_pre[q].data_ptr()
                    _lib.check(_lib.load().jxb_synapse_backward(C.byref(b), _stream()), "jxb_synapse_backward")
                    self.syn_launches += 1
                    if ty.kinetic:
                        g_s[q], g_s2[q] = g_s2[q], g_s[q]
        # the rows of the computed parameters in parameter order, zeros for the others
        g_par_acc = []
        for q, ty in enumerate(self.types):
            rows, k = [], 0
            for i in range(n_par[q]):
                if (need[q] >> i) & 1:
                    rows.append(g_rows[q][k])
                    k += 1
                else:
                    rows.append(torch.zeros(ty.E, dtype=self.dtype, device=self.device))
            g_par_acc.append(rows)
        return pgrad, g_par_acc

    def run(self, pscale: Optional[torch.Tensor] = None, syn_params: Optional[List[List[torch.Tensor]]] = None,
            n_steps: Optional[int] = None):
        """Recordings `(B, n_rec, T + 1)`; differentiable with respect to `pscale` and
        the synapse parameter tensors."""
        T = int(self.low.n_steps if n_steps is None else n_steps)
        if pscale is None:
            pscale = self.model.pscale
        if syn_params is None:
            syn_params = [ty.params for ty in self.types]
        flat = [p for ps in syn_params for p in ps]
        if torch.is_grad_enabled() and (pscale.requires_grad or any(p.requires_grad for p in flat)):
            return _NetFn.apply(self, T, [len(ps) for ps in syn_params], pscale, *flat)
        rec, _ = self.forward_raw(pscale.detach().contiguous(), [[p.detach() for p in ps] for ps in syn_params], T)
        if self.sim.check_finite:
            self.model.check_finite("network simulation")
        return rec.permute(1, 2, 0)


class _NetFn(torch.autograd.Function):
    @staticmethod
    def forward(ctx, net: NetworkSimulation, T: int, counts, pscale, *flat):
        ps = pscale.detach().to(net.dtype).contiguous()
        params, q = [], 0
        for c in counts:
            params.append([p.detach().to(net.dtype).contiguous() for p in flat[q:q + c]])
            q += c
        rec, saved = net.forward_raw(ps, params, T, keep=True)
        if net.sim.check_finite:
            net.model.check_finite("network simulation")
        ctx.net, ctx.T, ctx.counts, ctx.saved_data = net, T, counts, saved
        ctx.params = params
        ctx.wants = [p.requires_grad for p in flat]
        ctx.save_for_backward(ps)
        ctx.dtypes = (pscale.dtype, [p.dtype for p in flat])
        return rec.permute(1, 2, 0)

    @staticmethod
    def backward(ctx, grad_out):
        (ps,) = ctx.saved_tensors
        net = ctx.net
        rec_grad = grad_out.to(net.dtype).permute(2, 0, 1).contiguous()
        need, q = [], 0
        for c in ctx.counts:
            need.append(sum(1 << i for i in range(c) if ctx.wants[q + i]))
            q += c
        pgrad, g_par = net.backward_raw(ps, ctx.params, ctx.T, ctx.saved_data, rec_grad, need=need)
        if net.sim.check_finite:
            net.model.check_finite("network adjoint")
        out = [None, None, None, pgrad.to(ctx.dtypes[0])]
        dts = ctx.dtypes[1]
        q = 0
        for t, c in enumerate(ctx.counts):
            for i in range(c):
                out.append(g_par[t][i].to(dts[q]) if ctx.wants[q] else None)
                q += 1
        return tuple(out)


def config_network(n_cells: int = 2048, ncomp: int = 4, k: int = 64, batch: int = 32, n_steps: int = 2000,
                   seed: int = 0, rate_hz: float = 20.0, amp: float = 0.2, dt: float = 0.025) -> Problem:
    """Fixed in-degree network: `n_cells` cells of one branch x `ncomp` compartments
    with HH, `k` KineticSynapse and `k` SigmoidRateSynapse inputs on compartment 0 of
    every cell (presynaptic cells uniform without replacement, excluding the cell,
    ordered by postsynaptic cell; gS ~ U[0, 1e-3] uS), `batch` rows of Poisson input
    (rate_hz per cell, one-step pulses of `amp` nA on compartment 0)."""
    from . import synth

    rng = np.random.default_rng(seed)
    cells = [synth.morphology([-1], [ncomp], [np.full(ncomp, 1.0)], [np.full(ncomp, 10.0)]) for _ in range(n_cells)]
    chans = [[("HH", np.arange(ncomp), "HH", {})] for _ in range(n_cells)]
    t_max = n_steps * dt
    L = int(t_max // dt) + 2
    prob = synth.assemble(cells, chans, batch=1, dt=dt, n_steps=n_steps, v0=-65.0,
                          recordings=[("v", c, (0, 0)) for c in range(n_cells)])
    offs = np.cumsum([0] + [c["n"] for c in cells])
    soma = offs[:-1]
    # Poisson input: (batch, n_cells, L) one-step pulses
    spikes = rng.random((batch, n_cells, L)) < rate_hz * dt * 1e-3
    prob.stim_inds = soma.astype(np.int64)
    prob.stim = (spikes * amp).astype(np.float64)
    prob.batch = batch
    syns = []
    for model, name, pnames, pdef in [
        # defaults of synapses/kinetic.py:27-35 and synapses/sigmoid_rate.py:26-31
        (0, "KineticSynapse", ["gS", "e_syn", "alpha", "beta", "v_th", "delta"], [None, 0.0, 1.0, 0.2, -20.0, 2.0]),
        (1, "SigmoidRateSynapse", ["gS", "x_offset", "slope"], [None, -60.0, 0.25]),
    ]:
        pre = np.empty(n_cells * k, dtype=np.int64)
        for c in range(n_cells):
            choice = rng.choice(n_cells - 1, size=k, replace=False)
            choice[choice >= c] += 1
            pre[c * k:(c + 1) * k] = soma[np.sort(choice)]
        post = np.repeat(soma, k)
        params = [rng.uniform(0.0, 1e-3, size=n_cells * k)] + [np.full(n_cells * k, float(v)) for v in pdef[1:]]
        syns.append(SynapseType(model=model, name=name, pre=pre, post=post, k=k, targets=soma.copy(),
                                params=params, param_names=[f"{name}_{p}" for p in pnames],
                                state=np.zeros((1, n_cells * k)) if model == 0 else None))
    prob.synapses = syns
    return prob


def config_lm(n_cells: int = 2048, k_in: int = 100, exc_frac: float = 0.8, batch: int = 32,
              n_tokens: int = 10, steps_per_token: int = 200, seed: int = 0, dt: float = 0.025,
              input_scale: float = 6.0, w_exc: float = 0.02, w_inh: float = 0.1) -> Problem:
    """The Hodgkin-Huxley network of the reference's character-level language model
    (`examples/language_modeling/models.py:66-72, 74-100, 128-215`, published H100
    throughput in its README:94-116): `n_cells` point neurons (one compartment,
    radius 10 um, length 20 um, HH, v = -65 mV at steady state), `k_in`
    KineticSynapse inputs per neuron on its compartment, `exc_frac` of the neurons
    excitatory and `exc_frac * k_in` of every neuron's inputs drawn from them
    (distinct presynaptic cells, no autapses), excitatory inputs first; excitatory
    synapses e_syn 0 mV, beta 0.2 /ms, inhibitory -80 mV, 0.1 /ms (alpha 1 /ms, v_th
    -20 mV, delta 2 mV); gS = w * (100 / k_in) mS/cm^2 times a log-normal(0, 0.5)
    factor, converted to uS on the target's area. Input: `batch` streams of
    `n_tokens` random tokens, each held for `steps_per_token` steps as a constant
    current of N(0, input_scale) uA/cm^2 per neuron (converted to nA)."""
    from . import synth

    rng = np.random.default_rng(seed)
    radius, length = 10.0, 20.0
    cells = [synth.morphology([-1], [1], [np.full(1, radius)], [np.full(1, length)]) for _ in range(n_cells)]
    chans = [[("HH", np.arange(1), "HH", {})] for _ in range(n_cells)]
    T = n_tokens * steps_per_token
    prob = synth.assemble(cells, chans, batch=1, dt=dt, n_steps=T, v0=-65.0,
                          recordings=[("v", c, (0, 0)) for c in range(n_cells)])
    area_cm2 = 2 * np.pi * radius * length * 1e-8
    n_exc = int(round(exc_frac * n_cells))
    k_exc = int(round(exc_frac * k_in))
    pre_cells = np.empty((n_cells, k_in), dtype=np.int64)
    for j in range(n_cells):
        for lo, hi, kk, col in ((0, n_exc, k_exc, 0), (n_exc, n_cells, k_in - k_exc, k_exc)):
            pool = np.arange(lo, hi)
            pool = pool[pool != j]
            pre_cells[j, col:col + kk] = rng.choice(pool, size=kk, replace=False)
    pre = pre_cells.reshape(-1)
    post = np.repeat(np.arange(n_cells), k_in)
    exc = pre < n_exc
    w = np.where(exc, w_exc, w_inh) * (100.0 / k_in) * np.exp(rng.normal(0.0, 0.5, len(pre)))
    gs = w * area_cm2 * 1e3  # mS/cm^2 over the target's area -> uS
    params = [gs, np.where(exc, 0.0, -80.0), np.ones(len(pre)), np.where(exc, 0.2, 0.1),
              np.full(len(pre), -20.0), np.full(len(pre), 2.0)]
    names = ["gS", "e_syn", "alpha", "beta", "v_th", "delta"]
    prob.synapses = [SynapseType(model=KINETIC, name="KineticSynapse", pre=pre, post=post, k=k_in,
                                 targets=np.arange(n_cells), params=params,
                                 param_names=[f"KineticSynapse_{p}" for p in names],
                                 state=np.zeros((1, len(pre))))]
    tokens = rng.normal(0.0, input_scale, size=(batch, n_cells, n_tokens)) * area_cm2 * 1e3  # nA
    prob.stim_inds = np.arange(n_cells, dtype=np.int64)
    prob.stim = np.repeat(tokens, steps_per_token, axis=-1)
    prob.batch = batch
    return prob


# --------------------------------------------------------------------------------------
# Several GPUs: the batch rows are sharded over the ranks; parameters shared by all rows
# (the synaptic weights of a training step) get one summed gradient.
# --------------------------------------------------------------------------------------
def shard_rows(problem: Problem, rank: int, world: int) -> Problem:
    """The rows `[rank * B // world, (rank + 1) * B // world)` of a problem's batch as a
    problem of their own: every array with a batch dimension (parameters, states,
    stimuli, clamps, kinetic synapse states) is sliced, shared arrays are kept."""
    import copy

    B = int(problem.batch)
    lo, hi = rank * B // world, (rank + 1) * B // world
    if hi <= lo:
        raise ValueError(f"rank {rank} of {world} gets no rows of a batch of {B}")

    def rows(a, core: int):
        a = np.asarray(a)
        return a[lo:hi] if a.ndim > core and a.shape[0] == B and B > 1 else a

    p = copy.copy(problem)
    p.params = {k: rows(v, 1) for k, v in problem.params.items()}
    p.states = {k: rows(v, 1) for k, v in problem.states.items()}
    p.axial = rows(problem.axial, 1)
    p.stim = rows(problem.stim, 2) if problem.stim is not None else None
    p.clamps = [(k, i, rows(v, 2)) for k, i, v in problem.clamps]
    syns = []
    for syn in problem.synapses:
        s = copy.copy(syn)
        if syn.state is not None:
            s.state = rows(syn.state, 1)
        if syn.current is not None:
            s.current = rows(syn.current, 1)
        syns.append(s)
    p.synapses = syns
    p.batch = hi - lo
    return p


def allreduce_gradients(grads: Sequence[torch.Tensor], group=None) -> None:
    """Sums gradients over the ranks of `group` in place with one collective: the
    tensors are packed into one buffer, all-reduced (sum) and unpacked. A rank's
    gradients must come from a loss that is its rows' share of the whole batch's
    loss (e.g. the squared errors of its rows divided by the number of rows of all
    ranks), so that the sum is the whole batch's gradient."""
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size(group) == 1 or not grads:
        return
    flat = torch.cat([g.reshape(-1) for g in grads])
    dist.all_reduce(flat, op=dist.ReduceOp.SUM, group=group)
    q = 0
    for g in grads:
        n = g.numel()
        g.copy_(flat[q:q + n].view_as(g))
        q += n
