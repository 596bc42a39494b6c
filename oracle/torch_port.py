"""torch restatement of the reference's step loop, for the CPU baseline of the
forward + backward metric.

TEST INFRASTRUCTURE / BASELINE ONLY (see `oracle/__init__.py`). The reference runs
`jx.integrate` as eager torch operations on the CPU and differentiates it with
autograd (`integrate.py:396-666`, `modules/base.py:3214-3542`,
`solver_voltage.py:78-241`); this module does the same on a `Problem`, with the
same operation structure: gathers per channel, the finite-difference current slope,
`index_add` of the linear terms, the level-by-level tree solve. The parity of its
forward pass with `oracle.step` is checked by `tests/test_oracle_golden.py`.
"""
from __future__ import annotations

from typing import Dict, List, Optional

import numpy as np
import torch

from . import step as S

DIFF = S.DIFF
QT = S.QT


def _save_exp(x):
    return torch.exp(torch.clamp(x, max=20.0))


def _x_over_expm1(x, y):
    z = torch.clamp(x / y, max=20.0)
    small = torch.abs(z) < 1e-4
    z_safe = torch.where(small, torch.ones_like(z), z)
    series = y * (1.0 - z / 2.0 + z * z / 12.0)
    return torch.where(small, series, x / torch.expm1(z_safe))


def _gate_ab(x, dt, a, b):  # solver_gate.py:45-64
    tau = 1 / (a + b)
    e = _save_exp(-dt / tau)
    return x * e + a * tau * (1.0 - e)


def _gate_inf(x, dt, inf, tau):  # solver_gate.py:67-87
    e = _save_exp(-1.0 / tau * dt)
    return x * e + inf * (1.0 - e)


def _rates(g, v):
    """(alpha, beta) or (x_inf, tau) of every gate (same formulas as oracle.step)."""
    if g == "hh_m":
        return 0.1 * _x_over_expm1(-(v + 40), 10), 4.0 * _save_exp(-(v + 65) / 18)
    if g == "hh_h":
        return 0.07 * _save_exp(-(v + 65) / 20), 1.0 / (_save_exp(-(v + 35) / 10) + 1)
    if g == "hh_n":
        return 0.01 * _x_over_expm1(-(v + 55), 10), 0.125 * _save_exp(-(v + 65) / 80)
    if g in ("na_m38", "na_m32"):
        off = 38 if g == "na_m38" else 32
        a = (0.182 * (v + off + 1e-6)) / (1 - _save_exp(-(v + off + 1e-6) / 6))
        b = (0.124 * (-v - off + 1e-6)) / (1 - _save_exp(-(-v - off + 1e-6) / 6))
        return a / (a + b), 1 / (a + b) / QT
    if g in ("na_h66", "na_h60"):
        off = 66 if g == "na_h66" else 60
        a = (-0.015 * (v + off + 1e-6)) / (1 - _save_exp((v + off + 1e-6) / 6))
        b = (-0.015 * (-v - off + 1e-6)) / (1 - _save_exp((-v - off + 1e-6) / 6))
        return a / (a + b), 1 / (a + b) / QT
    if g == "skv31":
        return 1 / (1 + _save_exp((v - 18.7) / -9.7)), 0.2 * 20.0 / (1 + _save_exp((v + 46.56) / -44.14))
    if g == "mm":
        a = 3.3e-3 * _save_exp(2.5 * 0.04 * (v + 35))
        b = 3.3e-3 * _save_exp(-2.5 * 0.04 * (v + 35))
        return a / (a + b), (1 / (a + b)) / QT
    if g == "hm":
        a = 0.001 * 6.43 * (v + 154.9 + 1e-6) / (_save_exp((v + 154.9 + 1e-6) / 11.9) - 1)
        b = 0.001 * 193 * _save_exp(v / 33.1)
        return a / (a + b), 1 / (a + b)
    if g == "cahva_m":
        a = (0.055 * (-27 - v + 1e-6)) / (_save_exp((-27.0 - v + 1e-6) / 3.8) - 1.0)
        return a, 0.94 * _save_exp((-75.0 - v + 1e-6) / 17.0)
    if g == "cahva_h":
        return 0.000457 * _save_exp((-13.0 - v) / 50.0), 0.0065 / (_save_exp((-v - 15.0) / 28.0) + 1.0)
    if g == "calva_m":
        vs = v + 10
        return 1.0 / (1 + _save_exp((vs + 30) / -6)), (5.0 + 20.0 / (1 + _save_exp((vs + 25) / 5))) / QT
    if g == "calva_h":
        vs = v + 10
        return 1.0 / (1 + _save_exp((vs + 80) / 6.4)), (20.0 + 50.0 / (1 + _save_exp((vs + 40) / 7))) / QT
    if g == "nap_m":
        a = (0.182 * (v + 38 + 1e-6)) / (1 - _save_exp(-(v + 38 + 1e-6) / 6))
        b = (0.124 * (-v - 38 + 1e-6)) / (1 - _save_exp(-(-v - 38 + 1e-6) / 6))
        return 1.0 / (1 + _save_exp((v + 52.6) / -4.6)), 6 / (a + b) / QT
    if g == "nap_h":
        a = (-2.88e-6 * (v + 17 + 1e-6)) / (1 - _save_exp((v + 17 + 1e-6) / 4.63))
        b = (6.94e-6 * (v + 64.4 + 1e-6)) / (1 - _save_exp((-(v + 64.4) + 1e-6) / 2.63))
        return 1.0 / (1 + _save_exp((v + 48.8) / 10)), 1 / (a + b) / QT
    va = v + 10
    if g == "kpst_m":
        tau = torch.where(va < -50.0, (1.25 + 175.03 * _save_exp(va * 0.026)) / QT,
                          (1.25 + 13 * _save_exp(-va * 0.026)) / QT)
        return 1 / (1 + _save_exp(-(va + 1) / 12)), tau
    if g == "kpst_h":
        return (1 / (1 + _save_exp(-(va + 54) / -11)),
                (360 + (1010 + 24 * (va + 55)) * _save_exp(-(((va + 75) / 48) ** 2))) / QT)
    if g == "ktst_m":
        return 1 / (1 + _save_exp(-(va + 0) / 19)), (0.34 + 0.92 * _save_exp(-(((va + 71) / 59) ** 2))) / QT
    if g == "ktst_h":
        return 1 / (1 + _save_exp(-(va + 66) / -10)), (8 + 49 * _save_exp(-(((va + 73) / 23) ** 2))) / QT
    raise NotImplementedError(g)


_GATES = {
    "NapEt2": [("nap_m", "inf"), ("nap_h", "inf")],
    "KPst": [("kpst_m", "inf"), ("kpst_h", "inf")],
    "KTst": [("ktst_m", "inf"), ("ktst_h", "inf")],
    "HH": [("hh_m", "ab"), ("hh_h", "ab"), ("hh_n", "ab")],
    "NaTaT": [("na_m38", "inf"), ("na_h66", "inf")],
    "NaTs2T": [("na_m32", "inf"), ("na_h60", "inf")],
    "SKv3_1": [("skv31", "inf")],
    "M": [("mm", "inf")],
    "H": [("hm", "inf")],
    "CaHVA": [("cahva_m", "ab"), ("cahva_h", "ab")],
    "CaLVA": [("calva_m", "inf"), ("calva_h", "inf")],
}
_EXPONENT = {"NaTaT": 3, "NaTs2T": 3, "NapEt2": 3, "KPst": 2, "KTst": 4, "CaHVA": 2, "CaLVA": 2}


def _update(ch, st, dt, v, prm):
    t, Sn = ch.type_name, ch.states
    if t in _GATES:
        out = {}
        for q, (g, kind) in enumerate(_GATES[t]):
            r = _rates(g, v)
            out[Sn[q]] = _gate_ab(st[Sn[q]], dt, *r) if kind == "ab" else _gate_inf(st[Sn[q]], dt, *r)
        return out
    if t == "Leak":
        return {}
    if t == "SKE2":
        cai = st[Sn[1]]
        cai = torch.where(cai < 1e-7, cai + 1e-7, cai)
        zinf = 1 / (1 + (0.00043 / cai) ** 4.8)
        return {Sn[0]: _gate_inf(st[Sn[0]], dt, zinf, torch.ones_like(zinf))}
    if t == "CaPump":
        gamma, decay, depth, minCai = (prm[p] for p in ch.params)
        drive = -10_000.0 * st[ch.current] * gamma / (2 * 96485 * depth)
        e = _save_exp(-dt / decay)
        return {Sn[0]: st[Sn[0]] * e + (minCai + decay * drive) * (1.0 - e)}
    if t == "CaNernstReversal":
        F, T, R = ch.constants
        return {Sn[0]: R * T / (2 * F) * 1000 * torch.log(st[Sn[2]] / st[Sn[1]])}
    raise NotImplementedError(t)


def _current(ch, st, v, prm):
    t, Sn, P = ch.type_name, ch.states, ch.params
    if t == "HH":
        m, h, n = st[Sn[0]], st[Sn[1]], st[Sn[2]]
        return (prm[P[0]] * m**3 * h * (v - prm[P[3]]) + prm[P[1]] * n**4 * (v - prm[P[4]])
                + prm[P[2]] * (v - prm[P[5]]))
    if t == "Leak":
        return prm[P[0]] * (v - prm[P[1]])
    if t in _EXPONENT:
        e = st[Sn[2]] if t in ("CaHVA", "CaLVA") else prm[P[1]]
        return prm[P[0]] * st[Sn[0]] ** _EXPONENT[t] * st[Sn[1]] * (v - e)
    if t in ("SKv3_1", "M", "H", "SKE2"):
        return prm[P[0]] * st[Sn[0]] * (v - prm[P[1]])
    return torch.zeros_like(v)


def _synapse_terms(syn, prm, s, v, area_post, dt):
    """One synapse type's step (modules/network.py:434-478, synapses/kinetic.py:37-63,
    synapses/sigmoid_rate.py:43-50) in torch: the new kinetic state and the per-target
    slope and offset of the summed synaptic current, `(B, E)`, `(B, T)`, `(B, T)`."""
    pre = torch.as_tensor(np.asarray(syn.pre, dtype=np.int64))
    tgt = torch.as_tensor(np.repeat(np.asarray(syn.targets, dtype=np.int64), syn.k))
    vpre, vp = v[:, pre], v[:, tgt]
    gs = prm[0]
    if syn.model == 0:
        e_syn, alpha, beta, v_th, delta = prm[1:6]
        a = alpha * torch.sigmoid((vpre - v_th) / delta)
        rate = a + beta
        s_inf = a / rate
        s = s_inf + (s - s_inf) * torch.exp(-dt * rate)
        i0 = gs * s * (vp - e_syn)
        i1 = gs * s * ((vp + DIFF) - e_syn)
    else:
        x_off, slope = prm[1:3]
        i0 = -gs * torch.sigmoid((vpre - x_off) * slope)
        i1 = -gs * torch.sigmoid(((vpre + DIFF) - x_off) * slope)
    d0 = i0 / area_post * 100_000
    d1 = i1 / area_post * 100_000
    vt = (d1 - d0) / DIFF
    B = v.shape[0]
    return s, vt.reshape(B, -1, syn.k).sum(-1), (d0 - vt * vp).reshape(B, -1, syn.k).sum(-1)


def integrate(problem, params: Dict[str, torch.Tensor], n_steps: Optional[int] = None,
              dtype=torch.float32, init_steady: bool = False,
              syn_params: Optional[List[List[torch.Tensor]]] = None) -> torch.Tensor:
    """Recordings `(B, n_rec, T + 1)`; `params` maps parameter names to `(B, n)` or
    `(n,)` tensors, `syn_params` gives every synapse type's parameters as `(E,)`
    tensors in the reference order (default: the problem's); autograd flows into
    both."""
    p = problem
    B, n = p.batch, p.n_nodes
    T = p.n_steps if n_steps is None else int(n_steps)
    dt = p.dt
    st0 = {k: np.asarray(v, dtype=np.float64) for k, v in p.states.items()}
    if init_steady:
        st0 = S.init_steady_states(p, st0)
    st = {k: torch.as_tensor(np.broadcast_to(v, (B, v.shape[-1])).copy(), dtype=dtype)
          for k, v in st0.items()}

    def P(name):
        x = params[name] if name in params else torch.as_tensor(np.asarray(p.params[name]), dtype=dtype)
        return torch.broadcast_to(x, (B, n))

    area = P("area")
    cm = P("capacitance")
    comp = torch.as_tensor(np.asarray(p.comp_inds, dtype=np.int64))
    chans = []
    for ch in p.channels:
        inds = torch.as_tensor(np.asarray(ch.inds, dtype=np.int64))
        chans.append((ch, inds, {q: P(q)[:, inds] for q in ch.params}))
    cur_names = list(p.current_names)
    parent = np.asarray(p.parent_lookup)
    depth = S._depth(parent)
    levels = [torch.as_tensor(np.nonzero(depth == k)[0]) for k in range(int(depth.max()) + 1)]
    parent_t = torch.as_tensor(parent)
    order = torch.as_tensor(np.asarray(p.to_solve, dtype=np.int64))
    inv_order = torch.empty_like(order)
    inv_order[order] = torch.arange(n)
    ax = torch.as_tensor(np.asarray(p.axial), dtype=dtype) * dt
    sinks = torch.as_tensor(np.asarray(p.sinks, dtype=np.int64))
    lo = (-ax)[..., torch.as_tensor(p.map_lower)]
    up = (-ax)[..., torch.as_tensor(p.map_upper)]
    root = torch.as_tensor(parent < 0)
    lo = torch.where(root, torch.zeros_like(lo), lo)
    up = torch.where(root, torch.zeros_like(up), up)
    stim_inds = torch.as_tensor(np.asarray(p.stim_inds, dtype=np.int64))
    stim = torch.as_tensor(np.asarray(p.stim), dtype=dtype) if p.stim is not None else None

    def currents(st, v):
        lin = torch.zeros(B, n, dtype=dtype)
        const = torch.zeros(B, n, dtype=dtype)
        cs = {k: torch.zeros(B, n, dtype=dtype) for k in cur_names}
        for ch, inds, prm in chans:
            chs = {k: st[k][:, inds] for k in ch.states}
            vv = v[:, inds]
            i0 = torch.broadcast_to(_current(ch, chs, vv, prm), vv.shape)
            i1 = torch.broadcast_to(_current(ch, chs, vv + DIFF, prm), vv.shape)
            vt = (i1 - i0) / DIFF
            lin = lin.index_add(1, inds, vt)
            const = const.index_add(1, inds, -(i0 - vt * vv))
            cs[ch.current] = cs[ch.current].index_add(1, inds, i0)
        st.update(cs)
        return lin * 1000.0, const * 1000.0

    def solve(v, lin, const):
        diags = (dt * lin).index_add(1, comp, torch.ones(B, len(comp), dtype=dtype))
        diags = diags.index_add(1, sinks, torch.broadcast_to(ax, (B, ax.shape[-1])))
        vals = v[:, comp] + dt * const[:, comp]
        solves = torch.zeros(B, n, dtype=dtype).index_copy(1, comp, vals)
        if ax.shape[-1] == 0:
            return solves / diags
        d = diags[:, order]
        s = solves[:, order]
        l_ = torch.broadcast_to(lo, (B, n))
        u_ = torch.broadcast_to(up, (B, n))
        for lev in reversed(levels[1:]):  # solver_voltage.py:93-98
            par = parent_t[lev]
            mult = u_[:, lev] / d[:, lev]
            d = d.index_add(1, par, -l_[:, lev] * mult)
            s = s.index_add(1, par, -s[:, lev] * mult)
        ln = l_ / d
        s = s / d
        for lev in levels[1:]:  # solver_voltage.py:100-106
            s = s.index_add(1, lev, -s[:, parent_t[lev]] * ln[:, lev])
        return s[:, inv_order]

    syns = []
    for q, syn in enumerate(p.synapses):
        prm = (syn_params[q] if syn_params is not None
               else [torch.as_tensor(np.asarray(x), dtype=dtype) for x in syn.params])
        s0 = (torch.as_tensor(np.broadcast_to(np.asarray(syn.state), (B, len(syn.pre))).copy(), dtype=dtype)
              if syn.model == 0 else None)
        syns.append([syn, prm, s0, area[:, np.asarray(syn.post, dtype=np.int64)]])
    currents(st, st["v"])
    recs = [torch.stack([st[nm][:, i] for nm, i in p.recordings], dim=1)]
    for t in range(T):
        v = st["v"]
        st = dict(st)
        for ch, inds, prm in chans:
            names = list(dict.fromkeys(list(ch.states) + cur_names))
            chs = {k: st[k][:, inds] for k in names if k in st}
            for key, val in _update(ch, chs, dt, v[:, inds], prm).items():
                st[key] = st[key].index_copy(1, inds, val)
        lin, const = currents(st, v)
        for entry in syns:
            syn, prm, s_old, area_post = entry
            s_new, l_t, c_t = _synapse_terms(syn, prm, s_old, v, area_post, dt)
            entry[2] = s_new
            tg = torch.as_tensor(np.asarray(syn.targets, dtype=np.int64))
            lin = lin + torch.zeros(B, n, dtype=dtype).index_add(1, tg, l_t)
            const = const + torch.zeros(B, n, dtype=dtype).index_add(1, tg, -c_t)
        i_ext = torch.zeros(B, n, dtype=dtype)
        if stim is not None and len(stim_inds):
            cur = torch.broadcast_to(stim[:, :, t], (B, len(stim_inds))) / area[:, stim_inds] * 100_000
            i_ext = i_ext.index_add(1, stim_inds, cur)
        st["v"] = solve(v, lin / cm, (const + i_ext) / cm)
        recs.append(torch.stack([st[nm][:, i] for nm, i in p.recordings], dim=1))
    return torch.stack(recs, dim=-1)
