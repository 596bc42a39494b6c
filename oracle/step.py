"""numpy float64 restatement of jaxley-pytorch's `bwd_euler` + DHS step loop.

TEST INFRASTRUCTURE ONLY (see `oracle/__init__.py`). Every function cites the
reference lines it restates. Inputs are `jaxley_pytorch_b200.problem.Problem`
instances (reference node order).
"""
from __future__ import annotations

from typing import Dict, List, Optional, Tuple

import numpy as np

DIFF = 1e-3  # modules/base.py:3522 and modules/network.py:29
QT = 2.3 ** ((34 - 21) / 10)  # mech/channels/l5pc.py (every q10 factor)
FARADAY_PUMP = 96485  # mech/channels/l5pc.py:849


# --------------------------------------------------------------------------------------
# solver_gate.py
# --------------------------------------------------------------------------------------
def save_exp(x, max_value: float = 20.0):
    """solver_gate.py:8-11."""
    return np.exp(np.minimum(x, max_value))


def x_over_expm1(x, y=1.0):
    """solver_gate.py:14-30: `x / (exp(x/y) - 1)` with the series near 0."""
    x = np.asarray(x, dtype=np.float64)
    z = np.minimum(x / y, 20.0)
    small = np.abs(z) < 1e-4
    z_safe = np.where(small, 1.0, z)
    series = y * (1.0 - z / 2.0 + z * z / 12.0)
    with np.errstate(divide="ignore", invalid="ignore"):
        full = x / np.expm1(z_safe)
    return np.where(small, series, full)


def exponential_euler(x, dt, x_inf, x_tau):
    """solver_gate.py:56-64."""
    exp_term = save_exp(-dt / x_tau)
    return x * exp_term + x_inf * (1.0 - exp_term)


def solve_gate_exponential(x, dt, alpha, beta):
    """solver_gate.py:45-53."""
    tau = 1 / (alpha + beta)
    xinf = alpha * tau
    return exponential_euler(x, dt, xinf, tau)


def solve_inf_gate_exponential(x, dt, s_inf, tau_s):
    """solver_gate.py:67-87."""
    slope = -1.0 / tau_s
    exp_term = save_exp(slope * dt)
    return x * exp_term + s_inf * (1.0 - exp_term)


def _sigmoid(x):
    return 1.0 / (1.0 + np.exp(-x))


# --------------------------------------------------------------------------------------
# Channel models: update_states / compute_current / init_state
# --------------------------------------------------------------------------------------
def _hh_m(v):  # channels/hh.py:88-92
    return 0.1 * x_over_expm1(-(v + 40), 10), 4.0 * save_exp(-(v + 65) / 18)


def _hh_h(v):  # channels/hh.py:94-98
    return 0.07 * save_exp(-(v + 65) / 20), 1.0 / (save_exp(-(v + 35) / 10) + 1)


def _hh_n(v):  # channels/hh.py:100-104
    return 0.01 * x_over_expm1(-(v + 55), 10), 0.125 * save_exp(-(v + 65) / 80)


def _na_m(v, off):  # l5pc.py:95-103 (NaTaT, off=38), :177-185 (NaTs2T, off=32)
    alpha = (0.182 * (v + off + 1e-6)) / (1 - save_exp(-(v + off + 1e-6) / 6))
    beta = (0.124 * (-v - off + 1e-6)) / (1 - save_exp(-(-v - off + 1e-6) / 6))
    return alpha / (alpha + beta), 1 / (alpha + beta) / QT


def _na_h(v, off):  # l5pc.py:105-113 (off=66), :187-195 (off=60)
    alpha = (-0.015 * (v + off + 1e-6)) / (1 - save_exp((v + off + 1e-6) / 6))
    beta = (-0.015 * (-v - off + 1e-6)) / (1 - save_exp((-v - off + 1e-6) / 6))
    return alpha / (alpha + beta), 1 / (alpha + beta) / QT


def _nap_m(v):  # l5pc.py:268-276
    alpha = (0.182 * (v + 38 + 1e-6)) / (1 - save_exp(-(v + 38 + 1e-6) / 6))
    beta = (0.124 * (-v - 38 + 1e-6)) / (1 - save_exp(-(-v - 38 + 1e-6) / 6))
    tau_m = 6 / (alpha + beta) / QT
    m_inf = 1.0 / (1 + save_exp((v + 52.6) / -4.6))
    return m_inf, tau_m


def _nap_h(v):  # l5pc.py:278-289
    alpha = (-2.88e-6 * (v + 17 + 1e-6)) / (1 - save_exp((v + 17 + 1e-6) / 4.63))
    beta = (6.94e-6 * (v + 64.4 + 1e-6)) / (1 - save_exp((-(v + 64.4) + 1e-6) / 2.63))
    tau_h = 1 / (alpha + beta) / QT
    h_inf = 1.0 / (1 + save_exp((v + 48.8) / 10))
    return h_inf, tau_h


def _kpst_m(v):  # l5pc.py:355-369
    va = v + 10
    m_inf = 1 / (1 + save_exp(-(va + 1) / 12))
    tau_m = np.where(
        va < -50.0,
        (1.25 + 175.03 * save_exp(va * 0.026)) / QT,
        (1.25 + 13 * save_exp(-va * 0.026)) / QT,
    )
    return m_inf, tau_m


def _kpst_h(v):  # l5pc.py:371-381
    va = v + 10
    h_inf = 1 / (1 + save_exp(-(va + 54) / -11))
    tau_h = (360 + (1010 + 24 * (va + 55)) * save_exp(-(((va + 75) / 48) ** 2))) / QT
    return h_inf, tau_h


def _ktst_m(v):  # l5pc.py:444-451
    va = v + 10
    m_inf = 1 / (1 + save_exp(-(va + 0) / 19))
    tau_m = (0.34 + 0.92 * save_exp(-(((va + 71) / 59) ** 2))) / QT
    return m_inf, tau_m


def _ktst_h(v):  # l5pc.py:453-460
    va = v + 10
    h_inf = 1 / (1 + save_exp(-(va + 66) / -10))
    tau_h = (8 + 49 * save_exp(-(((va + 73) / 23) ** 2))) / QT
    return h_inf, tau_h


def _ske2_z(cai):  # l5pc.py:519-530
    cai = np.where(cai < 1e-7, cai + 1e-7, cai)
    return 1 / (1 + (0.00043 / cai) ** 4.8), 1.0


def _skv31_m(v):  # l5pc.py:585-590
    return 1 / (1 + save_exp((v - 18.7) / -9.7)), 0.2 * 20.0 / (1 + save_exp((v + 46.56) / -44.14))


def _mm_m(v):  # l5pc.py:653-661
    a = 3.3e-3 * save_exp(2.5 * 0.04 * (v + 35))
    b = 3.3e-3 * save_exp(-2.5 * 0.04 * (v + 35))
    return a / (a + b), (1 / (a + b)) / QT


def _cahva_m(v):  # l5pc.py:723-727
    alpha = (0.055 * (-27 - v + 1e-6)) / (save_exp((-27.0 - v + 1e-6) / 3.8) - 1.0)
    beta = 0.94 * save_exp((-75.0 - v + 1e-6) / 17.0)
    return alpha, beta


def _cahva_h(v):  # l5pc.py:729-734
    return 0.000457 * save_exp((-13.0 - v) / 50.0), 0.0065 / (save_exp((-v - 15.0) / 28.0) + 1.0)


def _calva_m(v):  # l5pc.py:795-802
    vs = v + 10
    return 1.0 / (1 + save_exp((vs + 30) / -6)), (5.0 + 20.0 / (1 + save_exp((vs + 25) / 5))) / QT


def _calva_h(v):  # l5pc.py:804-811
    vs = v + 10
    return 1.0 / (1 + save_exp((vs + 80) / 6.4)), (20.0 + 50.0 / (1 + save_exp((vs + 40) / 7))) / QT


def _h_m(v):  # l5pc.py:973-984
    a = 0.001 * 6.43 * (v + 154.9 + 1e-6) / (save_exp((v + 154.9 + 1e-6) / 11.9) - 1)
    b = 0.001 * 193 * save_exp(v / 33.1)
    return a / (a + b), 1 / (a + b)


_INF_TAU_2 = {  # (m gate, h gate, m exponent, h exponent) of x_inf/tau channels
    "NaTaT": (lambda v: _na_m(v, 38), lambda v: _na_h(v, 66), 3),
    "NaTs2T": (lambda v: _na_m(v, 32), lambda v: _na_h(v, 60), 3),
    "NapEt2": (_nap_m, _nap_h, 3),
    "KPst": (_kpst_m, _kpst_h, 2),
    "KTst": (_ktst_m, _ktst_h, 4),
    "CaLVA": (_calva_m, _calva_h, 2),
}
_INF_TAU_1 = {"SKv3_1": _skv31_m, "M": _mm_m, "H": _h_m}


# Pospischil channels (channels/pospischil.py). efun(x) = x / (exp(x) - 1).
def _efun(x):
    return x_over_expm1(x)


def _pna_m(v, vt):  # pospischil.py:124-131
    return 0.32 * _efun(-0.25 * (v - vt - 13.0)) / 0.25, 0.28 * _efun(0.2 * (v - vt - 40.0)) / 0.2


def _pna_h(v, vt):  # pospischil.py:133-140
    return 0.128 * save_exp(-(v - vt - 17.0) / 18.0), 4.0 / (save_exp(-(v - vt - 40.0) / 5.0) + 1.0)


def _pk_n(v, vt):  # pospischil.py:186-193
    return 0.032 * _efun(-0.2 * (v - vt - 15.0)) / 0.2, 0.5 * save_exp(-(v - vt - 10.0) / 40.0)


def _pkm_p(v, taumax):  # pospischil.py:242-249: (p_inf, tau_p)
    vp = v + 35.0
    return 1.0 / (1.0 + save_exp(-0.1 * vp)), taumax / (3.3 * save_exp(0.05 * vp) + save_exp(-0.05 * vp))


def _pcal_q(v):  # pospischil.py:301-308
    return 0.055 * _efun((-v - 27.0) / 3.8) * 3.8, 0.94 * save_exp((-v - 75.0) / 17.0)


def _pcal_r(v):  # pospischil.py:310-317
    return 0.000457 * save_exp((-v - 13.0) / 50), 0.0065 / (save_exp((-v - 15.0) / 28.0) + 1)


def _pcat_u(v, vx):  # pospischil.py:366-375: (u_inf, tau_u)
    u_inf = 1.0 / (1.0 + save_exp((v + vx + 81.0) / 4))
    tau = (30.8 + (211.4 + save_exp((v + vx + 113.2) / 5.0))) / (3.7 * (1 + save_exp((v + vx + 84.0) / 3.2)))
    return u_inf, tau


def channel_update(ch, st: Dict[str, np.ndarray], dt, v, prm: Dict[str, np.ndarray]):
    """`Channel.update_states` of every supported channel. `st` maps the reference
    state names (and current names) to arrays at the channel's nodes."""
    t = ch.type_name
    S = ch.states
    if t == "HH":  # channels/hh.py:37-50
        return {
            S[0]: solve_gate_exponential(st[S[0]], dt, *_hh_m(v)),
            S[1]: solve_gate_exponential(st[S[1]], dt, *_hh_h(v)),
            S[2]: solve_gate_exponential(st[S[2]], dt, *_hh_n(v)),
        }
    if t == "Leak":  # channels/pospischil.py:54-62
        return {}
    if t in _INF_TAU_2:  # e.g. l5pc.py:145-157
        mg, hg, _ = _INF_TAU_2[t]
        return {
            S[0]: solve_inf_gate_exponential(st[S[0]], dt, *mg(v)),
            S[1]: solve_inf_gate_exponential(st[S[1]], dt, *hg(v)),
        }
    if t in _INF_TAU_1:  # l5pc.py:556-567, 618-629, 942-953
        return {S[0]: solve_inf_gate_exponential(st[S[0]], dt, *_INF_TAU_1[t](v))}
    if t == "SKE2":  # l5pc.py:488-500
        return {S[0]: solve_inf_gate_exponential(st[S[0]], dt, *_ske2_z(st[S[1]]))}
    if t == "CaHVA":  # l5pc.py:688-700
        return {
            S[0]: solve_gate_exponential(st[S[0]], dt, *_cahva_m(v)),
            S[1]: solve_gate_exponential(st[S[1]], dt, *_cahva_h(v)),
            S[2]: st[S[2]],
        }
    if t == "CaPump":  # l5pc.py:842-861
        ica = st[ch.current]
        cai = st[S[0]]
        gamma, decay, depth, minCai = (prm[p] for p in ch.params)
        drive_channel = -10_000.0 * ica * gamma / (2 * FARADAY_PUMP * depth)
        cai_inf = minCai + decay * drive_channel
        return {S[0]: exponential_euler(cai, dt, cai_inf, decay)}
    if t == "CaNernstReversal":  # l5pc.py:891-902
        F, T, R = ch.constants
        Cai, Cao = st[S[1]], st[S[2]]
        C = R * T / (2 * F) * 1000
        return {S[0]: C * np.log(Cao / Cai), S[1]: Cai, S[2]: Cao}
    P = ch.params
    if t == "Na":  # pospischil.py:91-104
        vt = prm[P[2]]
        return {S[0]: solve_gate_exponential(st[S[0]], dt, *_pna_m(v, vt)),
                S[1]: solve_gate_exponential(st[S[1]], dt, *_pna_h(v, vt))}
    if t == "K":  # pospischil.py:158-169
        return {S[0]: solve_gate_exponential(st[S[0]], dt, *_pk_n(v, prm[P[2]]))}
    if t == "Km":  # pospischil.py:212-225
        return {S[0]: solve_inf_gate_exponential(st[S[0]], dt, *_pkm_p(v, prm[P[1]]))}
    if t == "CaL":  # pospischil.py:271-284
        return {S[0]: solve_gate_exponential(st[S[0]], dt, *_pcal_q(v)),
                S[1]: solve_gate_exponential(st[S[1]], dt, *_pcal_r(v))}
    if t == "CaT":  # pospischil.py:334-347
        return {S[0]: solve_inf_gate_exponential(st[S[0]], dt, *_pcat_u(v, prm[P[1]]))}
    raise NotImplementedError(t)


def channel_current(ch, st, v, prm):
    """`Channel.compute_current` (mA/cm^2) of every supported channel."""
    t = ch.type_name
    S = ch.states
    P = ch.params
    if t == "HH":  # channels/hh.py:52-67
        m, h, n = st[S[0]], st[S[1]], st[S[2]]
        gNa = prm[P[0]] * (m**3) * h
        gK = prm[P[1]] * n**4
        gLeak = prm[P[2]]
        return gNa * (v - prm[P[3]]) + gK * (v - prm[P[4]]) + gLeak * (v - prm[P[5]])
    if t == "Leak":  # channels/pospischil.py:64-68
        return prm[P[0]] * (v - prm[P[1]])
    if t in _INF_TAU_2:  # e.g. l5pc.py:159-167, 333-342
        p = _INF_TAU_2[t][2]
        cond = prm[P[0]] * (st[S[0]] ** p) * st[S[1]]
        e = st[S[2]] if t == "CaLVA" else prm[P[1]]
        return cond * (v - e)
    if t in _INF_TAU_1 or t == "SKE2":  # l5pc.py:502-511, 569-578, 631-640, 955-964
        return prm[P[0]] * st[S[0]] * (v - prm[P[1]])
    if t == "CaHVA":  # l5pc.py:702-711
        return prm[P[0]] * (st[S[0]] ** 2) * st[S[1]] * (v - st[S[2]])
    if t in ("CaPump", "CaNernstReversal"):  # l5pc.py:863-865, 904-906
        return np.zeros_like(v)
    if t == "Na":  # pospischil.py:106-115
        return prm[P[0]] * (st[S[0]] ** 3) * st[S[1]] * (v - prm[P[1]])
    if t == "K":  # pospischil.py:171-178
        return prm[P[0]] * (st[S[0]] ** 4) * (v - prm[P[1]])
    if t == "Km":  # pospischil.py:227-230
        return prm[P[0]] * st[S[0]] * (v - prm[P[2]])
    if t == "CaL":  # pospischil.py:286-292
        return prm[P[0]] * (st[S[0]] ** 2) * st[S[1]] * (v - prm[P[1]])
    if t == "CaT":  # pospischil.py:349-357
        s_inf = 1.0 / (1.0 + save_exp(-(v + prm[P[1]] + 57.0) / 6.2))
        return prm[P[0]] * (s_inf**2) * st[S[0]] * (v - prm[P[2]])
    raise NotImplementedError(t)


def channel_init(ch, v, prm):
    """`Channel.init_state` (steady state at `v`)."""
    t = ch.type_name
    S = ch.states
    if t == "HH":  # channels/hh.py:69-86
        out = {}
        for s, g in zip(S, (_hh_m, _hh_h, _hh_n)):
            a, b = g(v)
            out[s] = a / (a + b)
        return out
    if t in _INF_TAU_2:
        return {S[0]: _INF_TAU_2[t][0](v)[0], S[1]: _INF_TAU_2[t][1](v)[0]}
    if t in _INF_TAU_1:
        return {S[0]: _INF_TAU_1[t](v)[0]}
    if t == "SKE2":  # l5pc.py:513-517
        return {S[0]: _ske2_z(np.asarray(5e-05))[0] * np.ones_like(v)}
    if t == "CaHVA":  # l5pc.py:713-721
        am, bm = _cahva_m(v)
        ah, bh = _cahva_h(v)
        return {S[0]: am / (am + bm), S[1]: ah / (ah + bh)}
    P = ch.params
    # Pospischil init_state (pospischil.py:117-125, 180-184, 232-237, 294-303, 360-364):
    # alpha / (alpha + beta) of each gate's pair, also for the (x_inf, tau) pairs of Km
    # and CaT.
    pairs = {"Na": lambda: [_pna_m(v, prm[P[2]]), _pna_h(v, prm[P[2]])],
             "K": lambda: [_pk_n(v, prm[P[2]])], "Km": lambda: [_pkm_p(v, prm[P[1]])],
             "CaL": lambda: [_pcal_q(v), _pcal_r(v)], "CaT": lambda: [_pcat_u(v, prm[P[1]])]}
    if t in pairs:
        return {s_: a / (a + b) for s_, (a, b) in zip(S, pairs[t]())}
    return {}


# --------------------------------------------------------------------------------------
# Tree solve (solver_voltage.py:78-108, jaxley.dhs.cpu)
# --------------------------------------------------------------------------------------
def _depth(parent):
    parent = np.asarray(parent)
    depth = np.zeros(len(parent), dtype=np.int64)
    for j in range(len(parent)):  # parents precede children in solve order
        if parent[j] >= 0:
            depth[j] = depth[parent[j]] + 1
    return depth


def tree_solve(d, l, u, s, parent, depth=None):
    """Solve `A x = s` with `A[j,j]=d[j]`, `A[j,p]=l[j]`, `A[p,j]=u[j]` (`p` the
    parent of `j` in solve order). Triangularization leaves first, then sequential
    back-substitution, as `DHSSolver.raw_solve` (solver_voltage.py:90-106) with the
    levels given by the depth of every node. Arrays are `(B, n)`."""
    d = np.array(d, dtype=np.float64, copy=True)
    s = np.array(s, dtype=np.float64, copy=True)
    l = np.asarray(l, dtype=np.float64)
    u = np.asarray(u, dtype=np.float64)
    parent = np.asarray(parent)
    if depth is None:
        depth = _depth(parent)
    max_depth = int(depth.max()) if len(depth) else 0
    levels = [np.nonzero(depth == k)[0] for k in range(max_depth + 1)]
    dT, sT = d.T, s.T
    for k in range(max_depth, 0, -1):
        child = levels[k]
        par = parent[child]
        multiplier = u[:, child] / d[:, child]
        np.add.at(dT, par, (-l[:, child] * multiplier).T)
        np.add.at(sT, par, (-s[:, child] * multiplier).T)
    lowers_norm = l / d
    s = s / d
    for k in range(1, max_depth + 1):
        child = levels[k]
        s[:, child] = s[:, child] - s[:, parent[child]] * lowers_norm[:, child]
    return s


# --------------------------------------------------------------------------------------
# Synapses (modules/network.py:381-478; kernels/synapse_step.py:121-182)
# --------------------------------------------------------------------------------------
def synapse_step(model, v, s, pre, targets, k, params, area, dt, diff=DIFF,
                 targets_are_nodes=False):
    """The `synapse_step` op: returns `(s_new, current, lin, const)` with `lin`,
    `const` of shape `(B, T)` (`const` is the sum of the offsets, not negated),
    `kernels/synapse_step.py:121-182`, `modules/network.py:434-478`."""
    v = np.asarray(v, dtype=np.float64)
    B = v.shape[0]
    E = len(pre)
    T = E // k
    vpre = v[:, pre]  # (B, E)
    node = np.arange(T) if targets_are_nodes else np.asarray(targets)
    vp = np.repeat(v[:, node], k, axis=1)  # (B, E)
    gs = params[0][None]
    if model == 0:  # synapses/kinetic.py:37-63
        e_syn, alpha, beta, v_th, delta = (p[None] for p in params[1:6])
        transmitter = _sigmoid((vpre - v_th) / delta)
        a = alpha * transmitter
        rate = a + beta
        s_inf = a / rate
        s_new = s_inf + (s - s_inf) * np.exp(-dt * rate)
        i0 = gs * s_new * (vp - e_syn)
        i1 = gs * s_new * ((vp + diff) - e_syn)
    else:  # synapses/sigmoid_rate.py:43-50
        x_offset, slope = params[1][None], params[2][None]
        s_new = None
        i0 = -gs * _sigmoid((vpre - x_offset) * slope)
        i1 = -gs * _sigmoid(((vpre + diff) - x_offset) * slope)
    d0 = i0 / area[None] * 100000.0
    d1 = i1 / area[None] * 100000.0
    vt = (d1 - d0) / diff
    ct = d0 - vt * vp
    lin = vt.reshape(B, T, k).sum(-1)
    const = ct.reshape(B, T, k).sum(-1)
    return s_new, i0, lin, const


def synapse_step_backward(model, v, s, pre, targets, k, params, area, dt, g_s_new,
                          g_current, g_lin, g_const, diff=DIFF, targets_are_nodes=False):
    """Gradients of `synapse_step` (kernels/synapse_step.py:184-330): returns
    `(g_v (B, n), g_s (B, E) or None, [g_param (E,) summed over the batch])`."""
    v = np.asarray(v, dtype=np.float64)
    B, n = v.shape
    E = len(pre)
    T = E // k
    pre = np.asarray(pre)
    node = np.arange(T) if targets_are_nodes else np.asarray(targets)
    vpre = v[:, pre]
    vp = np.repeat(v[:, node], k, axis=1)
    glin = np.repeat(g_lin, k, axis=1)
    gconst = np.repeat(g_const, k, axis=1)
    gs = params[0][None]
    area = area[None]
    if model == 0:
        e_syn, alpha, beta, v_th, delta = (p[None] for p in params[1:6])
        x = (vpre - v_th) / delta
        transmitter = _sigmoid(x)
        a = alpha * transmitter
        rate = a + beta
        s_inf = a / rate
        decay = np.exp(-dt * rate)
        s_new = s_inf + (s - s_inf) * decay
        w0 = vp - e_syn
        w1 = (vp + diff) - e_syn
        i0 = gs * s_new * w0
        i1 = gs * s_new * w1
    else:
        x_offset, slope = params[1][None], params[2][None]
        u0 = vpre - x_offset
        u1 = (vpre + diff) - x_offset
        sig0 = _sigmoid(u0 * slope)
        sig1 = _sigmoid(u1 * slope)
        i0 = -gs * sig0
        i1 = -gs * sig1
    d0 = i0 / area * 100000.0
    d1 = i1 / area * 100000.0
    vt = (d1 - d0) / diff
    g_vt = glin - gconst * vp
    g_vp = -gconst * vt
    g_d1 = g_vt / diff
    g_d0 = gconst - g_d1
    g_i0 = g_d0 * 100000.0 / area
    g_i1 = g_d1 * 100000.0 / area
    if g_current is not None:
        g_i0 = g_i0 + g_current
    g_params = []
    g_s = None
    if model == 0:
        g_w = g_i0 * w0 + g_i1 * w1
        g_sn = gs * g_w
        if g_s_new is not None:
            g_sn = g_sn + g_s_new
        g_vp = g_vp + gs * s_new * (g_i0 + g_i1)
        g_sinf = g_sn * (1.0 - decay)
        g_rate = -dt * decay * g_sn * (s - s_inf) - g_sinf * s_inf / rate
        g_a = g_sinf / rate + g_rate
        g_x = g_a * alpha * transmitter * (1.0 - transmitter)
        g_vpre = g_x / delta
        g_s = g_sn * decay
        g_params = [
            (s_new * g_w).sum(0),
            (-gs * s_new * (g_i0 + g_i1)).sum(0),
            (g_a * transmitter).sum(0),
            g_rate.sum(0),
            (-g_vpre).sum(0),
            (-g_vpre * x).sum(0),
        ]
    else:
        g_z0 = -gs * g_i0 * sig0 * (1.0 - sig0)
        g_z1 = -gs * g_i1 * sig1 * (1.0 - sig1)
        g_vpre = (g_z0 + g_z1) * slope
        g_params = [
            (-(g_i0 * sig0 + g_i1 * sig1)).sum(0),
            (-g_vpre).sum(0),
            (g_z0 * u0 + g_z1 * u1).sum(0),
        ]
    g_v = np.zeros((B, n))
    np.add.at(g_v.T, pre, g_vpre.T)
    gpost = g_vp.reshape(B, T, k).sum(-1)
    np.add.at(g_v.T, node, gpost.T)
    return g_v, g_s, g_params


# --------------------------------------------------------------------------------------
# One step and the loop (modules/base.py:3214-3400, integrate.py:396-666)
# --------------------------------------------------------------------------------------
def _bn(a, B, n):
    a = np.asarray(a, dtype=np.float64)
    return np.broadcast_to(a, (B, n)).copy() if a.shape != (B, n) else a.copy()


def init_steady_states(problem, states: Dict[str, np.ndarray]):
    """`Module.init_states` (modules/base.py:2419-2474): every channel in insertion
    order is set to its steady state at the current voltage (with the parameters of
    the module, no batch)."""
    states = {k: np.array(v, dtype=np.float64, copy=True) for k, v in states.items()}
    for ch in problem.channels:
        inds = np.asarray(ch.inds)
        v = states["v"][..., inds]
        prm = {p: np.asarray(problem.params[p])[..., inds] for p in ch.params}
        for key, val in channel_init(ch, v, prm).items():
            states[key][..., inds] = val
    return states


class _Stepper:
    def __init__(self, problem, B):
        self.p = problem
        self.B = B
        n = problem.n_nodes
        self.n = n
        self.comp = np.asarray(problem.comp_inds)
        self.cm = _bn(problem.params["capacitance"], B, n)
        self.area = _bn(problem.params["area"], B, n)
        self.ch_params = []
        for ch in problem.channels:
            inds = np.asarray(ch.inds)
            self.ch_params.append(
                {q: _bn(problem.params[q], B, n)[:, inds] for q in ch.params}
            )
        self.parent = np.asarray(problem.parent_lookup)
        self.depth = _depth(self.parent)
        ax = np.asarray(problem.axial, dtype=np.float64)
        self.axial = np.broadcast_to(ax, (B, ax.shape[-1])) if ax.ndim == 2 else ax[None]
        self.cur_names = list(problem.current_names)

    def channel_currents(self, st, v):
        """Currents with the finite-difference slope (modules/base.py:3445-3542); also
        writes the current states. Returns `(lin, const)` in uA/cm^2."""
        p, B, n = self.p, self.B, self.n
        lin = np.zeros((B, n))
        const = np.zeros((B, n))
        cur_states = {k: np.zeros((B, n)) for k in self.cur_names}
        for ch, prm in zip(p.channels, self.ch_params):
            inds = np.asarray(ch.inds)
            chs = {k: st[k][:, inds] for k in ch.states}
            vv = v[:, inds]
            i0 = np.broadcast_to(channel_current(ch, chs, vv, prm), vv.shape)
            i1 = np.broadcast_to(channel_current(ch, chs, vv + DIFF, prm), vv.shape)
            voltage_term = (i1 - i0) / DIFF
            constant_term = i0 - voltage_term * vv
            np.add.at(lin.T, inds, voltage_term.T)
            np.add.at(const.T, inds, (-constant_term).T)
            np.add.at(cur_states[ch.current].T, inds, i0.T)
        for k in self.cur_names:
            st[k] = cur_states[k]
        return lin * 1000.0, const * 1000.0

    def step(self, st: Dict[str, np.ndarray], t: int) -> Dict[str, np.ndarray]:
        p, B, n, dt = self.p, self.B, self.n, self.p.dt
        st = dict(st)
        v = st["v"]
        # Stimulus, modules/base.py:3234-3242 (nA -> uA/cm^2, cell_utils.py:275-288).
        i_ext = np.zeros((B, n))
        if p.stim is not None and len(p.stim_inds):
            i_t = np.broadcast_to(p.stim[:, :, t], (B, len(p.stim_inds)))
            cur = i_t / self.area[:, p.stim_inds] * 100_000
            np.add.at(i_ext.T, p.stim_inds, cur.T)
        # Channel states, sequential over channels (modules/base.py:3414-3443).
        for ch, prm in zip(p.channels, self.ch_params):
            inds = np.asarray(ch.inds)
            names = list(dict.fromkeys(list(ch.states) + self.cur_names))
            chs = {k: st[k][:, inds] for k in names if k in st}
            upd = channel_update(ch, chs, dt, v[:, inds], prm)
            for key, val in upd.items():
                arr = st[key].copy()
                arr[:, inds] = val
                st[key] = arr
        lin, const = self.channel_currents(st, v)
        # Synapses (modules/network.py:350-478).
        syn_lin = np.zeros((B, n))
        syn_const = np.zeros((B, n))
        for syn in p.synapses:
            s_old = None
            if syn.model == 0:
                s_old = np.broadcast_to(st[f"{syn.name}_s"], (B, len(syn.pre)))
            area_post = self.area[0, syn.post]
            s_new, i0, l_t, c_t = synapse_step(
                syn.model, v, s_old, syn.pre, syn.targets, syn.k, syn.params,
                area_post, dt,
            )
            if syn.model == 0:
                st[f"{syn.name}_s"] = s_new
            if f"i_{syn.name}" in st:
                st[f"i_{syn.name}"] = i0
            np.add.at(syn_lin.T, syn.targets, l_t.T)
            np.add.at(syn_const.T, syn.targets, (-c_t).T)
        # Clamps of channel and synapse states after their step (modules/base.py:3305-3308).
        for name, nodes, vals in getattr(p, "clamps", []) or []:
            if name != "v":
                st[name] = self._clamped(st[name], nodes, vals, t)
        # Assemble (modules/base.py:3257-3264) and solve (solver_voltage.py:250-359).
        lin_t = (lin + syn_lin) / self.cm
        const_t = (const + i_ext + syn_const) / self.cm
        if getattr(p, "solver", "bwd_euler") == "crank_nicolson":
            # half a step of the implicit system, then v' = 2 v_half - v (base.py:3327-3365)
            st["v"] = 2.0 * self._solve(v, lin_t, const_t, dt=p.dt / 2) - v
        else:
            st["v"] = self._solve(v, lin_t, const_t)
        # Voltage clamps after the solve (modules/base.py:3396-3398).
        for name, nodes, vals in getattr(p, "clamps", []) or []:
            if name == "v":
                st["v"] = self._clamped(st["v"], nodes, vals, t)
        return st

    def _clamped(self, arr, nodes, vals, t):
        """`arr (B, n)` with the clamp values of step t set at `nodes` (`_set_last`:
        of repeated nodes the later entry wins)."""
        out = np.array(arr, dtype=np.float64, copy=True)
        vt = np.broadcast_to(np.asarray(vals)[..., t], (self.B, len(nodes)))
        for q, node in enumerate(np.asarray(nodes)):
            out[:, node] = vt[:, q]
        return out

    def _solve(self, v, lin, const, dt=None):
        p, B, n = self.p, self.B, self.n
        dt = p.dt if dt is None else dt
        ax = dt * self.axial
        diags = dt * lin
        diags[:, self.comp] += 1.0
        if ax.shape[-1] > 0:
            np.add.at(diags.T, np.asarray(p.sinks), np.broadcast_to(ax, (B, ax.shape[-1])).T)
        solves = np.zeros((B, n))
        solves[:, self.comp] = v[:, self.comp] + dt * const[:, self.comp]
        if ax.shape[-1] == 0:
            return solves / diags
        lu = np.broadcast_to(-ax, (B, ax.shape[-1]))
        order = np.asarray(p.to_solve)
        d = diags[:, order]
        s = solves[:, order]
        lo = lu[:, p.map_lower]
        up = lu[:, p.map_upper]
        root = self.parent < 0
        lo = np.where(root, 0.0, lo)
        up = np.where(root, 0.0, up)
        x = tree_solve(d, lo, up, s, self.parent, self.depth)
        out = np.empty_like(x)
        out[:, order] = x
        return out


def integrate(problem, n_steps: Optional[int] = None, return_states: bool = False,
              init_steady: bool = False):
    """`jx.integrate` for a `Problem` (integrate.py:396-666): recordings of shape
    `(B, n_rec, n_steps + 1)`, the first sample being the initial state.

    The initial channel currents are recomputed from the initial states
    (`_append_currents_with_plan`, modules/base.py:2375-2383); with `init_steady`,
    every channel first goes to its steady state (`Module.init_states`)."""
    B = problem.batch
    n = problem.n_nodes
    T = problem.n_steps if n_steps is None else n_steps
    st = {}
    for k, v in problem.states.items():
        st[k] = _bn(v, B, v.shape[-1]) if np.asarray(v).ndim else np.asarray(v)
    for syn in problem.synapses:
        if syn.model == 0:
            st[f"{syn.name}_s"] = _bn(syn.state, B, len(syn.pre))
        if syn.current is not None:
            st[f"i_{syn.name}"] = _bn(syn.current, B, len(syn.pre))
    stepper = _Stepper(problem, B)
    if init_steady:
        st = init_steady_states(problem, st)
    stepper.channel_currents(st, st["v"])

    def record(s):
        return np.stack([s[name][:, idx] for name, idx in problem.recordings], axis=1)

    recs = [record(st)]
    for t in range(T):
        st = stepper.step(st, t)
        recs.append(record(st))
    out = np.stack(recs, axis=-1)
    return (out, st) if return_states else out
