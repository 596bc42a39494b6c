"""Seeded synthetic problems of the benchmark configurations (no dataset involved).

`morphology()` builds what `jx.Cell(branches, parents)` builds (modules/cell.py,
`_init_comp_graph`): cylindrical compartments, one branchpoint node at the end of
every branch that has children, compartment edges of the five reference types and
their axial conductances (utils/morph_attributes.py:315-436, restated below). The
nodes are numbered in a breadth-first solve order (parents before children), so
`to_solve` is the identity.

Configurations (sizes from the benchmark description):

* `config_small`: 1 branch x 8 compartments, HH, step current at compartment 0,
  401 steps, float64, forward only.
* `config_l5pc_tree`: a near-balanced random binary tree of 300 branches x 4
  compartments (1200 compartments + branchpoints, height 35-45), branch lengths
  lognormal(ln 30 um, 0.5), radii tapering 2 -> 0.3 um with branch depth, the L5PC
  channel set (soma: NaTs2T, SKv3_1, SKE2, CaNernstReversal, CaPump, CaHVA, CaLVA;
  dendrites: NaTs2T, SKv3_1, M, H; Leak everywhere) with every conductance scaled by
  U[0.5, 1.5] per parameter set; batch 256, dt 0.025 ms, 4000 steps.
* `config_uneven`: 4096 cells of log-uniform(4, 3000) compartments and depth 1-60,
  HH or L5PC, each with its own step current (1 ms, delay U[1, 5] ms, amplitude
  U[0.05, 0.5] nA) and its own trainable conductances (one column per cell and
  conductance), 2000 steps.
"""
from __future__ import annotations

import bisect
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from .channels import SPECS, ChannelInstance, make_instance
from .problem import Problem, SynapseType

PI = np.pi


class CompIndex:
    """Node of compartment `(branch, comp)` of a cell: `index[(b, k)]`."""

    def __init__(self, start: np.ndarray, ncomp: np.ndarray):
        self.start, self.ncomp = start, ncomp

    def __getitem__(self, bk):
        b, k = int(bk[0]), int(bk[1])
        if not 0 <= k < int(self.ncomp[b]):
            raise KeyError(bk)
        return int(self.start[b]) + k


def morphology(branch_parents: Sequence[int], ncomp: Sequence[int], comp_radius: Sequence[np.ndarray],
               comp_length: Sequence[np.ndarray], r_a: float = 5000.0, cm: float = 1.0):
    """Nodes and the tree system of one cell. Returns a dict of node-order arrays
    (node order = solve order) and the compartment index of every (branch, comp).

    Branches are numbered breadth first; a branch contributes its compartments and,
    when it has children, one branchpoint node after them."""
    nb = len(branch_parents)
    bpar = np.asarray(branch_parents, dtype=np.int64)
    nc = np.asarray(ncomp, dtype=np.int64)
    children: List[List[int]] = [[] for _ in range(nb)]
    for b in range(1, nb):
        children[int(bpar[b])].append(b)
    bfs = [0]
    qi = 0
    while qi < len(bfs):
        bfs.extend(children[bfs[qi]])
        qi += 1
    bfs = np.asarray(bfs, dtype=np.int64)
    has_kids = np.bincount(bpar[1:], minlength=nb) > 0 if nb > 1 else np.zeros(nb, dtype=bool)
    size = nc + has_kids
    start = np.zeros(nb, dtype=np.int64)
    start[bfs] = np.concatenate([[0], np.cumsum(size[bfs])[:-1]])
    n = int(size.sum())
    bp_of = start + nc  # branchpoint node of a branch with children
    is_comp = np.ones(n, dtype=bool)
    is_comp[bp_of[has_kids]] = False
    parent = np.arange(-1, n - 1, dtype=np.int64)  # within a branch: the previous node
    first = start[bfs]
    parent[first] = np.where(bpar[bfs] >= 0, bp_of[np.maximum(bpar[bfs], 0)], -1)
    radius = np.ones(n)
    length = np.ones(n)
    cidx = np.repeat(start, nc) + (np.arange(int(nc.sum())) - np.repeat(np.cumsum(nc) - nc, nc))
    radius[cidx] = np.concatenate([np.asarray(comp_radius[b], dtype=np.float64)[:nc[b]] for b in range(nb)])
    length[cidx] = np.concatenate([np.asarray(comp_length[b], dtype=np.float64)[:nc[b]] for b in range(nb)])
    area = 2 * PI * radius * length
    rl = (length / 2) / (radius**2 * PI)  # resistive load of half a compartment
    ra = np.full(n, float(r_a))
    cmv = np.full(n, float(cm))
    # Axial conductances per directed edge (sink row), utils/morph_attributes.py:380-433.
    g_low = np.zeros(n)  # sink = node j, source = parent
    g_up = np.zeros(n)  # sink = parent, source = node j
    j = np.arange(1, n)
    p = parent[j]
    cc = is_comp[j] & is_comp[p]  # compartment to compartment
    c2bp = ~is_comp[j]  # j is a branchpoint, its parent a compartment
    r_cc = rl[p] * ra[p] + rl[j] * ra[j]
    r_pc = rl[p] * ra[p]
    r_jc = rl[j] * ra[j]  # compartment whose parent is a branchpoint
    g_low[j] = np.where(cc, 1 / r_cc / area[j] / cmv[j] * 1e7,
                        np.where(c2bp, 1 / r_pc, 1 / r_jc / area[j] / cmv[j] * 1e7))
    g_up[j] = np.where(cc, 1 / r_cc / area[p] / cmv[p] * 1e7,
                       np.where(c2bp, 1 / r_pc / area[p] / cmv[p] * 1e7, 1 / r_jc))
    depth_of_branch = np.zeros(nb, dtype=np.int64)
    for b in bfs[1:]:
        depth_of_branch[b] = depth_of_branch[bpar[b]] + 1
    return {
        "n": n, "parent": parent, "is_comp": is_comp, "area": area, "cm": cmv,
        "radius": radius, "length": length, "g_low": g_low, "g_up": g_up,
        "comp_node": CompIndex(start, nc), "branch_depth": depth_of_branch,
    }


def _edges(parent: np.ndarray, g_low: np.ndarray, g_up: np.ndarray):
    """Compartment-edge arrays (sinks, axial) and the lower/upper maps."""
    n = len(parent)
    nonroot = np.nonzero(parent >= 0)[0]
    m = len(nonroot)
    sinks = np.concatenate([nonroot, parent[nonroot]])
    axial = np.concatenate([g_low[nonroot], g_up[nonroot]])
    map_lower = np.zeros(n, dtype=np.int64)
    map_upper = np.zeros(n, dtype=np.int64)
    map_lower[nonroot] = np.arange(m)
    map_upper[nonroot] = m + np.arange(m)
    return sinks, axial, map_lower, map_upper


def assemble(cells: List[dict], channels_per_cell: List[List[Tuple[str, np.ndarray, str, Dict[str, object]]]],
             batch: int, dt: float, n_steps: int, v0: float = -70.0,
             stim: Optional[List[Tuple[int, Tuple[int, int], np.ndarray]]] = None,
             recordings: Optional[List[Tuple[str, int, Tuple[int, int]]]] = None) -> Problem:
    """Concatenate cells into one problem (a network without synapses).

    `channels_per_cell[c]` lists `(type, local node indices, instance name,
    {param name: value (scalar, (n_local,), or (batch, n_local))})` in insertion order;
    channels with the same instance name across cells are merged, as the reference
    merges equally named channels of a network. `stim` holds
    `(cell, (branch, comp), samples (batch or 1, steps))`, `recordings`
    `(state, cell, (branch, comp))`.
    """
    offs = np.cumsum([0] + [c["n"] for c in cells])
    N = int(offs[-1])
    parent = np.concatenate([np.where(c["parent"] >= 0, c["parent"] + o, -1) for c, o in zip(cells, offs)])
    g_low = np.concatenate([c["g_low"] for c in cells])
    g_up = np.concatenate([c["g_up"] for c in cells])
    sinks, axial, map_lower, map_upper = _edges(parent, g_low, g_up)
    is_comp = np.concatenate([c["is_comp"] for c in cells])
    params: Dict[str, np.ndarray] = {
        "capacitance": np.concatenate([c["cm"] for c in cells]),
        "area": np.concatenate([c["area"] for c in cells]),
        "radius": np.concatenate([c["radius"] for c in cells]),
        "length": np.concatenate([c["length"] for c in cells]),
    }
    states: Dict[str, np.ndarray] = {"v": np.full(N, float(v0))}
    inst: Dict[str, ChannelInstance] = {}
    order: List[str] = []
    pending: Dict[str, List[Tuple[np.ndarray, Dict[str, object]]]] = {}
    for c, chans in enumerate(channels_per_cell):
        for type_name, local, name, values in chans:
            glob = np.asarray(local, dtype=np.int64) + offs[c]
            if name not in inst:
                inst[name] = make_instance(type_name, np.zeros(0, np.int64), name=name,
                                           constants=values.get("__constants__"))
                order.append(name)
                pending[name] = []
            pending[name].append((glob, values))
    current_names: List[str] = []
    for name in order:
        ch = inst[name]
        spec = SPECS[ch.type_name]
        inds = np.concatenate([g for g, _ in pending[name]])
        ch.inds = inds
        for (suffix, default), pname in zip(spec.params, ch.params):
            if pname not in params:
                params[pname] = np.full(N, float(default))
        for (suffix, default), sname in zip(spec.states, ch.states):
            if sname not in states:
                states[sname] = np.full(N, np.nan)
            states[sname][inds] = np.where(np.isnan(states[sname][inds]), float(default),
                                           states[sname][inds])
        for glob, values in pending[name]:
            for key, val in values.items():
                if key == "__constants__":
                    continue
                val = np.asarray(val, dtype=np.float64)
                if val.ndim == 2 or params[key].ndim == 2:
                    if params[key].ndim == 1:
                        params[key] = np.broadcast_to(params[key], (batch, N)).copy()
                    params[key][:, glob] = np.broadcast_to(val, (batch, len(glob)))
                else:
                    params[key][glob] = val
        if ch.current not in current_names:
            current_names.append(ch.current)
    for cn in current_names:
        states[cn] = np.zeros(N)
    for k in list(states):
        states[k] = np.where(np.isnan(states[k]), 0.0, states[k])
    stim_inds, stim_arr = np.zeros(0, np.int64), None
    if stim:
        stim_inds = np.asarray([offs[c] + cells[c]["comp_node"][bc] for c, bc, _ in stim], dtype=np.int64)
        rows = max(np.atleast_2d(s).shape[0] for _, _, s in stim)
        stim_arr = np.zeros((rows, len(stim), n_steps))
        for q, (_, _, s) in enumerate(stim):
            s = np.atleast_2d(np.asarray(s, dtype=np.float64))
            L = min(n_steps, s.shape[1])
            stim_arr[:, q, :L] = s[:, :L]
    recs = []
    for name, c, bc in recordings or []:
        recs.append((name, int(offs[c] + cells[c]["comp_node"][bc])))
    return Problem(
        n_nodes=N, comp_inds=np.nonzero(is_comp)[0], sinks=sinks, axial=axial,
        parent_lookup=parent, to_solve=np.arange(N), map_lower=map_lower, map_upper=map_upper,
        channels=[inst[n] for n in order], params=params, states=states, dt=float(dt),
        n_steps=int(n_steps), stim_inds=stim_inds, stim=stim_arr, recordings=recs,
        batch=int(batch), current_names=current_names,
    )


def step_current(i_delay: float, i_dur: float, i_amp, delta_t: float, t_max: float) -> np.ndarray:
    """Step current of `int(t_max // delta_t) + 2` samples (stimulus.py:8-36): on for
    the samples from `int(i_delay / delta_t)` up to, not including,
    `int((i_delay + i_dur) / delta_t)` (both truncated, as the reference does)."""
    n = int(t_max // delta_t) + 2
    on = np.zeros(n)
    on[int(i_delay / delta_t):int((i_delay + i_dur) / delta_t)] = 1.0
    amp = np.asarray(i_amp, dtype=np.float64).reshape(-1, 1)
    return amp * on[None]


def config_small() -> Problem:
    cell = morphology([-1], [8], [np.full(8, 1.0)], [np.full(8, 10.0)])
    nodes = np.arange(cell["n"])
    prob = assemble([cell], [[("HH", nodes, "HH", {})]], batch=1, dt=0.025, n_steps=401,
                    stim=[(0, (0, 0), step_current(1.0, 1.0, 0.1, 0.025, 10.0))],
                    recordings=[("v", 0, (0, 0))])
    return prob


def balanced_random_tree(n_branches: int, rng: np.random.Generator, skew: float = 0.7) -> List[int]:
    """A random binary tree of `n_branches` branches, grown by attaching every new
    branch to an open slot: with probability `skew` to a slot of the shallowest
    branches, else to any open slot."""
    parents = [-1]
    depth = [0]
    nchild = [0]
    for b in range(1, n_branches):
        open_ = [q for q in range(b) if nchild[q] < 2]
        if rng.random() < skew:
            dmin = min(depth[q] for q in open_)
            cand = [q for q in open_ if depth[q] == dmin]
        else:
            cand = open_
        p = int(rng.choice(cand))
        parents.append(p)
        depth.append(depth[p] + 1)
        nchild[p] += 1
        nchild.append(0)
    return parents


def tree_height(parent: np.ndarray) -> int:
    n = len(parent)
    h = np.zeros(n, dtype=np.int64)
    for j in range(n - 1, 0, -1):
        p = parent[j]
        h[p] = max(h[p], h[j] + 1)
    return int(h.max()) if n else 0


L5PC_SOMA = [
    ("NaTs2T", "somatic_NaTs2T", {"somatic_NaTs2T_gNaTs2T": 0.983955}),
    ("SKv3_1", "somatic_SKv3_1", {"somatic_SKv3_1_gSKv3_1": 0.303472}),
    ("SKE2", "somatic_SKE2", {"somatic_SKE2_gSKE2": 0.008407}),
    ("CaNernstReversal", "CaNernstReversal", {"__constants__": {"T": 307.15}}),
    ("CaPump", "somatic_CaPump", {"somatic_CaPump_gamma": 0.000609, "somatic_CaPump_decay": 210.485291}),
    ("CaHVA", "somatic_CaHVA", {"somatic_CaHVA_gCaHVA": 0.000994}),
    ("CaLVA", "somatic_CaLVA", {"somatic_CaLVA_gCaLVA": 0.000333}),
]
L5PC_DEND = [
    ("NaTs2T", "apical_NaTs2T", {"apical_NaTs2T_gNaTs2T": 0.026145}),
    ("SKv3_1", "apical_SKv3_1", {"apical_SKv3_1_gSKv3_1": 0.004226}),
    ("M", "apical_M", {"apical_M_gM": 0.000143}),
    ("H", "apical_H", {"apical_H_gH": 8e-5}),
]
# Parameters that every parameter set scales by U[0.5, 1.5].
L5PC_SCALED = [
    "somatic_NaTs2T_gNaTs2T", "somatic_SKv3_1_gSKv3_1", "somatic_SKE2_gSKE2",
    "somatic_CaHVA_gCaHVA", "somatic_CaLVA_gCaLVA", "apical_NaTs2T_gNaTs2T",
    "apical_SKv3_1_gSKv3_1", "apical_M_gM", "apical_H_gH", "Leak_gLeak",
]


def l5pc_channels(cell: dict, scales: Optional[Dict[str, np.ndarray]] = None, ncomp_soma: int = 4):
    """Channel list of one L5PC-like cell: soma = the first branch's compartments."""
    soma = np.asarray([cell["comp_node"][(0, k)] for k in range(ncomp_soma)])
    comps = np.nonzero(cell["is_comp"])[0]
    dend = np.setdiff1d(comps, soma)
    scales = scales or {}

    def vals(d):
        out = {}
        for k, v in d.items():
            if k == "__constants__":
                out[k] = v
            elif k in scales:
                out[k] = np.asarray(v) * np.asarray(scales[k])[:, None]
            else:
                out[k] = v
        return out

    chans = [(t, soma, name, vals(v)) for t, name, v in L5PC_SOMA]
    chans += [(t, dend, name, vals(v)) for t, name, v in L5PC_DEND]
    leak = {"Leak_gLeak": 3e-05, "Leak_eLeak": -75.0}
    chans.append(("Leak", comps, "Leak", vals(leak)))
    return chans


def config_l5pc_tree(batch: int = 256, n_branches: int = 300, ncomp: int = 4, n_steps: int = 4000,
                     seed: int = 0, height_range=(35, 45), stim_amp: float = 0.3,
                     scale_seed: int = 1, stim_delay: float = 10.0) -> Problem:
    """The large-batch L5PC-like tree. `prob.meta` keeps what rebuilds the same cell
    elsewhere: branch parents, lengths and radii, the per-row conductance scales and
    the stimulus `(delay, duration, amplitude)`."""
    rng = np.random.default_rng(seed)
    for _ in range(1000):
        parents = balanced_random_tree(n_branches, rng)
        lengths = rng.lognormal(np.log(30.0), 0.5, size=n_branches)
        depth = np.zeros(n_branches, dtype=np.int64)
        for b in range(1, n_branches):
            depth[b] = depth[parents[b]] + 1
        dmax = max(int(depth.max()), 1)
        radius = 2.0 - (2.0 - 0.3) * depth / dmax
        cell = morphology(parents, [ncomp] * n_branches,
                          [np.full(ncomp, r) for r in radius],
                          [np.full(ncomp, L / ncomp) for L in lengths], r_a=100.0)
        h = tree_height(cell["parent"])
        if height_range[0] <= h <= height_range[1]:
            break
    else:
        raise RuntimeError("no tree within the height range")
    srng = np.random.default_rng(scale_seed)
    scales = {k: srng.uniform(0.5, 1.5, size=batch) for k in L5PC_SCALED}
    chans = l5pc_channels(cell, scales, ncomp_soma=ncomp)
    t_max = n_steps * 0.025
    prob = assemble([cell], [chans], batch=batch, dt=0.025, n_steps=n_steps, v0=-65.0,
                    stim=[(0, (0, 0), step_current(stim_delay, 80.0, stim_amp, 0.025, t_max))],
                    recordings=[("v", 0, (0, 0))])
    prob.states.setdefault("CaCon_e", np.full(prob.n_nodes, 2.0))
    prob.states["CaCon_i"] = np.where(prob.states.get("CaCon_i", np.zeros(prob.n_nodes)) == 0,
                                      5e-05, prob.states["CaCon_i"])
    prob.states["CaCon_e"] = np.where(prob.states["CaCon_e"] == 0, 2.0, prob.states["CaCon_e"])
    for k in ["eNa", "eK"]:
        if k in prob.params:
            prob.params[k] = np.full(prob.n_nodes, 50.0 if k == "eNa" else -85.0)
    prob.meta = {"height": h, "scales": scales, "parents": parents, "lengths": lengths,
                 "radius": radius, "ncomp": ncomp, "stim": (stim_delay, 80.0, stim_amp)}
    return prob


def config_uneven(n_cells: int = 4096, seed: int = 0, n_steps: int = 2000, min_comp: int = 4,
                  max_comp: int = 3000, max_depth: int = 60, l5pc_fraction: float = 0.5) -> Problem:
    """Cells of log-uniform compartment counts and bounded depth, HH or L5PC."""
    rng = np.random.default_rng(seed)
    cells, chans, stims, recs = [], [], [], []
    train_local = []  # per cell: [(param name, local node indices)]
    specs = []  # per cell: what rebuilds it elsewhere
    t_max = n_steps * 0.025
    for c in range(n_cells):
        ncomp_total = int(round(np.exp(rng.uniform(np.log(min_comp), np.log(max_comp)))))
        ncomp = 4 if ncomp_total >= 4 else ncomp_total
        nb = max(1, ncomp_total // ncomp)
        depth_cap = int(rng.integers(1, max_depth + 1))
        parents = [-1]
        bdepth = [0]
        elig = [0] if depth_cap > 0 else []  # branches that may take children, increasing
        for b in range(1, nb):
            lo = bisect.bisect_left(elig, b - 64)  # a parent among the 64 previous branches
            p = elig[lo + int(rng.integers(0, len(elig) - lo))] if lo < len(elig) else 0
            parents.append(p)
            bdepth.append(bdepth[p] + 1)
            if bdepth[b] < depth_cap:
                elig.append(b)
        lengths = rng.lognormal(np.log(30.0), 0.5, size=nb)
        radius = np.clip(2.0 - 0.05 * np.asarray(bdepth), 0.3, 2.0)
        cell = morphology(parents, [ncomp] * nb, [np.full(ncomp, r) for r in radius],
                          [np.full(ncomp, L / ncomp) for L in lengths], r_a=100.0)
        cells.append(cell)
        if rng.random() < l5pc_fraction and nb > 1:
            cl = l5pc_channels(cell, None, ncomp_soma=ncomp)
            chans.append(cl)
            train_local.append([(k, nodes) for _, nodes, _, vals in cl for k in vals if k in L5PC_SCALED])
            kind = "L5PC"
        else:
            comps = np.nonzero(cell["is_comp"])[0]
            chans.append([("HH", comps, "HH", {})])
            train_local.append([(k, comps) for k in ("HH_gNa", "HH_gK", "HH_gLeak")])
            kind = "HH"
        delay = float(rng.uniform(1, 5))
        amp = float(rng.uniform(0.05, 0.5))
        specs.append({"parents": parents, "ncomp": ncomp, "radius": radius, "lengths": lengths,
                      "kind": kind, "stim": (delay, 1.0, amp),
                      "train": [k for k, _ in train_local[-1]]})
        stims.append((c, (0, 0), step_current(delay, 1.0, amp, 0.025, t_max)))
        recs.append(("v", c, (0, 0)))
    prob = assemble(cells, chans, batch=1, dt=0.025, n_steps=n_steps, v0=-65.0, stim=stims,
                    recordings=recs)
    offs = np.cumsum([0] + [c["n"] for c in cells])
    prob.trainable = [(k, np.asarray(nodes) + offs[c]) for c in range(n_cells)
                      for k, nodes in train_local[c]]
    if "CaCon_i" in prob.states:
        prob.states["CaCon_i"] = np.where(prob.states["CaCon_i"] == 0, 5e-05, prob.states["CaCon_i"])
    if "CaCon_e" in prob.states:
        prob.states["CaCon_e"] = np.where(prob.states["CaCon_e"] == 0, 2.0, prob.states["CaCon_e"])
    # The L5PC cells' reversal potentials, as in the large-batch tree (HH keeps its own
    # HH_eNa / HH_eK).
    for k, val in (("eNa", 50.0), ("eK", -85.0)):
        if k in prob.params:
            prob.params[k] = np.full(prob.n_nodes, val)
    prob.meta = {"cells": specs}
    return prob


def reference_l5pc_cell(jx, parents, ncomp: int, radius, lengths):
    """The L5PC-like cell of `l5pc_channels` built with the reference's own module
    API (`jx` is the imported `jaxley_pytorch`): soma = branch 0 (NaTs2T, SKv3_1,
    SKE2, CaNernstReversal at 307.15 K, CaPump, CaHVA, CaLVA), dendrites = the other
    branches (NaTs2T, SKv3_1, M, H), Leak everywhere, axial resistivity 100 ohm cm,
    eNa 50 mV, eK -85 mV, v -65 mV; branch b has radius `radius[b]` and length
    `lengths[b]` split over its `ncomp` compartments (`examples/paper/
    fig2_l5pc_synthetic.py:100-152` sets up the same channel sets)."""
    from jaxley_pytorch.channels.pospischil import Leak
    from jaxley_pytorch.mech.channels import l5pc as ref_l5pc

    nb = len(parents)
    cell = jx.Cell([jx.Branch(jx.Compartment(), ncomp)] * nb, parents=list(parents))
    for b in range(nb):
        cell.branch(b).set("radius", float(radius[b]))
        cell.branch(b).set("length", float(lengths[b] / ncomp))
    cell.set("axial_resistivity", 100.0)
    for t, name, vals in L5PC_SOMA:
        if t == "CaNernstReversal":
            ch = ref_l5pc.CaNernstReversal()
            ch.channel_constants["T"] = 307.15
        else:
            ch = getattr(ref_l5pc, t)().change_name(name)
        cell.branch(0).insert(ch)
    cell.branch(0).set("CaCon_i", 5e-05)
    cell.branch(0).set("CaCon_e", 2.0)
    if nb > 1:
        dend = cell.branch(list(range(1, nb)))
        for t, name, vals in L5PC_DEND:
            dend.insert(getattr(ref_l5pc, t)().change_name(name))
    cell.insert(Leak())
    leak = ("Leak", "Leak", {"Leak_gLeak": 3e-05, "Leak_eLeak": -75.0})
    for t, name, vals in L5PC_SOMA + (L5PC_DEND if nb > 1 else []) + [leak]:
        for k, v in vals.items():
            if k != "__constants__":
                cell.set(k, v)
    cell.set("eNa", 50.0)
    cell.set("eK", -85.0)
    cell.set("v", -65.0)
    return cell
