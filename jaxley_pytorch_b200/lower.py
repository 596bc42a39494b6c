"""Lowering of a `Problem` into the flat arrays the CUDA simulation kernels read.

The reference keeps every state as a `(B, n_nodes)` array in node order and solves
the voltage system in the DHS solve order (`modules/base.py:1142-1266`). The kernels
use a third order, the *chain order*: every tree of the solve-order forest is cut into
chains (a node whose only child continues the chain), chains are laid out
parent-chain first and the nodes of a chain consecutively, so that one thread can
eliminate a chain in registers. Trees are packed into blocks (one CTA each).

Per node the state lives in a contiguous run of slots (slot 0 = v, then the states
of the node's channels and the channel currents): the state of one batch row is a
vector of `n_slots` values, and a block of trees is a contiguous range of it.
Parameters are `base[slot] * scale[b, col[slot]]` (column 0 is 1): parameters that
vary over the batch (``data_set`` with a batch dimension) get one column per
distinct batch profile, which is what the adjoint returns gradients for.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import numpy as np

from .channels import SPECS
from .problem import Problem

ENTRY_SHORTS = 18  # ChanEntry: type, ns, np, cur, s[6], p[8]


@dataclass
class Lowered:
    n_nodes: int
    batch: int
    int2node: np.ndarray  # internal index -> reference node index
    node2int: np.ndarray
    # topology (internal order)
    a_low: np.ndarray
    a_up: np.ndarray
    gsum: np.ndarray
    cm: np.ndarray
    area: np.ndarray
    node_class: np.ndarray
    soff: np.ndarray
    poff: np.ndarray  # (n_nodes,) first parameter slot of every node (shared runs)
    cls_ptr: np.ndarray
    cls_comp: np.ndarray
    cls_prog: np.ndarray  # (n_classes,) compile-time program id (0 = interpreted)
    entries: np.ndarray  # (n_entries, 18) int16
    pbase: np.ndarray
    pcol: np.ndarray
    pscale: np.ndarray  # (B, n_cols)
    col_info: List[Tuple[str, int]]  # (param name, reference node of first use) per column
    col_members: List[List[Tuple[str, int, float]]]  # (param name, node, base) per column
    # chains and blocks
    chain_top: np.ndarray
    chain_len: np.ndarray
    chain_ptop: np.ndarray
    chain_cptr: np.ndarray
    chain_child: np.ndarray
    level_ptr: np.ndarray
    blocks: np.ndarray  # (n_blocks, 12) int32 (JxbBlock)
    # stimulus / recordings
    stim_ptr: np.ndarray
    stim_idx: np.ndarray
    stim: Optional[np.ndarray]  # (steps, rows, n_stim) time-major
    gk: np.ndarray  # (n_pslots,) rank of a trainable parameter in its run, -1 if fixed
    gbase: np.ndarray  # (n_nodes,) first gradient slot of a node (block-relative)
    max_gslots: int  # largest number of gradient slots of a block
    parent: np.ndarray  # (n_nodes,) parent in internal order, -1 for roots
    kid_ptr: np.ndarray  # (n_nodes+1,) children CSR (internal order)
    kid: np.ndarray
    rec_ptr: np.ndarray
    rec_slot: np.ndarray
    rec_col: np.ndarray
    n_rec: int
    # state
    state0: np.ndarray  # (B, n_slots)
    slot_names: List[List[str]]  # per internal node
    dt: float
    n_steps: int
    max_levels: int = 0
    tree_ptr: np.ndarray = field(default_factory=lambda: np.zeros(1, np.int64))

    @property
    def n_slots(self) -> int:
        return int(self.soff[-1])

    @property
    def n_pslots(self) -> int:
        return int(len(self.pbase))

    @property
    def n_cols(self) -> int:
        return int(self.pscale.shape[1])


def _children(parent: np.ndarray) -> List[List[int]]:
    ch: List[List[int]] = [[] for _ in range(len(parent))]
    for j, p in enumerate(parent):
        if p >= 0:
            ch[p].append(j)
    return ch


def chain_order(parent: np.ndarray):
    """Chain decomposition of a solve-order forest.

    Returns `(order, trees, chains)`: `order[i]` is the solve index of chain-order
    node `i`; `trees` the chain-order start of every tree (plus the end);
    `chains` a list of `(top, length, parent_top_node, child_chain_ids)` in chain
    order (node indices in chain order).
    """
    parent = np.asarray(parent, dtype=np.int64)
    n = len(parent)
    roots = np.nonzero(parent < 0)[0]
    if n == 0 or len(roots) == 0 or roots[0] != 0:
        raise ValueError("the forest must start with a root")
    starts = roots
    ends = np.append(roots[1:], n)
    tree_of = np.repeat(np.arange(len(starts)), ends - starts)
    nonroot = parent >= 0
    idx = np.arange(n)
    if not (np.all(parent[nonroot] >= starts[tree_of[nonroot]]) and np.all(parent[nonroot] < idx[nonroot])):
        raise ValueError("every tree must be contiguous and parents must precede children")
    kids = _children(parent)
    order: List[int] = []
    chains: List[list] = []  # [top, len, ptop(chain order), [child chain ids]]
    trees = [0]
    for r in roots:
        queue = [(int(r), -1, -1)]  # (solve node, parent chain id, parent node chain order)
        qi = 0
        while qi < len(queue):
            node, pc, ptop = queue[qi]
            qi += 1
            cid = len(chains)
            top = len(order)
            cur = node
            order.append(cur)
            while len(kids[cur]) == 1:
                cur = kids[cur][0]
                order.append(cur)
            bot = len(order) - 1
            chains.append([top, bot - top + 1, ptop, []])
            if pc >= 0:
                chains[pc][3].append(cid)
            for c in kids[cur]:
                queue.append((c, cid, bot))
        trees.append(len(order))
    return np.asarray(order, dtype=np.int64), np.asarray(trees, dtype=np.int64), chains


def chain_levels(chains) -> np.ndarray:
    lev = np.zeros(len(chains), dtype=np.int64)
    for cid in range(len(chains) - 1, -1, -1):  # children come after parents
        kids = chains[cid][3]
        if kids:
            lev[cid] = 1 + max(lev[k] for k in kids)
    return lev


def pack_blocks(tree_ptr: np.ndarray, max_nodes: int, weights: Optional[np.ndarray] = None):
    """Consecutive trees packed into blocks of at most `max_nodes` nodes (a larger
    tree gets a block of its own)."""
    blocks = []
    s = 0
    for t in range(len(tree_ptr) - 1):
        a, b = int(tree_ptr[t]), int(tree_ptr[t + 1])
        if b - s > max_nodes and a > s:
            blocks.append((s, a))
            s = a
    blocks.append((s, int(tree_ptr[-1])))
    return blocks


# Compile-time programs of csrc/jxb_prog.cuh: channel type sequence -> id. A class
# runs one only if its slots and parameters have the program's consecutive layout.
PROGRAMS = {
    (SPECS["HH"].type_id,): 1,
    tuple(SPECS[t].type_id for t in ["NaTs2T", "SKv3_1", "M", "H", "Leak"]): 2,
}


def program_of(ents: np.ndarray) -> int:
    if len(ents) == 0:
        return 0
    prog = PROGRAMS.get(tuple(int(e[0]) for e in ents), 0)
    if not prog:
        return 0
    slot, par = 1, 0
    for e in ents:
        ns, npar, cur = int(e[1]), int(e[2]), int(e[3])
        if cur >= 0 or int(e[10]) != par:
            return 0
        if any(int(e[4 + q]) != slot + q for q in range(ns)):
            return 0
        slot += ns
        par += npar
    return prog


def lower(problem: Problem, max_block_nodes: int = 4096, dtype=np.float64,
          keep_currents: bool = True) -> Lowered:
    """Lower `problem`. With `keep_currents=False` a channel current gets a state slot
    only where a channel reads it (the calcium pump reads `i_Ca`) or it is recorded;
    the other currents are not kept in the resident state."""
    p = problem
    n = p.n_nodes
    B = p.batch
    parent_solve, g_low_s, g_up_s = p.solve_order_system()
    if np.asarray(g_low_s).ndim != 1:
        raise NotImplementedError("axial conductances with a batch dimension are not covered")
    order, tree_ptr, chains = chain_order(parent_solve)
    int2node = np.asarray(p.to_solve, dtype=np.int64)[order]
    node2int = np.empty(n, dtype=np.int64)
    node2int[int2node] = np.arange(n)
    solve2int = np.empty(n, dtype=np.int64)
    solve2int[order] = np.arange(n)

    def shared(name):
        a = np.asarray(p.params[name], dtype=np.float64)
        if a.ndim == 2:
            if not np.all(a == a[:1]):
                raise NotImplementedError(f"batched `{name}` is not covered")
            a = a[0]
        return a

    a_low = np.asarray(g_low_s, dtype=np.float64)[order]
    a_up = np.asarray(g_up_s, dtype=np.float64)[order]
    gsum = np.asarray(p.gsum(), dtype=np.float64)
    if gsum.ndim == 2:
        gsum = gsum[0]
    gsum = gsum[int2node]
    cm = shared("capacitance")[int2node]
    area = shared("area")[int2node]
    is_comp = np.zeros(n, dtype=bool)
    is_comp[np.asarray(p.comp_inds, dtype=np.int64)] = True

    # ---- node classes: channels, state slots and parameter slots of every node ----
    chan_at: List[List[int]] = [[] for _ in range(n)]
    for ci, ch in enumerate(p.channels):
        for r in np.asarray(ch.inds, dtype=np.int64):
            chan_at[int(r)].append(ci)

    cols: Dict[bytes, int] = {}
    col_vecs: List[np.ndarray] = [np.ones(B)]
    col_info: List[Tuple[str, int]] = [("", -1)]
    col_members: List[set] = [set()]

    def pval(name: str, r: int) -> Tuple[float, int]:
        a = np.asarray(p.params[name], dtype=np.float64)
        if a.ndim == 1:
            return float(a[r]), 0
        vec = np.broadcast_to(a[:, r], (B,))
        if np.all(vec == vec[0]):
            return float(vec[0]), 0
        base = float(vec[0]) if vec[0] != 0 else 1.0
        prof = vec / base
        key = name.encode() + b"|" + prof.tobytes()
        if key not in cols:
            cols[key] = len(col_vecs)
            col_vecs.append(prof)
            col_info.append((name, r))
            col_members.append(set())
        col_members[cols[key]].add((name, int(r), base))
        return base, cols[key]

    recorded = {(name, int(r)) for name, r in p.recordings}
    readers = {"CaPump"}  # channels whose update reads their current state

    classes: Dict[tuple, int] = {}
    cls_entries: List[np.ndarray] = []
    cls_comp: List[int] = []
    cls_nslots: List[int] = []
    node_class = np.zeros(n, dtype=np.int32)
    soff = np.zeros(n + 1, dtype=np.int64)
    node_pb: List[List[float]] = []
    node_pc: List[List[int]] = []
    slot_names: List[List[str]] = []
    for i in range(n):
        r = int(int2node[i])
        chs = chan_at[r]
        names = ["v"]
        for ci in chs:
            for s in p.channels[ci].states:
                if s not in names:
                    names.append(s)
        for ci in chs:
            cn = p.channels[ci].current
            need = (keep_currents or p.channels[ci].type_name in readers
                    or (cn, r) in recorded
                    or any(p.channels[cj].type_name in readers and p.channels[cj].current == cn
                           for cj in chs))
            if need and cn not in names:
                names.append(cn)
        ents = []
        pk = 0
        pbs: List[float] = []
        pcs: List[int] = []
        for ci in chs:
            ch = p.channels[ci]
            spec = SPECS[ch.type_name]
            e = np.zeros(ENTRY_SHORTS, dtype=np.int16)
            e[0] = spec.type_id
            e[1] = len(ch.states)
            e[2] = len(ch.params) + len(ch.constants)
            e[3] = names.index(ch.current) if ch.current in names else -1
            for q, s in enumerate(ch.states):
                e[4 + q] = names.index(s)
            e[10] = pk  # parameters are consecutive: p[0] is the first slot
            for q in range(int(e[2])):
                if 10 + q < ENTRY_SHORTS:
                    e[10 + q] = pk + q
            for q, pn in enumerate(ch.params):
                b, c = pval(pn, r)
                pbs.append(b)
                pcs.append(c)
            for cval in ch.constants:
                pbs.append(float(cval))
                pcs.append(0)
            pk += int(e[2])
            ents.append(e)
        key = (bool(is_comp[r]), tuple(names), tuple(tuple(e.tolist()) for e in ents))
        if key not in classes:
            classes[key] = len(cls_entries)
            cls_entries.append(np.stack(ents) if ents else np.zeros((0, ENTRY_SHORTS), np.int16))
            cls_comp.append(int(is_comp[r]))
            cls_nslots.append(len(names))
        node_class[i] = classes[key]
        soff[i + 1] = soff[i] + len(names)
        node_pb.append(pbs)
        node_pc.append(pcs)
        slot_names.append(names)
    cls_prog = np.asarray([program_of(e) for e in cls_entries], dtype=np.int32)
    cls_ptr = np.zeros(len(cls_entries) + 1, dtype=np.int32)
    for c, e in enumerate(cls_entries):
        cls_ptr[c + 1] = cls_ptr[c] + len(e)
    entries = (np.concatenate(cls_entries) if len(cls_entries) else np.zeros((0, ENTRY_SHORTS))).astype(np.int16)
    pscale = np.stack(col_vecs, axis=1) if B > 0 else np.ones((1, 1))

    # ---- initial state ----
    L = int(soff[-1])
    state0 = np.zeros((B, L), dtype=np.float64)
    for i in range(n):
        r = int(int2node[i])
        for k, nm in enumerate(slot_names[i]):
            a = np.asarray(p.states[nm], dtype=np.float64) if nm in p.states else None
            if a is None:
                continue
            state0[:, soff[i] + k] = a[..., r] if a.ndim == 1 else np.broadcast_to(a[:, r], (B,))

    # ---- blocks, chains ordered by level inside each block ----
    lev = chain_levels(chains)
    blocks_nodes = pack_blocks(tree_ptr, max_block_nodes)
    # Parameter blocks: nodes with identical parameters (values and columns) share
    # one run of parameter slots inside their block of trees.
    pbase: List[float] = []
    pcol: List[int] = []
    poff = np.zeros(n, dtype=np.int64)
    pranges = []
    for (n0, n1) in blocks_nodes:
        start = len(pbase)
        seen: Dict[tuple, int] = {}
        for i in range(n0, n1):
            key = (tuple(node_pb[i]), tuple(node_pc[i]))
            if key not in seen:
                seen[key] = len(pbase)
                pbase.extend(node_pb[i])
                pcol.extend(node_pc[i])
            poff[i] = seen[key]
        pranges.append((start, len(pbase) - start))
    chain_top, chain_len, chain_ptop, chain_cptr, chain_child = [], [], [], [0], []
    level_ptr: List[int] = []
    blocks = []
    tops = np.asarray([c[0] for c in chains], dtype=np.int64)
    cid_sorted = np.argsort(tops, kind="stable")
    tops_sorted = tops[cid_sorted]
    max_levels = 0
    for (n0, n1) in blocks_nodes:
        lo = np.searchsorted(tops_sorted, n0)
        hi = np.searchsorted(tops_sorted, n1)
        cids = cid_sorted[lo:hi]
        cids = cids[np.argsort(lev[cids], kind="stable")]
        nlev = int(lev[cids].max()) + 1 if len(cids) else 0
        max_levels = max(max_levels, nlev)
        chain0 = len(chain_top)
        level0 = len(level_ptr)
        counts = np.bincount(lev[cids], minlength=nlev)
        level_ptr.extend(np.concatenate([[0], np.cumsum(counts)]).tolist())
        for c in cids:
            top, ln, ptop, kids = chains[c]
            chain_top.append(top)
            chain_len.append(ln)
            chain_ptop.append(ptop)
            for k in kids:
                chain_child.append(chains[k][0])
            chain_cptr.append(len(chain_child))
        bi = len(blocks)
        blocks.append([n0, n1 - n0, int(soff[n0]), int(soff[n1] - soff[n0]), chain0, len(cids),
                       level0, nlev, pranges[bi][0], pranges[bi][1], 0, 0])

    # ---- stimulus CSR (internal node -> stimulus columns) ----
    stim_inds = np.asarray(p.stim_inds, dtype=np.int64)
    stim_lists: List[List[int]] = [[] for _ in range(n)]
    for q, r in enumerate(stim_inds):
        stim_lists[int(node2int[r])].append(q)
    stim_ptr = np.zeros(n + 1, dtype=np.int32)
    for i in range(n):
        stim_ptr[i + 1] = stim_ptr[i] + len(stim_lists[i])
    stim_idx = np.asarray([q for lst in stim_lists for q in lst], dtype=np.int32)
    stim = None
    if p.stim is not None and len(stim_inds):
        stim = np.ascontiguousarray(np.transpose(np.asarray(p.stim, dtype=np.float64), (2, 0, 1)))

    # ---- recordings CSR ----
    rec_lists: List[List[Tuple[int, int]]] = [[] for _ in range(n)]
    for col, (name, r) in enumerate(p.recordings):
        i = int(node2int[int(r)])
        if name in slot_names[i]:
            sl = slot_names[i].index(name)
        elif name in p.current_names or name in p.states:
            sl = -1
        else:
            raise NotImplementedError(f"recording of `{name}` is not covered")
        rec_lists[i].append((sl, col))
    rec_ptr = np.zeros(n + 1, dtype=np.int32)
    for i in range(n):
        rec_ptr[i + 1] = rec_ptr[i] + len(rec_lists[i])
    rec_slot = np.asarray([s for lst in rec_lists for s, _ in lst], dtype=np.int32)
    rec_col = np.asarray([c for lst in rec_lists for _, c in lst], dtype=np.int32)

    def i32(x):
        return np.ascontiguousarray(np.asarray(x, dtype=np.int32))

    # ---- gradient slots: every node owns one float32 accumulator per trainable
    # parameter (column != 0) for the adjoint kernel ----
    pcol_arr = np.asarray(pcol, dtype=np.int64)
    gk = np.full(len(pcol_arr), -1, dtype=np.int32)
    run_len = np.zeros(n, dtype=np.int64)
    for i in range(n):
        run_len[i] = len(node_pb[i])
    done_runs = set()
    for i in range(n):
        st0 = int(poff[i])
        key = (st0, int(run_len[i]))  # empty runs share their start with the next run
        if key in done_runs:
            continue
        done_runs.add(key)
        rk = 0
        for q in range(st0, st0 + int(run_len[i])):
            if pcol_arr[q] != 0:
                gk[q] = rk
                rk += 1
    gbase = np.zeros(n, dtype=np.int32)
    max_gslots = 0
    for (n0, n1) in blocks_nodes:
        acc = 0
        for i in range(n0, n1):
            gbase[i] = acc
            st0 = int(poff[i])
            acc += int(np.count_nonzero(pcol_arr[st0:st0 + int(run_len[i])]))
        max_gslots = max(max_gslots, acc)

    # ---- parent / children in internal order (for the delta form of the step) ----
    par_int = np.full(n, -1, dtype=np.int64)
    ps = np.asarray(parent_solve, dtype=np.int64)[order]
    has_par = ps >= 0
    par_int[has_par] = solve2int[ps[has_par]]
    kid_lists: List[List[int]] = [[] for _ in range(n)]
    for i in range(n):
        if par_int[i] >= 0:
            kid_lists[int(par_int[i])].append(i)
    kid_ptr = np.zeros(n + 1, dtype=np.int32)
    for i in range(n):
        kid_ptr[i + 1] = kid_ptr[i] + len(kid_lists[i])
    kid = np.asarray([c for lst in kid_lists for c in lst], dtype=np.int32)

    return Lowered(
        n_nodes=n,
        batch=B,
        int2node=int2node,
        node2int=node2int,
        a_low=a_low,
        a_up=a_up,
        gsum=gsum,
        cm=cm,
        area=area,
        node_class=i32(node_class),
        soff=i32(soff),
        poff=i32(poff),
        cls_ptr=i32(cls_ptr),
        cls_comp=i32(cls_comp),
        cls_prog=cls_prog,
        entries=np.ascontiguousarray(entries),
        pbase=np.asarray(pbase, dtype=np.float64),
        pcol=i32(pcol),
        pscale=np.ascontiguousarray(pscale),
        col_info=col_info,
        col_members=[sorted(m) for m in col_members],
        chain_top=i32(chain_top),
        chain_len=i32(chain_len),
        chain_ptop=i32(chain_ptop),
        chain_cptr=i32(chain_cptr),
        chain_child=i32(chain_child),
        level_ptr=i32(level_ptr),
        blocks=i32(blocks),
        stim_ptr=stim_ptr,
        stim_idx=stim_idx,
        stim=stim,
        gk=gk,
        gbase=gbase,
        max_gslots=int(max_gslots),
        parent=i32(par_int),
        kid_ptr=kid_ptr,
        kid=kid,
        rec_ptr=rec_ptr,
        rec_slot=rec_slot,
        rec_col=rec_col,
        n_rec=len(p.recordings),
        state0=state0,
        slot_names=slot_names,
        dt=float(p.dt),
        n_steps=int(p.n_steps),
        max_levels=max_levels,
        tree_ptr=tree_ptr,
    )


def emulate_block_solve(low: Lowered, D: np.ndarray, S: np.ndarray, al: np.ndarray,
                        au: np.ndarray) -> np.ndarray:
    """Host replay of the kernels' chain solve (same schedule, same operation order),
    used to check a schedule without a GPU. Arrays are `(B, n)` in internal order."""
    D = np.array(D, dtype=np.float64, copy=True)
    S = np.array(S, dtype=np.float64, copy=True)
    for blk in low.blocks:
        chain0, nch_tot, level0, nlev = blk[4], blk[5], blk[6], blk[7]
        lp = low.level_ptr[level0:level0 + nlev + 1]
        for h in range(nlev):
            for c in range(chain0 + lp[h], chain0 + lp[h + 1]):
                top = low.chain_top[c]
                bot = top + low.chain_len[c] - 1
                d, s = D[:, bot].copy(), S[:, bot].copy()
                for k in range(low.chain_cptr[c], low.chain_cptr[c + 1]):
                    ct = low.chain_child[k]
                    f = au[ct] / D[:, ct]
                    d -= al[ct] * f
                    s -= S[:, ct] * f
                D[:, bot], S[:, bot] = d, s
                for j in range(bot - 1, top - 1, -1):
                    f = au[j + 1] / d
                    d = D[:, j] - al[j + 1] * f
                    s = S[:, j] - s * f
                    D[:, j], S[:, j] = d, s
        for h in range(nlev - 1, -1, -1):
            for c in range(chain0 + lp[h], chain0 + lp[h + 1]):
                top = low.chain_top[c]
                bot = top + low.chain_len[c] - 1
                pt = low.chain_ptop[c]
                xp = S[:, pt] if pt >= 0 else 0.0
                for j in range(top, bot + 1):
                    x = (S[:, j] - al[j] * xp) / D[:, j]
                    S[:, j] = x
                    xp = x
    return S
