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
V_SOLVE = "__v_unclamped"  # last slot of a voltage-clamped node: the solve output before the clamp


class _SlotNames:
    """Slot names of every internal node (shared per node group)."""

    def __init__(self, grp_names, grp_int):
        self.grp_names = grp_names
        self.grp_int = grp_int

    def __getitem__(self, i):
        return self.grp_names[int(self.grp_int[i])]

    def __len__(self):
        return len(self.grp_int)


class _ColMembers:
    """`(param name, reference node, base value)` of every use of a column, built on
    access (a column of a trainable group can have millions of uses)."""

    def __init__(self, ncol, use_c, use_i, use_k, grp_pslots, grp_int, grp_base, row_in_grp,
                 int2node):
        self.ncol = ncol
        order = np.argsort(use_c, kind="stable")
        self.use_c = use_c[order]
        self.use_i = use_i[order]
        self.use_k = use_k[order]
        self.ptr = np.searchsorted(self.use_c, np.arange(ncol + 1))
        self.grp_pslots, self.grp_int, self.grp_base = grp_pslots, grp_int, grp_base
        self.row_in_grp, self.int2node = row_in_grp, int2node

    def __len__(self):
        return self.ncol

    def __getitem__(self, col):
        out = set()
        for q in range(self.ptr[col], self.ptr[col + 1]):
            i, k = int(self.use_i[q]), int(self.use_k[q])
            g = int(self.grp_int[i])
            out.add((self.grp_pslots[g][k][1], int(self.int2node[i]),
                     float(self.grp_base[g][self.row_in_grp[i], k])))
        return sorted(out)


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
    col_members: "_ColMembers"  # [col] -> (param name, node, base) of its uses
    train_cols: np.ndarray  # (n trainable groups,) column of every group (-1 none, -2 several)
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
    clamp_ptr: np.ndarray  # (n_nodes + 1,) clamp entries of every internal node
    clamp_slot: np.ndarray  # node-relative slot of an entry (0 = v)
    clamp_col: np.ndarray  # column of an entry in `clamp`
    clamp: Optional[np.ndarray]  # (steps, rows, n_clamp) time-major clamp values
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
    slot_names: "_SlotNames"  # [internal node] -> slot names
    dt: float
    n_steps: int
    max_levels: int = 0
    tree_ptr: np.ndarray = field(default_factory=lambda: np.zeros(1, np.int64))
    scheme: int = 0  # JxbSimArgs.scheme: 0 backward Euler, 1 Crank-Nicolson

    @property
    def n_slots(self) -> int:
        """Length of a row of the state vector: the nodes' slots, padded to a multiple
        of 4 (16 bytes of float32) so that rows start on the same 16-byte phase."""
        return int(self.state0.shape[1])

    @property
    def n_pslots(self) -> int:
        return int(len(self.pbase))

    @property
    def n_cols(self) -> int:
        return int(self.pscale.shape[1])

    def group_scale(self) -> Tuple[np.ndarray, np.ndarray]:
        """`(cols, base)` of every trainable group: its column and the base value its
        nodes share (parameter = base * scale), so that the gradient with respect to
        the group's value in row b is `pgrad[b, col] / base`. Groups without one
        column or without one base value get column -1 and base NaN."""
        cols = np.asarray(self.train_cols, dtype=np.int64)
        base = np.full(len(cols), np.nan)
        for g, c in enumerate(cols):
            if c < 0:
                continue
            vals = {round(b, 15) for _, _, b in self.col_members[int(c)]}
            if len(vals) == 1:
                base[g] = vals.pop()
            else:
                cols[g] = -1
        return cols, base


@dataclass
class ChainTable:
    """Chains of a forest in breadth-first chain order (arrays indexed by chain id)."""

    top: np.ndarray  # first node (chain order)
    length: np.ndarray
    ptop: np.ndarray  # chain-order index of the parent chain's last node, -1 at a root
    parent: np.ndarray  # parent chain id, -1 at a root
    kid_ptr: np.ndarray  # (n_chains + 1,) child chains CSR
    kid: np.ndarray
    depth: np.ndarray  # chain depth from the root chain

    def __len__(self):
        return len(self.top)

    def as_list(self):
        """`(top, length, parent_top_node, child_chain_ids)` per chain."""
        return [[int(self.top[c]), int(self.length[c]), int(self.ptop[c]),
                 self.kid[self.kid_ptr[c]:self.kid_ptr[c + 1]].tolist()] for c in range(len(self.top))]


def _unique_rows(a: np.ndarray):
    """`np.unique(a, axis=0, return_index=True, return_inverse=True)` for a 2-D array,
    with each distinct row's first index; sorts with `lexsort` over the columns."""
    m = a.shape[0]
    if m == 0:
        return a[:0], np.zeros(0, np.int64), np.zeros(0, np.int64)
    if a.shape[1] == 0:
        return a[:1], np.zeros(1, np.int64), np.zeros(m, np.int64)
    if a.shape[1] > 16:
        u, first, inv = np.unique(a, axis=0, return_index=True, return_inverse=True)
        return u, first, inv.reshape(-1)
    srt = np.lexsort(a.T[::-1])  # stable: equal rows keep their index order
    b = a[srt]
    new = np.ones(m, dtype=bool)
    new[1:] = np.any(b[1:] != b[:-1], axis=1)
    grp = np.cumsum(new) - 1
    inv = np.empty(m, dtype=np.int64)
    inv[srt] = grp
    return b[new], srt[new], inv


def presynaptic_lists(pre: np.ndarray) -> Tuple[np.ndarray, np.ndarray]:
    """Outgoing synapses of every presynaptic node, for the backward pass of the
    synapse step (the sum of the presynaptic voltage gradients without atomics).

    The synapses are sorted by presynaptic node (stably, so a node keeps its
    synapses in index order); a node's run in that order becomes one row, its rank
    inside the run the column. Returns `(nodes, lists)`: the distinct presynaptic
    nodes in increasing order (int32) and `lists (len(nodes), width)` int32, the
    synapse indices of every node followed by -1 up to `width`, the largest
    out-degree (at least 1)."""
    pre = np.asarray(pre, dtype=np.int64).reshape(-1)
    E = len(pre)
    if E == 0:
        return np.zeros(0, np.int32), np.full((0, 1), -1, np.int32)
    by_node = np.argsort(pre, kind="stable")
    sorted_pre = pre[by_node]
    run_start = np.empty(E, dtype=bool)
    run_start[0] = True
    run_start[1:] = sorted_pre[1:] != sorted_pre[:-1]
    row = np.cumsum(run_start) - 1
    # position of the first synapse of the run, carried forward over the run
    first = np.maximum.accumulate(np.where(run_start, np.arange(E), 0))
    col = np.arange(E) - first
    lists = np.full((int(row[-1]) + 1, int(col.max()) + 1), -1, dtype=np.int32)
    lists[row, col] = by_node
    return sorted_pre[run_start].astype(np.int32), lists


def _pointer_jump(ptr: np.ndarray, dist: np.ndarray):
    """List ranking: follow `ptr` to its fixed point, summing `dist` on the way."""
    while True:
        nxt = ptr[ptr]
        if np.array_equal(nxt, ptr):
            return ptr, dist
        dist = dist + dist[ptr]
        ptr = nxt


def chain_table(parent: np.ndarray):
    """Chain decomposition of a solve-order forest (vectorised).

    A node continues its parent's chain when it is the parent's only child. The
    chains of every tree are numbered breadth first (a chain's children in the order
    of their first nodes) and their nodes laid out consecutively. Returns
    `(order, trees, table)`: `order[i]` is the solve index of chain-order node `i`,
    `trees` the chain-order start of every tree (plus the end).
    """
    parent = np.asarray(parent, dtype=np.int64)
    n = len(parent)
    roots = np.nonzero(parent < 0)[0]
    if n == 0 or len(roots) == 0 or roots[0] != 0:
        raise ValueError("the forest must start with a root")
    ends = np.append(roots[1:], n)
    tree_of = np.repeat(np.arange(len(roots)), ends - roots)
    nonroot = parent >= 0
    idx = np.arange(n)
    if not (np.all(parent[nonroot] >= roots[tree_of[nonroot]]) and np.all(parent[nonroot] < idx[nonroot])):
        raise ValueError("every tree must be contiguous and parents must precede children")
    nkids = np.bincount(parent[nonroot], minlength=n)
    is_head = ~nonroot
    is_head[nonroot] = nkids[parent[nonroot]] != 1
    head_of, pos = _pointer_jump(np.where(is_head, idx, parent), (~is_head).astype(np.int64))
    heads = np.nonzero(is_head)[0]  # increasing node index
    H = len(heads)
    cid_of_head = np.full(n, -1, dtype=np.int64)
    cid_of_head[heads] = np.arange(H)
    ph = parent[heads]
    pc = np.where(ph >= 0, cid_of_head[head_of[np.maximum(ph, 0)]], -1)
    # breadth-first rank, one chain depth at a time
    depth = np.full(H, -1, dtype=np.int64)
    rank = np.zeros(H, dtype=np.int64)
    cur = np.nonzero(pc < 0)[0]  # root chains, in tree order
    depth[cur] = 0
    rank[cur] = np.arange(len(cur))
    d = 0
    while len(cur):
        at_d = np.zeros(H, dtype=bool)
        at_d[cur] = True
        nxt = np.nonzero((pc >= 0) & at_d[np.maximum(pc, 0)])[0]
        nxt = nxt[np.lexsort((heads[nxt], rank[pc[nxt]]))]
        d += 1
        depth[nxt] = d
        rank[nxt] = np.arange(len(nxt))
        cur = nxt
    bfs = np.lexsort((rank, depth, tree_of[heads]))  # chain ids in breadth-first order
    new_id = np.empty(H, dtype=np.int64)
    new_id[bfs] = np.arange(H)
    length = np.bincount(head_of, minlength=n)[heads][bfs]
    top = np.zeros(H, dtype=np.int64)
    top[1:] = np.cumsum(length)[:-1]
    order = np.empty(n, dtype=np.int64)
    order[top[new_id[cid_of_head[head_of]]] + pos] = idx
    cpar = np.where(pc[bfs] >= 0, new_id[np.maximum(pc[bfs], 0)], -1)
    ptop = np.where(cpar >= 0, top[np.maximum(cpar, 0)] + length[np.maximum(cpar, 0)] - 1, -1)
    child = np.nonzero(cpar >= 0)[0]
    child = child[np.argsort(cpar[child], kind="stable")]
    kid_ptr = np.zeros(H + 1, dtype=np.int64)
    kid_ptr[1:] = np.cumsum(np.bincount(cpar[child], minlength=H))
    trees = np.zeros(len(roots) + 1, dtype=np.int64)
    trees[1:] = np.cumsum(ends - roots)
    return order, trees, ChainTable(top, length, ptop, cpar, kid_ptr, child, depth[bfs])


def chain_order(parent: np.ndarray):
    """`chain_table` with the chains as a list of `(top, length, parent_top_node,
    child_chain_ids)`."""
    order, trees, table = chain_table(parent)
    return order, trees, table.as_list()


def chain_levels(chains) -> np.ndarray:
    """Height of every chain above its deepest descendant chain (0 for a leaf chain)."""
    if isinstance(chains, ChainTable):
        lev = np.zeros(len(chains), dtype=np.int64)
        for d in range(int(chains.depth.max(initial=0)), 0, -1):
            c = np.nonzero(chains.depth == d)[0]
            np.maximum.at(lev, chains.parent[c], lev[c] + 1)
        return lev
    lev = np.zeros(len(chains), dtype=np.int64)
    for cid in range(len(chains) - 1, -1, -1):  # children come after parents
        kids = chains[cid][3]
        if kids:
            lev[cid] = 1 + max(lev[k] for k in kids)
    return lev


def block_schedule(table: ChainTable, blocks_nodes, relative: bool = False):
    """Chains of every block sorted by level (height), children CSR by first node.

    Returns `(chain_top, chain_len, chain_ptop, chain_cptr, chain_child, level_ptr,
    per_block)` with `per_block[b] = (chain0, n_chains, level0, n_levels)`; with
    `relative` the node indices are relative to the block's first node.
    """
    lev = chain_levels(table)
    perm_parts, lp_parts, per_block = [], [], []
    n_ch = n_lp = 0
    for (n0, n1) in blocks_nodes:
        lo, hi = np.searchsorted(table.top, n0), np.searchsorted(table.top, n1)
        cids = np.arange(lo, hi)
        cids = cids[np.argsort(lev[cids], kind="stable")]
        nlev = int(lev[cids].max()) + 1 if len(cids) else 0
        counts = np.bincount(lev[cids], minlength=nlev)
        lp_parts.append(np.concatenate([[0], np.cumsum(counts)]))
        per_block.append((n_ch, len(cids), n_lp, nlev))
        perm_parts.append(cids)
        n_ch += len(cids)
        n_lp += nlev + 1
    perm = np.concatenate(perm_parts) if perm_parts else np.zeros(0, np.int64)
    shift = np.zeros(len(table), dtype=np.int64)
    if relative:
        for (n0, n1), part in zip(blocks_nodes, perm_parts):
            shift[part] = n0
    nk = table.kid_ptr[perm + 1] - table.kid_ptr[perm]
    cptr = np.zeros(len(perm) + 1, dtype=np.int64)
    cptr[1:] = np.cumsum(nk)
    kid_pos = np.repeat(table.kid_ptr[perm] - cptr[:-1], nk) + np.arange(int(cptr[-1]))
    kids = table.kid[kid_pos]
    child_top = table.top[kids] - np.repeat(shift[perm], nk)
    ptop = table.ptop[perm]
    ptop = np.where(ptop >= 0, ptop - shift[perm], -1)
    return (table.top[perm] - shift[perm], table.length[perm], ptop, cptr, child_top,
            np.concatenate(lp_parts) if lp_parts else np.zeros(0, np.int64), per_block)


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


# The somatic L5PC program (ProgL5pcSoma) shares calcium slots between channels; a
# class runs it only with exactly this layout: (channel, state slots, parameter
# count, first parameter, current slot) per entry, node-relative.
SOMA_LAYOUT = [
    ("NaTs2T", (1, 2), 2, 0, -1), ("SKv3_1", (3,), 2, 2, -1), ("SKE2", (4, 5), 2, 4, -1),
    ("CaNernstReversal", (6, 5, 7), 3, 6, 12), ("CaPump", (5,), 4, 9, 12),
    ("CaHVA", (8, 9, 6), 1, 13, 12), ("CaLVA", (10, 11, 6), 1, 14, 12), ("Leak", (), 2, 15, -1),
]
PROG_L5PC_SOMA = 3


def _is_soma_layout(ents: np.ndarray) -> bool:
    if len(ents) != len(SOMA_LAYOUT):
        return False
    for e, (name, slots, npar, p0, cur) in zip(ents, SOMA_LAYOUT):
        if int(e[0]) != SPECS[name].type_id or int(e[1]) != len(slots) or int(e[2]) != npar:
            return False
        if int(e[3]) != cur or int(e[10]) != p0:
            return False
        if any(int(e[4 + q]) != s for q, s in enumerate(slots)):
            return False
    return True


def program_of(ents: np.ndarray) -> int:
    if len(ents) == 0:
        return 0
    if _is_soma_layout(ents):
        return PROG_L5PC_SOMA
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
    the other currents are not kept in the resident state.

    The work is vectorised over groups of nodes with the same channels (and flags):
    a group shares its slot layout and node class, and its parameters are gathered
    as one `(nodes, slots)` matrix."""
    p = problem
    n = p.n_nodes
    B = p.batch
    parent_solve, g_low_s, g_up_s = p.solve_order_system()
    if np.asarray(g_low_s).ndim != 1:
        raise NotImplementedError("axial conductances with a batch dimension are not covered")
    order, tree_ptr, chains = chain_table(parent_solve)
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

    # ---- node groups: nodes with the same channels (and flags) share a layout ----
    C = len(p.channels)
    ch_member = np.zeros((n, max(C, 1)), dtype=bool)
    for ci, ch in enumerate(p.channels):
        ch_member[np.asarray(ch.inds, dtype=np.int64), ci] = True
    recorded = {(name, int(r)) for name, r in p.recordings}
    cur_names = sorted({ch.current for ch in p.channels})
    rec_cur = np.zeros((n, max(len(cur_names), 1)), dtype=bool)
    for name, r in p.recordings:
        if name in cur_names:
            rec_cur[int(r), cur_names.index(name)] = True
    # Nodes with a voltage clamp keep the unclamped solve output in one more slot,
    # their last (the adjoint needs it; the clamped value replaces v).
    vclamped = np.zeros(n, dtype=bool)
    for cname, cnodes, _ in getattr(p, "clamps", []) or []:
        if cname == "v":
            vclamped[np.asarray(cnodes, dtype=np.int64)] = True
    keymat = np.concatenate([is_comp[:, None], ch_member, rec_cur, vclamped[:, None]], axis=1)
    _, grp_rep, grp_of_node = _unique_rows(np.packbits(keymat, axis=1))
    readers = {"CaPump"}  # channels whose update reads their current state
    G = len(grp_rep)
    first_int = np.full(G, n, dtype=np.int64)
    np.minimum.at(first_int, grp_of_node[int2node], np.arange(n))
    classes: Dict[tuple, int] = {}
    cls_entries: List[np.ndarray] = []
    cls_comp: List[int] = []
    grp_class = np.zeros(G, dtype=np.int32)
    grp_names: List[List[str]] = [[] for _ in range(G)]
    grp_pslots: List[list] = [[] for _ in range(G)]
    for g in np.argsort(first_int, kind="stable"):  # class ids in order of first use
        r = int(grp_rep[g])
        chs = [int(ci) for ci in np.nonzero(ch_member[r, :C])[0]]
        names = ["v"]
        for ci in chs:
            for st_name in p.channels[ci].states:
                if st_name not in names:
                    names.append(st_name)
        for ci in chs:
            cn = p.channels[ci].current
            need = (keep_currents or p.channels[ci].type_name in readers
                    or (cn, r) in recorded
                    or any(p.channels[cj].type_name in readers and p.channels[cj].current == cn
                           for cj in chs))
            if need and cn not in names:
                names.append(cn)
        if vclamped[r]:
            names.append(V_SOLVE)
        ents, pslots, pk = [], [], 0
        for ci in chs:
            ch = p.channels[ci]
            spec = SPECS[ch.type_name]
            e = np.zeros(ENTRY_SHORTS, dtype=np.int16)
            e[0] = spec.type_id
            e[1] = len(ch.states)
            e[2] = len(ch.params) + len(ch.constants)
            e[3] = names.index(ch.current) if ch.current in names else -1
            for q, st_name in enumerate(ch.states):
                e[4 + q] = names.index(st_name)
            for q in range(int(e[2])):  # parameters are consecutive
                if 10 + q < ENTRY_SHORTS:
                    e[10 + q] = pk + q
            pslots += [("p", pn) for pn in ch.params] + [("c", float(cv)) for cv in ch.constants]
            pk += int(e[2])
            ents.append(e)
        key = (bool(is_comp[r]), tuple(names), tuple(tuple(e.tolist()) for e in ents))
        if key not in classes:
            classes[key] = len(cls_entries)
            cls_entries.append(np.stack(ents) if ents else np.zeros((0, ENTRY_SHORTS), np.int16))
            cls_comp.append(int(is_comp[r]))
        grp_class[g] = classes[key]
        grp_names[g] = names
        grp_pslots[g] = pslots
    grp_int = grp_of_node[int2node]  # group of every internal node
    node_class = grp_class[grp_int]
    nslots_g = np.asarray([len(nm) for nm in grp_names], dtype=np.int64)
    soff = np.zeros(n + 1, dtype=np.int64)
    soff[1:] = np.cumsum(nslots_g[grp_int])
    cls_prog = np.asarray([program_of(e) for e in cls_entries], dtype=np.int32)
    cls_ptr = np.zeros(len(cls_entries) + 1, dtype=np.int32)
    for c, e in enumerate(cls_entries):
        cls_ptr[c + 1] = cls_ptr[c] + len(e)
    entries = (np.concatenate(cls_entries) if len(cls_entries) else np.zeros((0, ENTRY_SHORTS))).astype(np.int16)
    grp_nodes = [np.nonzero(grp_int == g)[0] for g in range(G)]  # internal nodes, increasing
    row_in_grp = np.zeros(n, dtype=np.int64)
    for g in range(G):
        row_in_grp[grp_nodes[g]] = np.arange(len(grp_nodes[g]))

    # ---- parameter values and columns, per group (vectorised over its nodes) ----
    # A parameter that varies over the batch gets one column per distinct batch
    # profile (value / row-0 value); a node of a trainable group gets its group's
    # column (one per distinct profile of the group). Columns are numbered at the
    # end in order of first use (internal node, then parameter slot).
    col_vecs: List[np.ndarray] = [np.ones(B)]
    col_keys: Dict[bytes, int] = {}
    tgroup_of: Dict[str, np.ndarray] = {}
    for gi, (gname, gnodes) in enumerate(getattr(p, "trainable", []) or []):
        if gname not in tgroup_of:
            tgroup_of[gname] = np.full(n, -1, dtype=np.int64)
        tgroup_of[gname][np.asarray(gnodes, dtype=np.int64)] = gi

    def col_ids(prefix: bytes, rows: np.ndarray, tag: Optional[np.ndarray] = None) -> np.ndarray:
        """Column of every row of `rows` (m, B): one column per distinct (tag, row)."""
        keyed = rows if tag is None else np.concatenate([tag[:, None].astype(np.float64), rows], axis=1)
        urows, _, inv = _unique_rows(keyed)
        ids = np.empty(len(urows), dtype=np.int64)
        for u, row in enumerate(urows):
            pre = prefix if tag is None else prefix + str(int(row[0])).encode() + b"|"
            vec = row if tag is None else row[1:]
            kb = pre + np.ascontiguousarray(vec).tobytes()
            if kb not in col_keys:
                col_keys[kb] = len(col_vecs)
                col_vecs.append(np.asarray(vec, dtype=np.float64))
            ids[u] = col_keys[kb]
        return ids[inv]

    grp_base: List[np.ndarray] = []
    grp_col: List[np.ndarray] = []
    group_uses: List[Tuple[np.ndarray, np.ndarray]] = []  # (trainable group, column) per use
    for g in range(G):
        R = int2node[grp_nodes[g]]
        m = len(R)
        P = len(grp_pslots[g])
        base = np.zeros((m, P))
        colm = np.zeros((m, P), dtype=np.int64)
        for k, (kind, val) in enumerate(grp_pslots[g]):
            if kind == "c":
                base[:, k] = val
                continue
            a = np.asarray(p.params[val], dtype=np.float64)
            b0 = a[R] if a.ndim == 1 else a[0, R]
            safe = np.where(b0 != 0, b0, 1.0)
            tg = tgroup_of[val][R] if val in tgroup_of else np.full(m, -1, dtype=np.int64)
            trained = tg >= 0
            base[:, k] = b0
            if a.ndim == 2:
                vals = np.broadcast_to(a[:, R], (B, m))
                vary = np.nonzero(~np.all(vals == vals[:1], axis=0) & ~trained)[0]
                if len(vary):
                    base[vary, k] = safe[vary]
                    colm[vary, k] = col_ids(val.encode() + b"|", (vals[:, vary] / safe[vary]).T)
            idx = np.nonzero(trained)[0]
            if len(idx):
                base[idx, k] = safe[idx]
                prof = (np.ones((len(idx), B)) if a.ndim == 1
                        else (np.broadcast_to(a[:, R[idx]], (B, len(idx))) / safe[idx]).T)
                colm[idx, k] = col_ids(b"group|", prof, tag=tg[idx])
                group_uses.append((tg[idx], colm[idx, k].copy()))
        grp_base.append(base)
        grp_col.append(colm)

    # renumber the columns in order of first use
    ncol = len(col_vecs)
    Pmax = max([len(ps) for ps in grp_pslots] + [1])
    first_use = np.full(ncol, np.iinfo(np.int64).max, dtype=np.int64)
    first_use[0] = -1
    use_i, use_k, use_c = [], [], []
    for g in range(G):
        ii, kk = np.nonzero(grp_col[g])
        use_i.append(grp_nodes[g][ii])
        use_k.append(kk)
        use_c.append(grp_col[g][ii, kk])
    use_i = np.concatenate(use_i) if use_i else np.zeros(0, np.int64)
    use_k = np.concatenate(use_k) if use_k else np.zeros(0, np.int64)
    use_c = np.concatenate(use_c) if use_c else np.zeros(0, np.int64)
    np.minimum.at(first_use, use_c, use_i * Pmax + use_k)
    new_of = np.empty(ncol, dtype=np.int64)
    new_of[np.argsort(first_use, kind="stable")] = np.arange(ncol)
    grp_col = [new_of[c] for c in grp_col]
    old_of = np.argsort(new_of)
    col_vecs = [col_vecs[c] for c in old_of]
    pscale = np.stack(col_vecs, axis=1) if B > 0 else np.ones((1, 1))
    fu = first_use[old_of]
    col_info: List[Tuple[str, int]] = [("", -1)]
    for c in range(1, ncol):
        i_f, k_f = int(fu[c] // Pmax), int(fu[c] % Pmax)
        col_info.append((grp_pslots[grp_int[i_f]][k_f][1], int(int2node[i_f])))
    col_members = _ColMembers(ncol, new_of[use_c], use_i, use_k, grp_pslots, grp_int,
                              grp_base, row_in_grp, int2node)
    # The column of every trainable group: -1 if no node of the group has the
    # parameter, -2 if its nodes span several columns (different batch profiles).
    n_groups = len(getattr(p, "trainable", []) or [])
    train_cols = np.full(n_groups, -1, dtype=np.int64)
    if group_uses:
        tgs = np.concatenate([t for t, _ in group_uses])
        cls_ = new_of[np.concatenate([c for _, c in group_uses])]
        pairs = np.unique(np.stack([tgs, cls_], 1), axis=0)  # sorted by group, then column
        gids, first, counts = np.unique(pairs[:, 0], return_index=True, return_counts=True)
        train_cols[gids] = np.where(counts == 1, pairs[first, 1], -2)

    # ---- initial state ----
    L = int(soff[-1])
    state0 = np.zeros((B, (L + 3) // 4 * 4), dtype=np.float64)  # padded row (unused tail)
    for g in range(G):
        I = grp_nodes[g]
        R = int2node[I]
        for k, nm in enumerate(grp_names[g]):
            if nm not in p.states:
                continue
            a = np.asarray(p.states[nm], dtype=np.float64)
            state0[:, soff[I] + k] = a[R][None, :] if a.ndim == 1 else np.broadcast_to(a[:, R], (B, len(R)))

    # ---- blocks: parameter runs, chains ordered by level inside each block ----
    blocks_nodes = pack_blocks(tree_ptr, max_block_nodes)
    # Nodes of a block with identical parameters (values and columns) share one run
    # of parameter slots; runs are laid out in order of first use inside the block.
    pbase_parts: List[np.ndarray] = []
    pcol_parts: List[np.ndarray] = []
    gk_parts: List[np.ndarray] = []
    poff = np.zeros(n, dtype=np.int64)
    pranges = []
    total = 0
    for (n0, n1) in blocks_nodes:
        start = total
        runs: Dict[bytes, list] = {}  # content -> [first node, base, col, node lists]
        for g in np.unique(grp_int[n0:n1]):
            gn = grp_nodes[g]
            I = gn[np.searchsorted(gn, n0):np.searchsorted(gn, n1)]
            P = len(grp_pslots[g])
            rb = grp_base[g][row_in_grp[I]]
            rc = grp_col[g][row_in_grp[I]]
            rows = np.concatenate([rb, rc.astype(np.float64)], axis=1) if P else np.zeros((len(I), 1))
            urows, ufirst, inv_r = _unique_rows(rows)
            if len(urows) > 1:
                srt = np.argsort(inv_r, kind="stable")
                splits = np.split(I[srt], np.cumsum(np.bincount(inv_r, minlength=len(urows)))[:-1])
            else:
                splits = [I]
            for u in range(len(urows)):
                kb = (np.ascontiguousarray(rb[ufirst[u]]).tobytes() + b"|"
                      + np.ascontiguousarray(rc[ufirst[u]]).tobytes())
                if kb in runs:
                    ent = runs[kb]
                    ent[0] = min(ent[0], int(I[ufirst[u]]))
                    ent[3].append(splits[u])
                else:
                    runs[kb] = [int(I[ufirst[u]]), rb[ufirst[u]], rc[ufirst[u]], [splits[u]]]
        for first, rbase, rcol, node_lists in sorted(runs.values(), key=lambda e: e[0]):
            for nl in node_lists:
                poff[nl] = total
            pbase_parts.append(rbase)
            pcol_parts.append(rcol)
            nzr = rcol != 0
            gk_parts.append(np.where(nzr, np.cumsum(nzr) - 1, -1))
            total += len(rbase)
        pranges.append((start, total - start))
    pbase = np.concatenate(pbase_parts) if pbase_parts else np.zeros(0)
    pcol = np.concatenate(pcol_parts).astype(np.int64) if pcol_parts else np.zeros(0, dtype=np.int64)
    gk = (np.concatenate(gk_parts) if gk_parts else np.zeros(0)).astype(np.int32)
    (chain_top, chain_len, chain_ptop, chain_cptr, chain_child, level_ptr,
     per_block) = block_schedule(chains, blocks_nodes)
    max_levels = max([pb[3] for pb in per_block] + [0])
    blocks = [[n0, n1 - n0, int(soff[n0]), int(soff[n1] - soff[n0]), pb[0], pb[1], pb[2], pb[3],
               pr[0], pr[1], 0, 0] for (n0, n1), pb, pr in zip(blocks_nodes, per_block, pranges)]

    # ---- clamps: CSR over internal nodes of (node-relative slot, clamp column) ----
    cl_int, cl_slot, cl_col, cl_vals = [], [], [], []
    ncl = 0
    for cname, cnodes, cvals in getattr(p, "clamps", []) or []:
        cnodes = np.asarray(cnodes, dtype=np.int64).reshape(-1)
        cvals = np.asarray(cvals, dtype=np.float64)
        cvals = cvals.reshape(-1, len(cnodes), cvals.shape[-1])
        for q, node in enumerate(cnodes):
            i = int(node2int[node])
            names = grp_names[grp_int[i]]
            if cname not in names:
                continue  # the node has no such state: nothing to clamp
            cl_int.append(i)
            cl_slot.append(names.index(cname))
            cl_col.append(ncl + q)
        cl_vals.append(cvals)
        ncl += len(cnodes)
    clamp = None
    clamp_ptr = np.zeros(n + 1, dtype=np.int32)
    clamp_slot = np.zeros(0, dtype=np.int32)
    clamp_col = np.zeros(0, dtype=np.int32)
    if cl_int:
        rows = max(v.shape[0] for v in cl_vals)
        steps = min(v.shape[-1] for v in cl_vals)
        full = np.concatenate([np.broadcast_to(v[..., :steps], (rows,) + v.shape[1:2] + (steps,))
                               for v in cl_vals], axis=1)
        clamp = np.ascontiguousarray(np.transpose(full, (2, 0, 1)))  # (steps, rows, ncl)
        cl_int = np.asarray(cl_int, dtype=np.int64)
        by_node = np.argsort(cl_int, kind="stable")  # keeps the given order per node: last wins
        clamp_slot = np.asarray(cl_slot, dtype=np.int32)[by_node]
        clamp_col = np.asarray(cl_col, dtype=np.int32)[by_node]
        clamp_ptr[1:] = np.cumsum(np.bincount(cl_int, minlength=n))

    # ---- stimulus CSR (internal node -> stimulus columns) ----
    stim_inds = np.asarray(p.stim_inds, dtype=np.int64)
    s_int = node2int[stim_inds] if len(stim_inds) else np.zeros(0, np.int64)
    stim_idx = np.argsort(s_int, kind="stable").astype(np.int32)
    stim_ptr = np.zeros(n + 1, dtype=np.int32)
    stim_ptr[1:] = np.cumsum(np.bincount(s_int, minlength=n))
    stim = None
    if p.stim is not None and len(stim_inds):
        stim = np.ascontiguousarray(np.transpose(np.asarray(p.stim, dtype=np.float64), (2, 0, 1)))

    # ---- recordings CSR ----
    rec_int, rec_sl = [], []
    for name, r in p.recordings:
        i = int(node2int[int(r)])
        names = grp_names[grp_int[i]]
        if name in names:
            sl = names.index(name)
        elif name in p.current_names or name in p.states:
            sl = -1
        else:
            raise NotImplementedError(f"recording of `{name}` is not covered")
        rec_int.append(i)
        rec_sl.append(sl)
    rec_int = np.asarray(rec_int, dtype=np.int64)
    r_order = np.argsort(rec_int, kind="stable")
    rec_slot = np.asarray(rec_sl, dtype=np.int32)[r_order] if len(rec_sl) else np.zeros(0, np.int32)
    rec_col = r_order.astype(np.int32)
    rec_ptr = np.zeros(n + 1, dtype=np.int32)
    if len(rec_int):
        rec_ptr[1:] = np.cumsum(np.bincount(rec_int, minlength=n))

    def i32(x):
        return np.ascontiguousarray(np.asarray(x, dtype=np.int32))

    # ---- gradient slots: every node owns one accumulator per trainable parameter
    # (column != 0) of its run for the adjoint kernel (ranks in `gk`) ----
    n_train = np.zeros(n, dtype=np.int64)
    for g in range(G):
        if len(grp_pslots[g]) and len(grp_nodes[g]):
            n_train[grp_nodes[g]] = np.count_nonzero(grp_col[g], axis=1)
    gbase = np.zeros(n, dtype=np.int32)
    max_gslots = 0
    for bi, (n0, n1) in enumerate(blocks_nodes):
        c = np.cumsum(n_train[n0:n1])
        gbase[n0:n1] = np.concatenate([[0], c[:-1]])
        blocks[bi][10] = int(c[-1]) if len(c) else 0  # gradient slots of the block
        max_gslots = max(max_gslots, blocks[bi][10])

    # ---- parent / children in internal order (for the delta form of the step) ----
    par_int = np.full(n, -1, dtype=np.int64)
    ps = np.asarray(parent_solve, dtype=np.int64)[order]
    has_par = ps >= 0
    par_int[has_par] = solve2int[ps[has_par]]
    child = np.nonzero(has_par)[0]
    kid = child[np.argsort(par_int[child], kind="stable")].astype(np.int32)
    kid_ptr = np.zeros(n + 1, dtype=np.int32)
    kid_ptr[1:] = np.cumsum(np.bincount(par_int[child], minlength=n))

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
        col_members=col_members,
        train_cols=train_cols,
        chain_top=i32(chain_top),
        chain_len=i32(chain_len),
        chain_ptop=i32(chain_ptop),
        chain_cptr=i32(chain_cptr),
        chain_child=i32(chain_child),
        level_ptr=i32(level_ptr),
        blocks=i32(blocks),
        stim_ptr=stim_ptr,
        clamp_ptr=clamp_ptr,
        clamp_slot=clamp_slot,
        clamp_col=clamp_col,
        clamp=clamp,
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
        slot_names=_SlotNames(grp_names, grp_int),
        dt=float(p.dt),
        scheme=1 if getattr(p, "solver", "bwd_euler") == "crank_nicolson" else 0,
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
