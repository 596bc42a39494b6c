"""Tree solve of the DHS voltage step on sm_100a: the drop-in for jaxley-pytorch's
`kernels/tree_solve.py`.

Same public surface as the reference module: `build_forest_schedule`,
`build_level_schedule`, `TreeSolveKernel` / `LevelTreeSolveKernel` with `.solve()` and
`.fused()`, `make_tree_solve_kernel(parent, device, mode)` honouring
`JAXLEY_PYTORCH_TREE_KERNEL=auto|registers|levels` (`tree_solve.py:485-513`), the custom
ops `tree_solve` / `tree_solve_levels` with the reference's argument lists and a
backward that is the transposed solve (`tree_solve.py:516-630`), and
`fused_tree_solve`. The schedule tensors are this implementation's own (chain
schedule, warp-register blocks); the kernels are `jxb_tree_solve_levels` and
`jxb_tree_solve_registers` of libjxb. There is no torch fallback: the reference
returns `None` for orders it cannot handle, this module raises.

The custom ops are registered as `jaxley_pytorch_b200::tree_solve[_levels]`: the
reference's names and schemas under a namespace of their own, so that this module
and the reference's Triton module can be loaded in one process.
"""
from __future__ import annotations

import ctypes as C
import os
import weakref
from collections import OrderedDict
from typing import Dict, Optional

import numpy as np
import torch

from .. import _lib
from ..lower import block_schedule, chain_table
from . import OP_NAMESPACE

MAX_BLOCK = 8192  # registers variant: up to 256 nodes in one warp, larger blocks in a CTA
# Registers variant: trees are packed into blocks of at least this many nodes by
# default. Measured on B200 on 512 trees of 40 nodes x 32 rows: blocks of 64 / 128 /
# 256 nodes (one warp each) took 81 / 116 / 257 us per solve, blocks of 512 nodes (a
# CTA each) 71 us, of 8192 nodes 166 us.
REG_MIN_BLOCK = 512
LEVEL_BLOCK = 4096  # levels variant: largest block of trees (shared memory bound)
# Levels variant: a forest of many small trees is cut into at least this many blocks
# (one CTA per block and batch row), so that even a small batch fills the SMs; blocks
# keep at least LEVEL_MIN_BLOCK nodes. Measured on 512 trees of 40 nodes x 32 rows:
# blocks of 4096 / 1280 / 640 / 320 / 160 nodes took 36.3 / 27.7 / 22.0 / 19.9 /
# 27.5 us per solve.
LEVEL_MIN_BLOCKS = 64
LEVEL_MIN_BLOCK = 256


def _forest(parent: np.ndarray):
    parent = np.asarray(parent, dtype=np.int64)
    n = len(parent)
    roots = np.nonzero(parent < 0)[0]
    if n == 0 or len(roots) == 0 or roots[0] != 0:
        raise ValueError("the node order must start with a root")
    ends = np.append(roots[1:], n)
    tree_of = np.repeat(np.arange(len(roots)), ends - roots)
    nonroot = parent >= 0
    idx = np.arange(n)
    if not (np.all(parent[nonroot] >= roots[tree_of[nonroot]]) and np.all(parent[nonroot] < idx[nonroot])):
        raise ValueError("trees must be contiguous with parents before children")
    return parent, roots, ends


def _depth_height(parent: np.ndarray):
    n = len(parent)
    depth = np.zeros(n, dtype=np.int64)
    for j in range(n):
        if parent[j] >= 0:
            depth[j] = depth[parent[j]] + 1
    height = np.zeros(n, dtype=np.int64)
    for j in range(n - 1, -1, -1):
        p = parent[j]
        if p >= 0:
            height[p] = max(height[p], height[j] + 1)
    return depth, height


def _pack(roots, ends, max_nodes):
    blocks, s = [], 0
    for a, b in zip(roots, ends):
        if b - s > max_nodes and a > s:
            blocks.append((s, int(a)))
            s = int(a)
    blocks.append((s, int(ends[-1])))
    return blocks


def build_forest_schedule(parent: np.ndarray, max_block: Optional[int] = None) -> Dict[str, np.ndarray]:
    """Schedule of the registers variant: whole trees packed into blocks of at most
    `max_block` (<= 8192) nodes; per block the parent, height, depth and child slots
    of every node (block-relative), cf. reference `tree_solve.py:45-138`. The block
    width is a power of two: up to 256 one warp holds a block, above it a CTA. By
    default a block holds up to the largest tree or REG_MIN_BLOCK nodes, whichever is
    more."""
    parent, roots, ends = _forest(parent)
    if max_block is None:
        max_block = min(MAX_BLOCK, max(REG_MIN_BLOCK, int((ends - roots).max())))
    if int((ends - roots).max()) > max_block:
        raise ValueError(f"a tree has more than {max_block} nodes: use the levels variant")
    depth, height = _depth_height(parent)
    n = len(parent)
    blocks = _pack(roots, ends, max_block)
    size = max(b - a for a, b in blocks)
    regs = 1
    while 32 * regs < size:
        regs *= 2
    W = 32 * regs
    kids = [[] for _ in range(n)]
    for j in range(n):
        if parent[j] >= 0:
            kids[parent[j]].append(j)
    num_slots = max(1, max(len(k) for k in kids))
    nb = len(blocks)
    rel_parent = np.tile(np.arange(W, dtype=np.int32), (nb, 1))
    rel_height = -np.ones((nb, W), dtype=np.int32)
    rel_depth = -np.ones((nb, W), dtype=np.int32)
    rel_children = -np.ones((nb, num_slots, W), dtype=np.int32)
    block_info = np.zeros((nb, 4), dtype=np.int32)
    for b, (s, e) in enumerate(blocks):
        ln = e - s
        p = parent[s:e]
        rel_parent[b, :ln] = np.where(p >= 0, p - s, np.arange(ln))
        rel_height[b, :ln] = height[s:e]
        rel_depth[b, :ln] = depth[s:e]
        for j in range(s, e):
            for k, c in enumerate(kids[j]):
                rel_children[b, k, j - s] = c - s
        block_info[b] = [s, ln, int(height[s:e].max()), int(depth[s:e].max())]
    return {"parent": parent, "block_info": block_info, "rel_parent": rel_parent,
            "rel_height": rel_height, "rel_depth": rel_depth, "rel_children": rel_children,
            "block_size": W, "regs_per_lane": regs, "num_slots": num_slots, "num_nodes": n}


def build_level_schedule(parent: np.ndarray, block_nodes: Optional[int] = None) -> Dict[str, np.ndarray]:
    """Schedule of the levels variant: trees packed into blocks of about
    `block_nodes` nodes (a larger tree gets its own block), each block's nodes in
    chain order with its chains sorted by level (cf. reference `tree_solve.py:142-224`).
    By default a block holds up to LEVEL_BLOCK nodes, fewer (down to LEVEL_MIN_BLOCK)
    when that leaves a forest in fewer than LEVEL_MIN_BLOCKS blocks."""
    parent, roots, ends = _forest(parent)
    n = len(parent)
    if int((ends - roots).max()) > 32767:
        raise ValueError("trees of more than 32767 nodes are not supported")
    if block_nodes is None:
        block_nodes = min(LEVEL_BLOCK, max(LEVEL_MIN_BLOCK, -(-n // LEVEL_MIN_BLOCKS)))
    order, tree_ptr, chains = chain_table(parent)
    blocks = _pack(roots, ends, block_nodes)
    # chain_table keeps the trees in order, so a block is the same range in both orders.
    (chain_top, chain_len, chain_ptop, chain_cptr, chain_child, level_ptr,
     per_block) = block_schedule(chains, blocks, relative=True)
    block_info = [[n0, n1 - n0, pb[0], pb[2]] for (n0, n1), pb in zip(blocks, per_block)]
    block_levels = [pb[3] for pb in per_block]
    i32 = lambda x: np.ascontiguousarray(np.asarray(x, dtype=np.int32))  # noqa: E731
    return {"parent": parent, "block_info": i32(block_info), "block_levels": i32(block_levels),
            "perm": i32(order), "chain_top": i32(chain_top), "chain_len": i32(chain_len),
            "chain_ptop": i32(chain_ptop), "chain_cptr": i32(chain_cptr),
            "chain_child": i32(chain_child if len(chain_child) else [0]), "level_ptr": i32(level_ptr),
            "max_block_nodes": int(max(b - a for a, b in blocks)),
            "max_levels": int(max(block_levels)), "num_nodes": n,
            "num_slots": int(max(1, np.diff(chains.kid_ptr).max(initial=0)))}


def _code(t: torch.Tensor) -> int:
    if t.dtype == torch.float32:
        return _lib.F32
    if t.dtype == torch.float64:
        return _lib.F64
    raise TypeError(f"unsupported dtype {t.dtype}")


def _prep(diags, lowers, uppers, solves, n):
    assert diags.shape[-1] == n, (diags.shape, n)
    batch = torch.broadcast_shapes(diags.shape, lowers.shape, uppers.shape, solves.shape)[:-1]
    ts = [torch.broadcast_to(t, (*batch, n)).reshape(-1, n).contiguous()
          for t in (diags, lowers, uppers, solves)]
    dt = ts[0].dtype
    ts = [t.to(dt) for t in ts]
    return batch, ts


class TreeSolveKernel:
    """Registers variant (blocks of small trees); schedule on the GPU."""

    def __init__(self, schedule: Dict[str, np.ndarray], device):
        self.device = torch.device(device)
        dev = self.device
        self.num_nodes = schedule["num_nodes"]
        self.block_size = schedule["block_size"]
        self.num_slots = schedule["num_slots"]
        self.num_warps = schedule["regs_per_lane"]  # the op's third int: registers per lane
        self.t = {k: torch.as_tensor(schedule[k], device=dev).contiguous()
                  for k in ["block_info", "rel_parent", "rel_height", "rel_depth", "rel_children"]}
        parents = np.asarray(schedule["parent"], dtype=np.int64)
        self.has_parent = torch.as_tensor(parents >= 0, device=dev)
        self.parent_safe = torch.as_tensor(np.where(parents >= 0, parents, 0), device=dev)
        s = _lib.JxbRegSchedule()
        s.n_nodes = self.num_nodes
        s.n_blocks = int(schedule["block_info"].shape[0])
        s.regs_per_lane = schedule["regs_per_lane"]
        s.num_slots = self.num_slots
        for k in ["block_info", "rel_parent", "rel_height", "rel_depth", "rel_children"]:
            setattr(s, k, self.t[k].data_ptr())
        self.sched = s

    def raw(self, d, l, u, s):
        x = torch.empty_like(s)
        st = torch.cuda.current_stream(d.device).cuda_stream
        rc = _lib.load().jxb_tree_solve_registers(_code(d), d.data_ptr(), l.data_ptr(), u.data_ptr(),
                                                  s.data_ptr(), x.data_ptr(), d.shape[0],
                                                  C.byref(self.sched), C.c_void_p(st))
        _lib.check(rc, "jxb_tree_solve_registers")
        return x

    def solve(self, diags, lowers, uppers, solves):
        """Solve; all inputs have shape `(..., num_nodes)` (broadcast)."""
        batch, (d, l, u, s) = _prep(diags, lowers, uppers, solves, self.num_nodes)
        return self.raw(d, l, u, s).reshape(*batch, self.num_nodes)

    def fused(self, diags, lowers, uppers, solves):
        """Differentiable solve (custom op)."""
        _register(self)
        return tree_solve_op(diags, lowers, uppers, solves, self.t["block_info"],
                             self.t["rel_parent"], self.t["rel_height"], self.t["rel_children"],
                             self.parent_safe, self.has_parent, self.block_size, self.num_slots,
                             self.num_warps)


class LevelTreeSolveKernel:
    """Levels variant (chain schedule in shared memory); schedule on the GPU."""

    W = 0  # kept for interface parity (the reference's chunk width); unused here

    def __init__(self, schedule: Dict[str, np.ndarray], device):
        self.device = torch.device(device)
        dev = self.device
        self.num_nodes = schedule["num_nodes"]
        self.num_slots = schedule["num_slots"]
        keys = ["block_info", "block_levels", "perm", "chain_top", "chain_len", "chain_ptop",
                "chain_cptr", "chain_child", "level_ptr"]
        self.t = {k: torch.as_tensor(schedule[k], device=dev).contiguous() for k in keys}
        parents = np.asarray(schedule["parent"], dtype=np.int64)
        self.has_parent = torch.as_tensor(parents >= 0, device=dev)
        self.parent_safe = torch.as_tensor(np.where(parents >= 0, parents, 0), device=dev)
        s = _lib.JxbTreeSchedule()
        s.n_nodes = self.num_nodes
        s.n_blocks = int(schedule["block_info"].shape[0])
        s.max_block_nodes = schedule["max_block_nodes"]
        s.max_levels = schedule["max_levels"]
        for k in keys:
            setattr(s, k, self.t[k].data_ptr())
        self.sched = s
        self.block_info = self.t["block_info"]

    def raw(self, d, l, u, s):
        x = torch.empty_like(s)
        st = torch.cuda.current_stream(d.device).cuda_stream
        rc = _lib.load().jxb_tree_solve_levels(_code(d), d.data_ptr(), l.data_ptr(), u.data_ptr(),
                                               s.data_ptr(), x.data_ptr(), d.shape[0],
                                               C.byref(self.sched), C.c_void_p(st))
        _lib.check(rc, "jxb_tree_solve_levels")
        return x

    def solve(self, diags, lowers, uppers, solves):
        batch, (d, l, u, s) = _prep(diags, lowers, uppers, solves, self.num_nodes)
        return self.raw(d, l, u, s).reshape(*batch, self.num_nodes)

    def fused(self, diags, lowers, uppers, solves):
        _register(self)
        t = self.t
        return tree_solve_levels_op(diags, lowers, uppers, solves, t["block_info"], t["level_ptr"],
                                    t["perm"], t["chain_ptop"], t["chain_child"], self.parent_safe,
                                    self.has_parent, self.num_slots, 0)


def make_tree_solve_kernel(parent: np.ndarray, device, mode: Optional[str] = None):
    """The solver for the forest given by `parent` (solve order, -1 for roots).

    `mode` (default: `JAXLEY_PYTORCH_TREE_KERNEL`, else `auto`): `registers` for
    blocks of trees held in registers, `levels` for any tree (chain schedule); `auto`
    picks `levels`, the faster of the two on every shape measured on B200 (a 1364-node
    tree x 256 rows: 20 against 51 us; 512 trees of 40 nodes x 32 rows: 20 against
    71 us)."""
    mode = mode or os.environ.get("JAXLEY_PYTORCH_TREE_KERNEL", "auto")
    if mode not in ("auto", "registers", "levels"):
        raise ValueError(f"JAXLEY_PYTORCH_TREE_KERNEL={mode}: expected auto, registers or levels")
    parent, roots, ends = _forest(parent)
    if mode == "auto":
        mode = "levels"
    if mode == "registers":
        return TreeSolveKernel(build_forest_schedule(parent), device)
    return LevelTreeSolveKernel(build_level_schedule(parent), device)


# ----------------------------------------------------------------------------------
# Custom ops (registered on first use; the registry maps schedule tensors to kernels)
# ----------------------------------------------------------------------------------
# Kernels whose `fused` was called, by the address of their block_info tensor; held
# weakly, so that an entry goes with its kernel (the solver that built it).
_KERNELS: "weakref.WeakValueDictionary[int, object]" = weakref.WeakValueDictionary()
# Kernels built for schedule tensors that reached an op without their kernel object
# (a caller that calls the op with tensors of its own): the last few, by the addresses
# of block_info and parent_safe and the node count.
_ADOPTED: "OrderedDict[tuple, object]" = OrderedDict()
_ADOPTED_MAX = 8
_NS = None
tree_solve_op = None
tree_solve_levels_op = None


def _register(kernel) -> None:
    _KERNELS[kernel.t["block_info"].data_ptr()] = kernel
    if _NS is None:
        _define_ops()


def _kernel_for(block_info: torch.Tensor, parent_safe: torch.Tensor, has_parent: torch.Tensor,
                mode: str):
    """The kernel of an op call: the one whose schedule tensors these are, else one
    built from the tree the op's `parent_safe` / `has_parent` describe."""
    k = _KERNELS.get(block_info.data_ptr())
    if k is not None and k.parent_safe.data_ptr() == parent_safe.data_ptr():
        return k
    key = (block_info.data_ptr(), parent_safe.data_ptr(), int(parent_safe.shape[-1]), mode)
    k = _ADOPTED.get(key)
    if k is None:
        parent = np.where(has_parent.cpu().numpy(), parent_safe.cpu().numpy(), -1)
        k = make_tree_solve_kernel(parent, parent_safe.device, mode=mode)
        _ADOPTED[key] = k
        while len(_ADOPTED) > _ADOPTED_MAX:
            _ADOPTED.popitem(last=False)
    else:
        _ADOPTED.move_to_end(key)
    return k


def _transposed_backward(kernel_op, ctx, grad_x, args_after):
    diags, lowers, uppers, x, parent_safe, has_parent = ctx.saved_tensors
    lam = kernel_op(diags, uppers, lowers, grad_x.contiguous(), *args_after)
    g_diags = -lam * x
    g_uppers = torch.where(has_parent, -lam[..., parent_safe] * x, torch.zeros_like(x))
    g_lowers = torch.where(has_parent, -lam * x[..., parent_safe], torch.zeros_like(x))
    return g_diags, g_lowers, g_uppers, lam


def _define_ops():
    global _NS
    _define_in(OP_NAMESPACE)
    _NS = OP_NAMESPACE


def _define_in(ns: str):
    global tree_solve_op, tree_solve_levels_op

    @torch.library.custom_op(f"{ns}::tree_solve", mutates_args=())
    def _tree_solve(diags: torch.Tensor, lowers: torch.Tensor, uppers: torch.Tensor,
                    solves: torch.Tensor, block_info: torch.Tensor, rel_parent: torch.Tensor,
                    rel_height: torch.Tensor, rel_children: torch.Tensor,
                    parent_safe: torch.Tensor, has_parent: torch.Tensor, block_size: int,
                    num_slots: int, num_warps: int) -> torch.Tensor:
        """Registers-variant tree solve (reference `tree_solve.py:518-563`)."""
        return _kernel_for(block_info, parent_safe, has_parent, "registers").solve(diags, lowers, uppers, solves)

    @_tree_solve.register_fake
    def _(diags, lowers, uppers, solves, *args):
        return torch.empty_like(solves)

    def _setup(ctx, inputs, output):
        ctx.save_for_backward(inputs[0], inputs[1], inputs[2], output, inputs[8], inputs[9])
        ctx.rest = inputs[4:]

    def _backward(ctx, grad_x):
        g = _transposed_backward(_tree_solve, ctx, grad_x, ctx.rest)
        return g + (None,) * 9

    _tree_solve.register_autograd(_backward, setup_context=_setup)

    @torch.library.custom_op(f"{ns}::tree_solve_levels", mutates_args=())
    def _tree_solve_levels(diags: torch.Tensor, lowers: torch.Tensor, uppers: torch.Tensor,
                           solves: torch.Tensor, block_info: torch.Tensor,
                           level_ptr: torch.Tensor, ordered_nodes: torch.Tensor,
                           ordered_parent: torch.Tensor, ordered_children: torch.Tensor,
                           parent_safe: torch.Tensor, has_parent: torch.Tensor, num_slots: int,
                           w: int) -> torch.Tensor:
        """Levels-variant tree solve (reference `tree_solve.py:589-609`)."""
        return _kernel_for(block_info, parent_safe, has_parent, "levels").solve(diags, lowers, uppers, solves)

    @_tree_solve_levels.register_fake
    def _(diags, lowers, uppers, solves, *args):
        return torch.empty_like(solves)

    def _setup_l(ctx, inputs, output):
        ctx.save_for_backward(inputs[0], inputs[1], inputs[2], output, inputs[9], inputs[10])
        ctx.rest = inputs[4:]

    def _backward_l(ctx, grad_x):
        g = _transposed_backward(_tree_solve_levels, ctx, grad_x, ctx.rest)
        return g + (None,) * 9

    _tree_solve_levels.register_autograd(_backward_l, setup_context=_setup_l)
    tree_solve_op = _tree_solve
    tree_solve_levels_op = _tree_solve_levels


def fused_tree_solve(kernel, diags, lowers, uppers, solves):
    """Differentiable fused tree solve (reference `tree_solve.py:633-635`)."""
    return kernel.fused(diags, lowers, uppers, solves)
