"""Device-side model and launches of the fused simulation kernels.

`DeviceModel` uploads a `Lowered` model once (the reference uploads its index tensors
once per step plan, `modules/base.py:3010-3023`) and builds the `JxbSimArgs` of a
launch. `Simulation` runs the step loop of `jx.integrate` (`integrate.py:396-666`):
one launch computes the initial currents and the first recording, the step launches
follow either one per step (the plain per-step drop-in) or one per segment of
`segment` steps (the persistent form, states resident in shared memory).
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Optional

import numpy as np
import torch

from . import _lib
from .lower import Lowered, lower
from .problem import Problem


def _dtype_code(dtype: torch.dtype) -> int:
    if dtype == torch.float32:
        return _lib.F32
    if dtype == torch.float64:
        return _lib.F64
    raise TypeError(f"unsupported dtype {dtype}")


def _ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else t.data_ptr()


class DeviceModel:
    """A lowered model resident on one GPU."""

    def __init__(self, low: Lowered, dtype: torch.dtype = torch.float32, device="cuda",
                 rows_per_item: int = 1):
        self.low = low
        self.dtype = dtype
        self.device = torch.device(device)
        self.code = _dtype_code(dtype)
        dev = self.device

        def f(x):
            return torch.as_tensor(np.asarray(x, dtype=np.float64), dtype=dtype, device=dev).contiguous()

        def i(x):
            return torch.as_tensor(np.asarray(x, dtype=np.int32), device=dev).contiguous()

        self.t = {
            "node_class": i(low.node_class), "soff": i(low.soff), "poff": i(low.poff),
            "a_low": f(low.a_low), "a_up": f(low.a_up), "gsum": f(low.gsum), "cm": f(low.cm),
            "area": f(low.area), "cls_ptr": i(low.cls_ptr), "cls_comp": i(low.cls_comp),
            "entries": torch.as_tensor(low.entries.astype(np.int16), device=dev).contiguous(),
            "pbase": f(low.pbase), "pcol": i(low.pcol), "blocks": i(low.blocks),
            "chain_top": i(low.chain_top), "chain_len": i(low.chain_len),
            "chain_ptop": i(low.chain_ptop), "chain_cptr": i(low.chain_cptr),
            "chain_child": i(low.chain_child) if len(low.chain_child) else i(np.zeros(1)),
            "level_ptr": i(low.level_ptr), "stim_ptr": i(low.stim_ptr),
            "stim_idx": i(low.stim_idx) if len(low.stim_idx) else i(np.zeros(1)),
            "rec_ptr": i(low.rec_ptr),
            "rec_slot": i(low.rec_slot) if len(low.rec_slot) else i(np.zeros(1)),
            "rec_col": i(low.rec_col) if len(low.rec_col) else i(np.zeros(1)),
        }
        self.pscale = f(low.pscale)
        self.stim = f(low.stim) if low.stim is not None else None
        self.set_rows_per_item(rows_per_item)

    def set_rows_per_item(self, rows: int) -> None:
        low = self.low
        B = low.batch
        rows = max(1, min(int(rows), B))
        items = []
        for b in range(len(low.blocks)):
            for r0 in range(0, B, rows):
                items.append([b, r0, min(rows, B - r0), 0])
        # Largest blocks first: CTAs are scheduled roughly in index order.
        sizes = np.asarray([low.blocks[it[0]][1] for it in items])
        order = np.argsort(-sizes, kind="stable")
        items = [items[k] for k in order]
        self.rows_per_item = rows
        self.items = torch.as_tensor(np.asarray(items, dtype=np.int32), device=self.device).contiguous()
        self.n_items = len(items)

    def args(self, state: torch.Tensor, n_steps: int, t0: int, rec_out: Optional[torch.Tensor],
             mode: int = 0, ckpt=None, ckpt_every: int = 0, ckpt_base: int = 0, traj=None,
             pscale: Optional[torch.Tensor] = None, syn_lin=None, syn_const=None,
             adj=None, rec_grad=None, pgrad=None) -> _lib.JxbSimArgs:
        low, t = self.low, self.t
        a = _lib.JxbSimArgs()
        a.dtype = self.code
        a.batch = low.batch
        a.n_nodes = low.n_nodes
        a.n_slots = low.n_slots
        a.n_pslots = low.n_pslots
        a.n_cols = low.n_cols
        a.n_items = self.n_items
        a.n_steps = n_steps
        a.t0 = t0
        a.max_rows = self.rows_per_item
        a.max_nodes = int(low.blocks[:, 1].max())
        a.max_slots = int(low.blocks[:, 3].max())
        a.dt = low.dt
        for k in ["node_class", "soff", "poff", "a_low", "a_up", "gsum", "cm", "cls_ptr",
                  "cls_comp", "entries", "pbase", "pcol", "blocks", "chain_top", "chain_len",
                  "chain_ptop", "chain_cptr", "chain_child", "level_ptr", "stim_ptr", "stim_idx",
                  "area", "rec_ptr", "rec_slot", "rec_col"]:
            setattr(a, k, t[k].data_ptr())
        a.items = self.items.data_ptr()
        a.n_classes = len(low.cls_comp)
        a.n_entries = int(low.entries.shape[0])
        a.pscale = (pscale if pscale is not None else self.pscale).data_ptr()
        if self.stim is not None:
            a.stim = self.stim.data_ptr()
            a.n_stim = self.stim.shape[2]
            a.stim_steps = self.stim.shape[0]
            a.stim_rows = self.stim.shape[1]
        a.syn_lin = _ptr(syn_lin)
        a.syn_const = _ptr(syn_const)
        a.rec_out = _ptr(rec_out)
        a.n_rec = low.n_rec
        a.state = state.data_ptr()
        a.ckpt = _ptr(ckpt)
        a.ckpt_every = ckpt_every
        a.ckpt_base = ckpt_base
        a.traj = _ptr(traj)
        a.adj = _ptr(adj)
        a.rec_grad = _ptr(rec_grad)
        a.pgrad = _ptr(pgrad)
        a.mode = mode
        return a

    def launch_forward(self, args: _lib.JxbSimArgs, stream=None) -> None:
        lib = _lib.load()
        s = stream if stream is not None else torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(lib.jxb_sim_forward(C.byref(args), C.c_void_p(s)), "jxb_sim_forward")

    def launch_backward(self, args: _lib.JxbSimArgs, stream=None) -> None:
        lib = _lib.load()
        s = stream if stream is not None else torch.cuda.current_stream(self.device).cuda_stream
        _lib.check(lib.jxb_sim_backward(C.byref(args), C.c_void_p(s)), "jxb_sim_backward")

    def initial_state(self) -> torch.Tensor:
        return torch.as_tensor(self.low.state0, dtype=self.dtype, device=self.device).contiguous()


class Simulation:
    """`jx.integrate` for a `Problem` on the CUDA kernels.

    `segment` is the number of steps per launch (1 = the plain per-step drop-in;
    `None` = the whole horizon in one persistent launch).
    """

    def __init__(self, problem: Problem, dtype=torch.float32, device="cuda",
                 max_block_nodes: int = 4096, rows_per_item: int = 1,
                 segment: Optional[int] = None, init_steady: bool = False,
                 low: Optional[Lowered] = None):
        self.problem = problem
        self.low = low if low is not None else lower(problem, max_block_nodes=max_block_nodes)
        self.model = DeviceModel(self.low, dtype, device, rows_per_item)
        self.segment = segment
        self.init_steady = init_steady

    def run(self, n_steps: Optional[int] = None, pscale: Optional[torch.Tensor] = None,
            return_state: bool = False):
        m = self.model
        low = self.low
        T = low.n_steps if n_steps is None else int(n_steps)
        state = m.initial_state()
        rec = torch.zeros((T + 1, low.batch, low.n_rec), dtype=m.dtype, device=m.device)
        m.launch_forward(m.args(state, 0, 0, rec, mode=2 if self.init_steady else 1, pscale=pscale))
        seg = T if not self.segment else int(self.segment)
        t = 0
        while t < T:
            k = min(seg, T - t)
            m.launch_forward(m.args(state, k, t, rec, pscale=pscale))
            t += k
        out = rec.permute(1, 2, 0)
        return (out, state) if return_state else out
