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
from .problem import Problem, host_mode, unwrap


def _dtype_code(dtype: torch.dtype) -> int:
    if dtype == torch.float32:
        return _lib.F32
    if dtype == torch.float64:
        return _lib.F64
    raise TypeError(f"unsupported dtype {dtype}")


def _ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else t.data_ptr()


def class_costs(low: Lowered) -> np.ndarray:
    """Relative cost of one node of every class in the per-node phases: a channel
    costs its overhead plus its gates, the interpreter (classes without a
    compile-time program) about 1.7 times a program, a branchpoint (no channels)
    only its assembly."""
    out = np.zeros(len(low.cls_comp))
    for c in range(len(out)):
        if not low.cls_comp[c]:
            out[c] = 0.15
            continue
        ents = low.entries[low.cls_ptr[c]:low.cls_ptr[c + 1]]
        cost = 0.3 + sum(0.5 + 1.5 * int(e[1]) for e in ents)
        out[c] = cost * (1.0 if low.cls_prog[c] else 1.7)
    return out


def node_schedule(low: Lowered, n_warps: int):
    """Per block, the nodes every warp visits in the per-node phases: the block's nodes
    are cut into chunks of up to 32 nodes of one class (in node order), and the
    chunks go, most expensive first, to the warp with the least work so far. Returns
    `(sched_ptr (n_blocks + 1,) int32, sched int16)` in the layout of
    `JxbSimArgs.sched`."""
    import heapq

    cost = class_costs(low)
    parts, ptr = [], [0]
    for b in low.blocks:
        n0, nn = int(b[0]), int(b[1])
        cls = low.node_class[n0:n0 + nn]
        chunks = []  # (cost, node indices)
        for c in np.unique(cls):
            nodes = np.nonzero(cls == c)[0]
            for k in range(0, len(nodes), 32):
                chunks.append((float(cost[c]), nodes[k:k + 32]))
        order = sorted(range(len(chunks)), key=lambda q: -chunks[q][0])
        heap = [(0.0, w) for w in range(n_warps)]
        lists: List[List[int]] = [[] for _ in range(n_warps)]
        for q in order:
            load, w = heapq.heappop(heap)
            lists[w].append(q)
            heapq.heappush(heap, (load + chunks[q][0], w))
        kmax = max(1, max(len(x) for x in lists))
        arr = np.full((n_warps, kmax, 32), -1, dtype=np.int16)
        for w in range(n_warps):
            for k, q in enumerate(lists[w]):
                nodes = chunks[q][1]
                arr[w, k, :len(nodes)] = nodes
        parts.append(arr.reshape(-1))
        ptr.append(ptr[-1] + arr.size)
    return np.asarray(ptr, dtype=np.int32), np.concatenate(parts)


class DeviceModel:
    """A lowered model resident on one GPU."""

    def __init__(self, low: Lowered, dtype: torch.dtype = torch.float32, device="cuda",
                 rows_per_item: int = 1, threads: int = 256, programs: bool = True,
                 smem_limit: Optional[int] = None, schedule: bool = True,
                 forward_threads: Optional[int] = None, forward_wide: bool = False,
                 tangent: bool = False, gm_threads: Optional[int] = None):
        self.low = low
        self.dtype = dtype
        self.device = torch.device(device)
        self.code = _dtype_code(dtype)
        # With `tangent`, every floating-point array holds (value, tangent) pairs in a
        # trailing dimension of 2 (tangents zero) and only forward launches are taken
        # (`jxb_sim_tangent`, the forward kernel in dual numbers).
        self.tangent = bool(tangent)
        self.itemsize = torch.empty((), dtype=dtype).element_size() * (2 if tangent else 1)
        dev = self.device

        def f(x):
            x = torch.as_tensor(np.asarray(x, dtype=np.float64), dtype=dtype, device=dev)
            if tangent:
                x = torch.stack([x, torch.zeros_like(x)], -1)
            return x.contiguous()

        def i(x):
            return torch.as_tensor(np.asarray(x, dtype=np.int32), device=dev).contiguous()

        self.t = {
            "node_class": i(low.node_class), "soff": i(low.soff), "poff": i(low.poff),
            "a_low": f(low.a_low), "a_up": f(low.a_up), "gsum": f(low.gsum), "cm": f(low.cm),
            "area": f(low.area), "cls_ptr": i(low.cls_ptr), "cls_comp": i(low.cls_comp),
            "cls_prog": i(low.cls_prog),
            "entries": torch.as_tensor(low.entries.astype(np.int16), device=dev).contiguous(),
            "pbase": f(low.pbase), "pcol": i(low.pcol), "blocks": i(low.blocks),
            "chain_top": i(low.chain_top), "chain_len": i(low.chain_len),
            "chain_ptop": i(low.chain_ptop), "chain_cptr": i(low.chain_cptr),
            "chain_child": i(low.chain_child) if len(low.chain_child) else i(np.zeros(1)),
            "level_ptr": i(low.level_ptr), "stim_ptr": i(low.stim_ptr),
            "stim_idx": i(low.stim_idx) if len(low.stim_idx) else i(np.zeros(1)),
            "gk": i(low.gk) if len(low.gk) else i(np.zeros(1)), "gbase": i(low.gbase),
            "rec_ptr": i(low.rec_ptr), "parent": i(low.parent), "kid_ptr": i(low.kid_ptr),
            "kid": i(low.kid) if len(low.kid) else i(np.zeros(1)),
            "rec_slot": i(low.rec_slot) if len(low.rec_slot) else i(np.zeros(1)),
            "rec_col": i(low.rec_col) if len(low.rec_col) else i(np.zeros(1)),
        }
        if not programs:
            self.t["cls_prog"] = torch.zeros_like(self.t["cls_prog"])
        self.pscale = f(low.pscale)
        self.stim = f(low.stim) if low.stim is not None else None
        self.clamp = None
        if getattr(low, "clamp", None) is not None:
            self.clamp = f(low.clamp)
            self.t["clamp_ptr"] = i(low.clamp_ptr)
            self.t["clamp_slot"] = i(low.clamp_slot)
            self.t["clamp_col"] = i(low.clamp_col)
        self.threads = threads
        # Failure flag of the launches (JXB_NONFINITE when a result is not finite).
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)
        self.launches = 0  # kernel launches issued through this model
        self.timed_kind: Optional[str] = None  # "forward"/"backward": record events
        self.events: List = []
        # With `group_timing`, every group launch records (kind, group key, items,
        # start, end) events on the stream it runs on, in `group_events`.
        self.group_timing = False
        self.group_events: List = []
        self._sides: List[torch.cuda.Stream] = []
        self._scratch: Dict[str, torch.Tensor] = {}
        self.smem_limit = smem_limit if smem_limit is not None else self._device_smem_limit()
        # Threads per CTA of each launch kind (the forward may use fewer, with the wide
        # register budget of JxbSimArgs.wide) and a node schedule for each warp count.
        self.kind_threads = {"forward": int(forward_threads or threads), "backward": int(threads)}
        if tangent:
            self.kind_threads["forward"] = min(self.kind_threads["forward"], 512)
        self.forward_wide = bool(forward_wide) and not tangent
        # adjoint launches on the kernels of two CTAs per SM with up to 128 registers
        # (float32, up to 256 threads; set by callers whose items fit in one wave)
        self.backward_wide = False
        # Threads per CTA of the groups whose work areas live in global memory (blocks
        # too large for shared memory; they run one CTA per SM at most, so they can
        # use more threads than the shared-memory groups).
        self.gm_threads = int(gm_threads) if gm_threads else None
        if tangent and self.gm_threads:
            self.gm_threads = min(self.gm_threads, 512)
        self.sched_warps = 0
        self.kind_sched: Dict[str, tuple] = {}
        self.gm_sched: Optional[tuple] = None
        if schedule:
            by_warps: Dict[int, tuple] = {}

            def sched_for(th):
                w = th // 32
                if w not in by_warps:
                    sp, sc = node_schedule(low, w)
                    by_warps[w] = (w, i(sp), torch.as_tensor(sc, device=dev).contiguous())
                return by_warps[w]

            for kind, th in self.kind_threads.items():
                if th % 32:
                    continue
                self.kind_sched[kind] = sched_for(th)
            if self.gm_threads and self.gm_threads % 32 == 0:
                self.gm_sched = sched_for(self.gm_threads)
            if "backward" in self.kind_sched:
                w, sp_t, sc_t = self.kind_sched["backward"]
                self.t["sched_ptr"], self.t["sched"], self.sched_warps = sp_t, sc_t, w
        self.set_rows_per_item(rows_per_item)

    def _device_smem_limit(self) -> int:
        if self.device.type == "cuda" and torch.cuda.is_available():
            props = torch.cuda.get_device_properties(self.device)
            v = getattr(props, "shared_memory_per_block_optin", 0)
            if v:
                return int(v)
        return 227 * 1024

    def _block_maxima(self, bidx: np.ndarray) -> Dict[str, int]:
        blocks = self.low.blocks[bidx]
        cp = self.low.chain_cptr
        return {
            "max_nodes": int(blocks[:, 1].max()), "max_slots": int(blocks[:, 3].max()),
            "max_chains": int(blocks[:, 5].max()), "max_levels": int(blocks[:, 7].max()),
            "max_pslots": max(1, int(blocks[:, 9].max())), "max_gslots": max(1, int(blocks[:, 10].max())),
            "max_child": int(max(cp[b[4] + b[5]] - cp[b[4]] for b in blocks)),
        }

    def _layout_bytes(self, maxima: Dict[str, int], backward: bool) -> int:
        a = _lib.JxbSimArgs()
        a.dtype = self.code
        a.max_rows = self.rows_per_item
        if backward:
            a.gacc = 256  # gradient slots in global memory (placeholder address for sizing)
        for k, v in maxima.items():
            setattr(a, k, v)
        a.n_entries = int(self.low.entries.shape[0])
        a.n_classes = len(self.low.cls_comp)
        if self.tangent and not backward:
            return int(_lib.load().jxb_sim_tangent_smem_bytes(C.byref(a)))
        return int(_lib.load().jxb_sim_smem_bytes(C.byref(a), int(backward)))

    def set_rows_per_item(self, rows: int) -> None:
        """Work items = (block, rows), grouped per launch kind by the shared memory
        their block needs: one launch per size class (up to a quarter, a half, all of
        a CTA's shared memory, so that small blocks keep several CTAs per SM) and one
        for blocks over the limit, whose work areas live in global scratch. The
        groups run concurrently on forked streams."""
        low = self.low
        B = low.batch
        rows = max(1, min(int(rows), B))
        self.rows_per_item = rows
        nb = len(low.blocks)
        limits = [self.smem_limit // 4, self.smem_limit // 2, self.smem_limit]
        self.groups: Dict[str, list] = {}
        for kind in ("forward", "backward"):
            bwd = kind == "backward"
            own = [self._block_maxima(np.asarray([b])) for b in range(nb)]
            need = np.asarray([self._layout_bytes(mx, bwd) for mx in own])
            # A class's layout is sized by the maxima over its blocks (nodes of one,
            # slots of another...): admit blocks smallest first while it still fits.
            cls = np.full(nb, -1, dtype=np.int64)  # -1: global scratch
            run: List[Optional[Dict[str, int]]] = [None] * len(limits)
            for b in np.argsort(need, kind="stable"):
                for c, lim in enumerate(limits):
                    if need[b] > lim:
                        continue
                    cand = own[b] if run[c] is None else {k: max(v, own[b][k]) for k, v in run[c].items()}
                    if self._layout_bytes(cand, bwd) <= lim:
                        cls[b] = c
                        run[c] = cand
                        break
            groups = []
            for c in [-1] + list(range(len(limits) - 1, -1, -1)):  # longest items first
                sel = np.nonzero(cls == c)[0]
                if len(sel) == 0:
                    continue
                items = [[int(b), r0, min(rows, B - r0), 0] for b in sel for r0 in range(0, B, rows)]
                # Largest blocks first: CTAs are scheduled roughly in index order.
                sizes = np.asarray([low.blocks[it[0]][1] for it in items])
                items = [items[k] for k in np.argsort(-sizes, kind="stable")]
                maxima = self._block_maxima(sel)
                stride = (self._layout_bytes(maxima, bwd) + 255) // 256 * 256
                gstride = (rows * maxima["max_gslots"] * self.itemsize + 255) // 256 * 256
                groups.append({
                    "gm": c < 0, "maxima": maxima, "n_items": len(items), "stride": stride,
                    "gacc_stride": gstride if bwd else 0, "key": (kind, c),
                    "items": torch.as_tensor(np.asarray(items, dtype=np.int32), device=self.device).contiguous(),
                })
            self.groups[kind] = groups
        self.n_items = sum(g["n_items"] for g in self.groups["forward"])

    def args(self, state: torch.Tensor, n_steps: int, t0: int, rec_out: Optional[torch.Tensor],
             mode: int = 0, ckpt=None, ckpt_every: int = 0, ckpt_base: int = 0, traj=None,
             pscale: Optional[torch.Tensor] = None, syn_lin=None, syn_const=None,
             adj=None, rec_grad=None, pgrad=None) -> _lib.JxbSimArgs:
        """Arguments of a launch; the per-group fields (items, block maxima, global
        scratch) are filled in by `launch_forward` / `launch_backward`."""
        low, t = self.low, self.t
        a = _lib.JxbSimArgs()
        a.dtype = self.code
        a.batch = low.batch
        a.n_nodes = low.n_nodes
        a.n_slots = low.n_slots
        a.n_pslots = low.n_pslots
        a.n_cols = low.n_cols
        a.n_steps = n_steps
        a.t0 = t0
        a.max_rows = self.rows_per_item
        a.threads = self.threads
        a.dt = low.dt
        for k in ["node_class", "soff", "poff", "a_low", "a_up", "gsum", "cm", "cls_ptr",
                  "cls_comp", "cls_prog", "entries", "pbase", "pcol", "blocks", "chain_top", "chain_len",
                  "chain_ptop", "chain_cptr", "chain_child", "level_ptr", "stim_ptr", "stim_idx",
                  "area", "rec_ptr", "rec_slot", "rec_col", "parent", "kid_ptr", "kid",
                  "gk", "gbase"]:
            setattr(a, k, t[k].data_ptr())
        a.n_classes = len(low.cls_comp)
        a.n_entries = int(low.entries.shape[0])
        a.pscale = (pscale if pscale is not None else self.pscale).data_ptr()
        if self.stim is not None:
            a.stim = self.stim.data_ptr()
            a.n_stim = self.stim.shape[2]
            a.stim_steps = self.stim.shape[0]
            a.stim_rows = self.stim.shape[1]
        if self.clamp is not None:
            a.clamp_ptr = t["clamp_ptr"].data_ptr()
            a.clamp_slot = t["clamp_slot"].data_ptr()
            a.clamp_col = t["clamp_col"].data_ptr()
            a.clamp = self.clamp.data_ptr()
            a.clamp_steps, a.clamp_rows, a.n_clamp = self.clamp.shape[:3]
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
        a.status = self.status.data_ptr()
        a.scheme = int(getattr(low, "scheme", 0))
        if self.sched_warps:
            a.sched_ptr = t["sched_ptr"].data_ptr()
            a.sched = t["sched"].data_ptr()
            a.sched_warps = self.sched_warps
        return a

    def scratch(self, kind: str, group) -> torch.Tensor:
        """Global work areas of a group of oversized blocks (allocated once)."""
        return self._buffer(("work", kind), group["n_items"] * group["stride"] + 256)

    def group_args(self, args: _lib.JxbSimArgs, kind: str, group) -> _lib.JxbSimArgs:
        """A copy of `args` completed for one item group of a launch kind."""
        a = _lib.JxbSimArgs.from_buffer_copy(args)
        for k, v in group["maxima"].items():
            setattr(a, k, v)
        if kind in self.kind_threads:
            a.threads = self.kind_threads[kind]
            a.wide = int((kind == "forward" and self.forward_wide)
                         or (kind == "backward" and self.backward_wide))
            ks = self.kind_sched.get(kind)
            if group["gm"] and self.gm_threads:
                a.threads, a.wide, ks = self.gm_threads, 0, self.gm_sched
            if ks is not None:
                a.sched_warps, a.sched_ptr, a.sched = ks[0], ks[1].data_ptr(), ks[2].data_ptr()
        a.items = group["items"].data_ptr()
        a.n_items = group["n_items"]
        if group["gm"]:
            buf = self.scratch(kind, group)
            a.gscratch = (buf.data_ptr() + 255) // 256 * 256
            a.gscratch_stride = group["stride"]
        if group["gacc_stride"]:
            buf = self._buffer(("gacc",) + group["key"], group["n_items"] * group["gacc_stride"] + 256)
            a.gacc = (buf.data_ptr() + 255) // 256 * 256
            a.gacc_stride = group["gacc_stride"]
        return a

    def _buffer(self, key, nbytes: int) -> torch.Tensor:
        buf = self._scratch.get(key)
        if buf is None or buf.numel() < nbytes:
            buf = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
            self._scratch[key] = buf
        return buf

    def _launch(self, kind: str, fn, args, stream) -> None:
        st = torch.cuda.current_stream(self.device)
        main = stream if stream is not None else st.cuda_stream
        groups = self.groups[kind]
        timed = self.timed_kind == kind and stream is None
        if timed:
            e0 = torch.cuda.Event(enable_timing=True)
            e0.record(st)
        fork = len(groups) > 1 and stream is None
        if fork:  # every group but the last on its own side stream, joined below
            while len(self._sides) < len(groups) - 1:
                self._sides.append(torch.cuda.Stream(self.device))
            for side in self._sides[:len(groups) - 1]:
                side.wait_stream(st)
        for gi, g in enumerate(groups):
            a = self.group_args(args, kind, g)
            side = self._sides[gi] if (fork and gi < len(groups) - 1) else None
            s = side.cuda_stream if side is not None else main
            ev = None
            if self.group_timing and stream is None:
                ev = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
                ev[0].record(side if side is not None else st)
            _lib.check(fn(C.byref(a), C.c_void_p(s)), f"jxb_sim_{kind}")
            if ev is not None:
                ev[1].record(side if side is not None else st)
                self.group_events.append((kind, g["key"], g["n_items"], ev[0], ev[1]))
            self.launches += 1
        if fork:
            for side in self._sides[:len(groups) - 1]:
                st.wait_stream(side)
        if timed:
            e1 = torch.cuda.Event(enable_timing=True)
            e1.record(st)
            self.events.append((e0, e1, args.n_steps))

    def check_finite(self, what: str) -> None:
        """Raises `FloatingPointError` when a launch since the last check produced a value
        that is not finite (the kernels' status flag; reading it synchronises the
        device). Skipped while a CUDA graph is being captured: the flag stays set until
        the next check outside a capture."""
        if torch.cuda.is_current_stream_capturing():
            return
        flag = int(self.status.item())
        if flag:
            self.status.zero_()
            if flag & _lib.JXB_TIMEOUT:
                raise RuntimeError(f"a wait for an asynchronous copy in the {what} gave up (results invalid)")
            raise FloatingPointError(f"the {what} produced values that are not finite (NaN or inf)")

    def launch_forward(self, args: _lib.JxbSimArgs, stream=None) -> None:
        lib = _lib.load()
        self._launch("forward", lib.jxb_sim_tangent if self.tangent else lib.jxb_sim_forward, args, stream)

    def launch_backward(self, args: _lib.JxbSimArgs, stream=None) -> None:
        if self.tangent:
            raise RuntimeError("a tangent model runs forward launches only")
        self._launch("backward", _lib.load().jxb_sim_backward, args, stream)

    def initial_state(self) -> torch.Tensor:
        """A fresh copy of the initial state (uploaded once, copied on the device);
        (value, zero tangent) pairs for a tangent model."""
        if getattr(self, "_state0", None) is None:
            s0 = torch.as_tensor(self.low.state0, dtype=self.dtype, device=self.device)
            if self.tangent:
                s0 = torch.stack([s0, torch.zeros_like(s0)], -1)
            self._state0 = s0.contiguous()
        return self._state0.clone()


class Simulation:
    """`jx.integrate` for a `Problem` on the CUDA kernels.

    `segment` is the number of steps per launch (1 = the plain per-step drop-in;
    `None` = the whole horizon in one persistent launch). `checkpoint` is the number
    of steps per adjoint launch. `store_trajectory`: the forward stores the state
    before every step and the pivots of every step, and the adjoint reads them
    instead of recomputing each segment from a stored state every `checkpoint` steps
    (`"auto"`: for persistent launches, when the trajectory takes at most
    `store_fraction` of the free device memory). `threads` is the CTA size of the
    launches; `forward_threads` (default: `threads`) that of the forward launches,
    which with `forward_wide` (float32, up to 256 threads) use kernels of two CTAs per
    SM with up to 128 registers a thread instead of 64. `gm_threads` (default: as the
    kind's) is the CTA size of the launches of blocks whose work areas live in global
    memory. With `check_finite`, a run whose final states or gradients hold a NaN or
    an infinity raises `FloatingPointError` (the kernels flag it on the device).
    """

    def __init__(self, problem: Problem, dtype=torch.float32, device="cuda",
                 max_block_nodes: int = 4096, rows_per_item: int = 1,
                 segment: Optional[int] = None, init_steady: bool = False,
                 low: Optional[Lowered] = None, checkpoint: int = 100, threads: int = 256,
                 keep_currents: bool = True, programs: bool = True, schedule: bool = True,
                 store_trajectory="auto", store_fraction: float = 0.5,
                 forward_threads: Optional[int] = None, forward_wide: bool = False,
                 check_finite: bool = True, gm_threads: Optional[int] = None):
        self.problem = problem
        self.low = low if low is not None else lower(problem, max_block_nodes=max_block_nodes,
                                                     keep_currents=keep_currents)
        self.model = DeviceModel(self.low, dtype, device, rows_per_item, threads=threads,
                                 programs=programs, schedule=schedule,
                                 forward_threads=forward_threads, forward_wide=forward_wide,
                                 gm_threads=gm_threads)
        self.segment = segment
        self.init_steady = init_steady
        self.checkpoint = int(checkpoint)
        if store_trajectory not in (True, False, "auto"):
            raise ValueError("store_trajectory must be True, False or 'auto'")
        self.store_trajectory = store_trajectory
        self.store_fraction = float(store_fraction)
        self._store_free: Optional[int] = None
        # Raise FloatingPointError when a run's final states or gradients are not
        # finite (as the reference's trainer does for a non-finite loss,
        # training/engine.py:229-230); one device synchronisation per run.
        self.check_finite = bool(check_finite)

    def n_steps(self, n_steps: Optional[int] = None) -> int:
        return self.low.n_steps if n_steps is None else int(n_steps)

    def trajectory_bytes(self, T: int) -> int:
        """Device bytes of a stored trajectory of T steps (states and pivots)."""
        low = self.low
        item = torch.empty((), dtype=self.model.dtype).element_size()
        return ((T + 1) * low.n_slots + T * low.n_nodes) * low.batch * item

    def stores_trajectory(self, T: int) -> bool:
        """Whether a differentiable run of T steps stores its trajectory."""
        if self.store_trajectory != "auto":
            return bool(self.store_trajectory)
        if self.segment is not None:
            return False
        if self._store_free is None:  # sampled once, outside any graph capture
            if torch.cuda.is_current_stream_capturing():
                return False
            self._store_free = torch.cuda.mem_get_info(self.model.device)[0]
        return self.trajectory_bytes(T) <= self.store_fraction * self._store_free

    def forward_raw(self, pscale: torch.Tensor, T: int, ckpt: Optional[torch.Tensor] = None,
                    traj: Optional[torch.Tensor] = None, piv: Optional[torch.Tensor] = None):
        """Runs the forward pass; returns `(rec (T+1, B, n_rec), final state)`. With
        `traj (T+1, B, n_slots)` and `piv (T, B, n_nodes)` it also stores the state
        before every step (and after the last) and the reciprocal pivots."""
        m = self.model
        low = self.low
        state = m.initial_state()
        rec = torch.zeros((T + 1, low.batch, low.n_rec), dtype=m.dtype, device=m.device)
        m.launch_forward(m.args(state, 0, 0, rec, mode=2 if self.init_steady else 1, pscale=pscale))
        seg = T if not self.segment else int(self.segment)
        if ckpt is not None:
            seg = min(seg, self.checkpoint) if self.segment else self.checkpoint * max(1, seg // self.checkpoint)
        t = 0
        while t < T:
            k = min(seg, T - t)
            a = m.args(state, k, t, rec, pscale=pscale, ckpt=ckpt,
                       ckpt_every=self.checkpoint if ckpt is not None else 0,
                       traj=traj[t] if traj is not None else None)
            if piv is not None:
                a.traj_piv = piv[t].data_ptr()
            m.launch_forward(a)
            t += k
        self.last_state = state  # the final state of the latest forward run (B, n_slots)
        return rec, state

    def backward_raw(self, pscale: torch.Tensor, T: int, ckpt: torch.Tensor,
                     rec_grad: torch.Tensor) -> torch.Tensor:
        """Adjoint of the recordings' gradient `rec_grad (T+1, B, n_rec)`: returns
        d loss / d pscale, float64 `(B, n_cols)`."""
        m = self.model
        low = self.low
        K = self.checkpoint
        nseg = (T + K - 1) // K
        adj = torch.zeros((low.batch, low.n_slots), dtype=m.dtype, device=m.device)
        pgrad = torch.zeros((low.batch, low.n_cols), dtype=torch.float64, device=m.device)
        traj = torch.empty((min(K, T), low.batch, low.n_slots), dtype=m.dtype, device=m.device)
        piv = torch.empty((min(K, T), low.batch, low.n_nodes), dtype=m.dtype, device=m.device)
        rec_grad = rec_grad.contiguous()
        for sgi in range(nseg - 1, -1, -1):
            t0 = sgi * K
            k = min(K, T - t0)
            a = m.args(ckpt[sgi], k, t0, None, pscale=pscale, traj=traj, adj=adj,
                       rec_grad=rec_grad, pgrad=pgrad)
            a.ckpt = ckpt[sgi].data_ptr()
            a.traj_piv = piv.data_ptr()
            m.launch_backward(a)
        return pgrad

    def backward_stored(self, pscale: torch.Tensor, T: int, traj: torch.Tensor, piv: torch.Tensor,
                        rec_grad: torch.Tensor) -> torch.Tensor:
        """`backward_raw` on the trajectory the forward stored (`forward_raw` with
        `traj`, `piv`): one adjoint launch per `checkpoint` steps, no recompute."""
        m = self.model
        low = self.low
        K = self.checkpoint
        nseg = (T + K - 1) // K
        adj = torch.zeros((low.batch, low.n_slots), dtype=m.dtype, device=m.device)
        pgrad = torch.zeros((low.batch, low.n_cols), dtype=torch.float64, device=m.device)
        rec_grad = rec_grad.contiguous()
        for sgi in range(nseg - 1, -1, -1):
            t0 = sgi * K
            k = min(K, T - t0)
            a = m.args(traj[t0], k, t0, None, pscale=pscale, traj=traj[t0], adj=adj,
                       rec_grad=rec_grad, pgrad=pgrad)
            a.ckpt = traj[t0].data_ptr()
            a.traj_piv = piv[t0].data_ptr()
            a.traj_stored = 1
            m.launch_backward(a)
        return pgrad

    def tangent_model(self) -> DeviceModel:
        """The model's arrays as (value, tangent) pairs, for `jvp` (built once)."""
        if getattr(self, "_tangent", None) is None:
            m = self.model
            self._tangent = DeviceModel(self.low, m.dtype, m.device, m.rows_per_item, threads=m.threads,
                                        schedule=bool(m.kind_sched), tangent=True, gm_threads=m.gm_threads)
        return self._tangent

    def jvp(self, pscale: torch.Tensor, pscale_tangent: torch.Tensor, n_steps: Optional[int] = None,
            state_tangent: Optional[torch.Tensor] = None):
        """Forward-mode derivative: returns the recordings `(B, n_rec, T + 1)` and their
        directional derivative along `pscale_tangent` (the tangent of the per-row
        parameter scales `(B, n_cols)`) and `state_tangent` (that of the initial state
        `(B, n_slots)`, default zero), as `torch.func.jvp` through the reference's
        `integrate` gives them (its tree solve's forward-mode rule,
        `solver_voltage.py:190-224`). One launch sequence of the forward kernel in dual
        numbers; the steps are the same launches as `run`'s."""
        if self.problem.synapses:
            raise NotImplementedError("forward-mode derivatives cover cells without synapses")
        tm = self.tangent_model()
        low = self.low
        T = self.n_steps(n_steps)
        dt = tm.dtype
        ps = torch.stack([pscale.detach().to(device=tm.device, dtype=dt),
                          pscale_tangent.detach().to(device=tm.device, dtype=dt)], -1).contiguous()
        state = tm.initial_state()
        if state_tangent is not None:
            state[..., 1] = state_tangent.to(device=tm.device, dtype=dt)
        rec = torch.zeros((T + 1, low.batch, low.n_rec, 2), dtype=dt, device=tm.device)
        tm.launch_forward(tm.args(state, 0, 0, rec, mode=2 if self.init_steady else 1, pscale=ps))
        seg = T if not self.segment else int(self.segment)
        t = 0
        while t < T:
            k = min(seg, T - t)
            tm.launch_forward(tm.args(state, k, t, rec, pscale=ps))
            t += k
        if self.check_finite:
            tm.check_finite("forward-mode derivative")
        out = rec.permute(1, 2, 0, 3)
        self.last_state_tangent = state  # (B, n_slots, 2)
        return out[..., 0], out[..., 1]

    def run(self, n_steps: Optional[int] = None, pscale: Optional[torch.Tensor] = None,
            return_state: bool = False):
        """Recordings `(B, n_rec, T + 1)`; differentiable with respect to `pscale`
        (the per-row scales of the parameter columns) when it requires grad."""
        T = self.n_steps(n_steps)
        if pscale is None:
            pscale = self.model.pscale
        reverse = pscale.requires_grad and torch.is_grad_enabled()
        if reverse or torch.autograd.forward_ad._current_level >= 0:
            return _IntegrateFn.apply(pscale, self, T, _Stash(reverse))
        rec, state = self.forward_raw(pscale.detach().contiguous(), T)
        if self.check_finite:
            self.model.check_finite("simulation")
        out = rec.permute(1, 2, 0)
        return (out, state) if return_state else out


class _Stash:
    """Hands `_IntegrateFn.forward`'s saved tensors to its `setup_context` (an object,
    so that `torch.func` passes it through unchanged)."""

    def __init__(self, reverse: bool):
        self.reverse = reverse
        self.saved = None


class _IntegrateFn(torch.autograd.Function):
    """Forward: the fused step kernels, storing the trajectory (states and pivots of
    every step) or a checkpoint every `sim.checkpoint` steps. Backward: the adjoint
    kernel per segment of `sim.checkpoint` steps, in reverse order (reverse sweep over
    the stored trajectory, or recompute + reverse sweep), instead of autograd through
    every operation of every step. Forward-mode rule (`torch.autograd.forward_ad`,
    `torch.func.jvp`): the steps once more in dual numbers (`Simulation.jvp`).

    With `stash.reverse` false (forward mode only) the forward stores no trajectory.
    Under `torch.func.jvp` / `torch.func.grad` the rules unwrap their operands and run
    the kernels with the functorch layers off (`host_mode`)."""

    @staticmethod
    def forward(pscale, sim, T, stash):
        low = sim.low
        K = sim.checkpoint
        nseg = (T + K - 1) // K
        ps = pscale.detach().to(sim.model.dtype).contiguous()
        dev, dt = sim.model.device, sim.model.dtype
        stored = stash.reverse and sim.stores_trajectory(T)
        if not stash.reverse:
            rec, _ = sim.forward_raw(ps, T)
            stash.saved = (False, ps)
        elif stored:
            traj = torch.empty((T + 1, low.batch, low.n_slots), dtype=dt, device=dev)
            piv = torch.empty((T, low.batch, low.n_nodes), dtype=dt, device=dev)
            rec, _ = sim.forward_raw(ps, T, traj=traj, piv=piv)
            stash.saved = (True, ps, traj, piv)
        else:
            ckpt = torch.empty((nseg, low.batch, low.n_slots), dtype=dt, device=dev)
            rec, _ = sim.forward_raw(ps, T, ckpt=ckpt)
            stash.saved = (False, ps, ckpt)
        if sim.check_finite:
            sim.model.check_finite("simulation")
        # Contiguous, so that a forward-mode tangent can have the output's layout.
        return rec.permute(1, 2, 0).contiguous()

    @staticmethod
    def setup_context(ctx, inputs, output):
        pscale, sim, T, stash = inputs
        ctx.sim, ctx.T = sim, T
        ctx.in_dtype = pscale.dtype
        ctx.saved = stash.saved  # (functorch may call this more than once per forward)

    @staticmethod
    def backward(ctx, grad_out):
        sim = ctx.sim
        if len(ctx.saved) < 3:
            raise RuntimeError("the simulation ran for forward-mode derivatives only (no trajectory stored)")
        with host_mode():
            rec_grad = unwrap(grad_out).detach().to(sim.model.dtype).permute(2, 0, 1).contiguous()
            if ctx.saved[0]:
                _, ps, traj, piv = ctx.saved
                pgrad = sim.backward_stored(ps, ctx.T, traj, piv, rec_grad)
            else:
                _, ps, ckpt = ctx.saved
                pgrad = sim.backward_raw(ps, ctx.T, ckpt, rec_grad)
            if sim.check_finite:
                sim.model.check_finite("adjoint")
            pgrad = pgrad.to(ctx.in_dtype)
        return pgrad, None, None, None

    @staticmethod
    def jvp(ctx, t_pscale, _sim, _T, _stash):
        sim = ctx.sim
        with host_mode():
            _, rec_t = sim.jvp(ctx.saved[1], unwrap(t_pscale).detach(), ctx.T)
            rec_t = rec_t.to(ctx.in_dtype).contiguous()
        return rec_t
