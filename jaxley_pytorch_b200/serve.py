"""Serving loop: continuous batching of simulation and gradient requests.

A request is one problem (a cell or a small network with its stimulus and
recordings), a horizon, and whether the gradient of its recordings' sum with respect
to its parameter columns is wanted. The server admits requests by an HBM budget,
keeps every admitted request's model, state and buffers resident on the device, and
advances all of them together: every tick issues one multi-request forward launch
(each request moves by up to `chunk` steps, storing checkpoints when it wants a
gradient) and, concurrently on a second stream, one multi-request adjoint launch
(each gradient request whose forward is complete runs one checkpoint segment, in
reverse order). Requests that arrive while others run join at the next tick;
finished requests are retired and their memory returns to the budget. The
reference has no such loop: `jx.integrate` simulates one module per call
(`integrate.py:396-666`); `serve_plain` is that per-request path on the same
kernels, for comparison.
"""
from __future__ import annotations

import ctypes as C
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import _lib
from .lower import Lowered, lower
from .problem import Problem
from .sim import DeviceModel, Simulation


def step_cost_us(low: Lowered, threads: int = 256) -> float:
    """Estimated microseconds of one forward step of a lowered problem's largest work
    item on an SM of its own: a fixed part, the chain levels of the tree solve (one
    pass down and one up each) and the per-node channel work spread over the CTA's
    threads (coefficients from per-phase timings of the fused kernel on the 300 x 4
    L5PC tree: solve 0.55 us per level and pass, channels 0.9 us per node a thread)."""
    blocks = np.asarray(low.blocks)
    levels = int(blocks[:, 7].max()) if len(blocks) else 1
    nodes = int(blocks[:, 1].max()) if len(blocks) else 1
    return 2.0 + 1.1 * levels + 0.9 * -(-nodes // max(1, threads))


@dataclass
class Request:
    """A simulation request. `grad`: also return d(sum of recordings)/d(parameter
    scale columns), float64 `(batch, n_cols)`."""

    problem: Problem
    n_steps: int
    grad: bool = False
    arrival: float = 0.0  # seconds after the start of the stream
    rid: int = -1
    # results
    recordings: Optional[np.ndarray] = None  # (batch, n_rec, n_steps + 1)
    gradient: Optional[np.ndarray] = None
    admitted: float = float("nan")
    finished: float = float("nan")
    service: float = float("nan")  # seconds of the request served alone (per-request path)

    @property
    def latency(self) -> float:
        return self.finished - self.arrival

    @property
    def slowdown(self) -> float:
        """Latency over the request's own latency when served alone."""
        return self.latency / self.service


def request_bytes(low: Lowered, n_steps: int, grad: bool, checkpoint: int, itemsize: int = 4) -> int:
    """Device memory a request holds while admitted: its lowered model, state,
    recordings and, for a gradient, the stored states, one segment's trajectory and
    pivots, the adjoint and the gradient."""
    B = low.batch
    model = (low.n_nodes * (8 * itemsize + 10 * 4) + low.n_pslots * (itemsize + 8)
             + len(low.chain_top) * 20 + low.entries.size * 2 + low.pscale.size * itemsize)
    b = model + B * low.n_slots * itemsize + (n_steps + 1) * B * max(low.n_rec, 1) * itemsize
    if grad:
        K = min(checkpoint, n_steps)
        b += ((n_steps + K - 1) // K) * B * low.n_slots * itemsize
        b += K * B * (low.n_slots + low.n_nodes) * itemsize
        b += B * low.n_slots * itemsize + B * low.n_cols * 8 + (n_steps + 1) * B * max(low.n_rec, 1) * itemsize
    return int(b)


class _Active:
    """An admitted request: its device model and buffers."""

    def __init__(self, req: Request, server: "Server"):
        self.req = req
        dev, dtype = server.device, server.dtype
        self.low = lower(req.problem, max_block_nodes=server.max_block_nodes, keep_currents=False)
        self.model = DeviceModel(self.low, dtype, dev, 1, threads=server.threads,
                                 smem_limit=server.smem_limit)
        # all items of the request in one set for the multi-request launches
        low = self.low
        items = np.asarray([[b, r, 1, 0] for b in range(len(low.blocks)) for r in range(low.batch)],
                           dtype=np.int32)
        items = items[np.argsort(-low.blocks[items[:, 0], 1], kind="stable")]
        self.item_nodes = low.blocks[items[:, 0], 1].astype(np.int64)  # nodes of every item
        group = {"maxima": self.model._block_maxima(np.arange(len(low.blocks))),
                 "items": torch.as_tensor(items, device=dev).contiguous(), "n_items": len(items)}
        self.group_f = self.group_b = group
        m, low = self.model, self.low
        self.T = int(req.n_steps)
        if server.slice_us:
            # time slice: every request gets about the same GPU time per tick, so a
            # request of fast steps advances by more of them and short requests are
            # not held to the pace of long ones
            self.chunk = int(min(self.T, max(server.min_chunk,
                                             round(server.slice_us / step_cost_us(low, server.threads)))))
        elif server.progress_ticks:
            # equal progress: every request needs about `progress_ticks` ticks (a gradient
            # request half of them forward, half adjoint), whatever its horizon
            n = max(1, server.progress_ticks // (2 if req.grad else 1))
            self.chunk = max(server.min_chunk, -(-self.T // n))
        else:
            self.chunk = server.chunk
        self.K = min(self.chunk if (server.progress_ticks or server.slice_us) else server.checkpoint, self.T)
        self.nseg = (self.T + self.K - 1) // self.K
        self.state = m.initial_state()
        self.rec = torch.zeros((self.T + 1, low.batch, low.n_rec), dtype=dtype, device=dev)
        self.pscale = m.pscale
        self.t = 0
        self.phase = "fwd"
        self.bytes = request_bytes(low, self.T, req.grad, server.checkpoint,
                                   torch.empty((), dtype=dtype).element_size())
        self.gm = {k: m._layout_bytes(g["maxima"], k == "backward") > server.smem_limit
                   for k, g in (("forward", self.group_f), ("backward", self.group_b))}
        if req.grad:
            self.ckpt = torch.empty((self.nseg, low.batch, low.n_slots), dtype=dtype, device=dev)
            self.traj = torch.empty((self.K, low.batch, low.n_slots), dtype=dtype, device=dev)
            self.piv = torch.empty((self.K, low.batch, low.n_nodes), dtype=dtype, device=dev)
            self.adj = torch.zeros((low.batch, low.n_slots), dtype=dtype, device=dev)
            self.pgrad = torch.zeros((low.batch, low.n_cols), dtype=torch.float64, device=dev)
            self.rec_grad = torch.ones((self.T + 1, low.batch, low.n_rec), dtype=dtype, device=dev)
            self.seg = self.nseg - 1
        # initial currents (and the first recording)
        a = m.args(self.state, 0, 0, self.rec, mode=1, pscale=self.pscale)
        m.launch_forward(a)
        # argument templates: a tick only sets the time window (and the checkpoint)
        self.base_f = self._items(m.args(self.state, 1, 0, self.rec, pscale=self.pscale,
                                         ckpt=self.ckpt if req.grad else None,
                                         ckpt_every=self.K if req.grad else 0), self.group_f)
        if req.grad:
            b = m.args(self.ckpt[0], 1, 0, None, pscale=self.pscale, traj=self.traj, adj=self.adj,
                       rec_grad=self.rec_grad, pgrad=self.pgrad)
            b.traj_piv = self.piv.data_ptr()
            self.base_b = self._items(b, self.group_b)
            self.ckpt_ptr0 = self.ckpt.data_ptr()
            self.ckpt_stride = self.ckpt[0].numel() * self.ckpt.element_size()
        self.sizes = {k: np.asarray([int(getattr(self.base_f, f)) for f in _SIZE_FIELDS], dtype=np.int64)
                      for k in ("forward", "backward")}

    def forward_args(self) -> Tuple[_lib.JxbSimArgs, int]:
        k = min(self.chunk, self.T - self.t)
        a = _lib.JxbSimArgs.from_buffer_copy(self.base_f)
        a.n_steps = k
        a.t0 = self.t
        return a, k

    def backward_args(self) -> _lib.JxbSimArgs:
        t0 = self.seg * self.K
        a = _lib.JxbSimArgs.from_buffer_copy(self.base_b)
        a.n_steps = min(self.K, self.T - t0)
        a.t0 = t0
        a.ckpt = self.ckpt_ptr0 + self.seg * self.ckpt_stride
        return a

    @staticmethod
    def _items(a: _lib.JxbSimArgs, group) -> _lib.JxbSimArgs:
        # the request's own items and block sizes (launch-level buffers are the server's)
        for k, v in group["maxima"].items():
            setattr(a, k, v)
        a.items = group["items"].data_ptr()
        a.n_items = group["n_items"]
        return a

    def finish(self) -> None:
        r = self.req
        r.recordings = self.rec.permute(1, 2, 0).cpu().numpy()
        if r.grad:
            r.gradient = self.pgrad.cpu().numpy()


_SIZE_FIELDS = ("max_rows", "max_nodes", "max_slots", "max_chains", "max_child", "max_levels",
                "max_pslots", "max_gslots", "n_entries", "n_classes")


def launch_sizes(args: Sequence[_lib.JxbSimArgs]) -> Dict[str, int]:
    """Work-area sizing of a multi-request launch: the maxima over its requests."""
    return {f: max([int(getattr(a, f)) for a in args] + [1]) for f in _SIZE_FIELDS}


def _stacked_sizes(sizes: Sequence[np.ndarray]) -> Dict[str, int]:
    mx = np.max(np.stack(sizes), axis=0) if len(sizes) else np.ones(len(_SIZE_FIELDS), np.int64)
    return {f: max(1, int(v)) for f, v in zip(_SIZE_FIELDS, mx)}


def pair_list(item_nodes: Sequence[np.ndarray]) -> np.ndarray:
    """(request, item) of every CTA of a multi-request launch, items of more nodes
    first (CTAs are scheduled roughly in index order). `item_nodes[r]` holds the node
    count of every item of request r."""
    req = np.concatenate([np.full(len(n), r, dtype=np.int64) for r, n in enumerate(item_nodes)] or [np.zeros(0, np.int64)])
    itm = np.concatenate([np.arange(len(n)) for n in item_nodes] or [np.zeros(0, np.int64)])
    size = np.concatenate(list(item_nodes) or [np.zeros(0, np.int64)])
    order = np.argsort(-size, kind="stable")
    return np.ascontiguousarray(np.stack([req[order], itm[order]], axis=1).astype(np.int32))


class Server:
    """Continuous batching of requests on one GPU (see the module docstring)."""

    def __init__(self, device="cuda", dtype=torch.float32, hbm_budget: Optional[int] = None,
                 chunk: int = 200, threads: int = 256, checkpoint: int = 100,
                 max_block_nodes: int = 4096, max_active: int = 4096, progress_ticks: int = 0,
                 min_chunk: int = 20, slice_ms: float = 0.0):
        self.device = torch.device(device)
        self.dtype = dtype
        self.code = _lib.F32 if dtype == torch.float32 else _lib.F64
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            hbm_budget = int(free * 0.5)
        self.hbm_budget = int(hbm_budget)
        self.chunk = int(chunk)
        # Scheduling policy: with `slice_ms`, every request advances per tick by the
        # steps that take about `slice_ms` of GPU time (step_cost_us); else with
        # `progress_ticks`, by 1 / progress_ticks of its horizon; else by `chunk` steps.
        self.slice_us = float(slice_ms) * 1e3
        self.progress_ticks = int(progress_ticks)
        self.min_chunk = int(min_chunk)
        self.threads = int(threads)
        self.checkpoint = int(checkpoint)
        self.max_block_nodes = int(max_block_nodes)
        self.max_active = int(max_active)
        props = torch.cuda.get_device_properties(self.device)
        self.smem_limit = int(getattr(props, "shared_memory_per_block_optin", 0) or 227 * 1024)
        self.queue: List[Request] = []
        self.active: List[_Active] = []
        self.done: List[Request] = []
        self.used = 0
        self.streams = [torch.cuda.Stream(self.device) for _ in range(4)]
        self._bufs: Dict[str, torch.Tensor] = {}
        self.ticks = 0
        self.launches = 0
        self.comp_steps = 0
        self._t0 = None

    # ---- host-side bookkeeping ----
    def clock(self) -> float:
        return time.perf_counter() - self._t0

    def submit(self, req: Request) -> None:
        self.queue.append(req)

    def _admit(self) -> None:
        now = self.clock()
        while self.queue and self.queue[0].arrival <= now and len(self.active) < self.max_active:
            req = self.queue[0]
            est = request_bytes_estimate(req, self.checkpoint)
            if self.used + est > self.hbm_budget and self.active:
                break  # wait until running requests free memory
            self.queue.pop(0)
            act = _Active(req, self)
            act.bytes = max(act.bytes, est)
            self.used += act.bytes
            req.admitted = self.clock()
            self.active.append(act)

    def _buf(self, key: str, nbytes: int) -> torch.Tensor:
        b = self._bufs.get(key)
        if b is None or b.numel() < nbytes:
            b = torch.empty(max(nbytes, 1 << 20), dtype=torch.uint8, device=self.device)
            self._bufs[key] = b
        return b

    def _launch(self, kind: str, gm: bool, acts: List[_Active], args: List[_lib.JxbSimArgs], stream) -> None:
        if not args:
            return
        lib = _lib.load()
        L = _lib.JxbSimArgs()
        L.dtype = self.code
        L.threads = self.threads
        for f, v in _stacked_sizes([act.sizes[kind] for act in acts]).items():
            setattr(L, f, v)
        pairs = pair_list([act.item_nodes for act in acts])
        n = len(pairs)
        if gm:
            stride = (int(lib.jxb_sim_smem_bytes(C.byref(L), int(kind == "backward"))) + 255) // 256 * 256
            buf = self._buf(f"work_{kind}", n * stride + 256)
            L.gscratch = (buf.data_ptr() + 255) // 256 * 256
            L.gscratch_stride = stride
        if kind == "backward":
            gstride = (L.max_rows * L.max_gslots * (4 if self.code == _lib.F32 else 8) + 255) // 256 * 256
            buf = self._buf(f"gacc_{gm}", n * gstride + 256)
            L.gacc = (buf.data_ptr() + 255) // 256 * 256
            L.gacc_stride = gstride
        need = int(lib.jxb_sim_multi_scratch_bytes(len(args), n))
        sc = self._buf(f"multi_{kind}_{gm}", need + 256)
        arr = (_lib.JxbSimArgs * len(args))(*args)
        fn = lib.jxb_sim_backward_multi if kind == "backward" else lib.jxb_sim_forward_multi
        with torch.cuda.stream(stream):
            rc = fn(C.byref(L), arr, len(args), pairs.ctypes.data, n,
                    C.c_void_p((sc.data_ptr() + 255) // 256 * 256), need, C.c_void_p(stream.cuda_stream))
        _lib.check(rc, f"jxb_sim_{kind}_multi")
        self.launches += 1

    def tick(self) -> None:
        """Admit arrivals, advance every active request by one chunk (forward) or one
        segment (adjoint), retire the finished ones."""
        self._admit()
        if not self.active:
            return
        main = torch.cuda.current_stream(self.device)
        for s in self.streams:
            s.wait_stream(main)  # initial-current launches of the newly admitted
        groups: Dict[Tuple[str, bool], Tuple[List[_Active], List]] = {}
        steps: Dict[int, int] = {}
        for act in self.active:
            if act.phase == "fwd":
                a, k = act.forward_args()
                steps[id(act)] = k
                key = ("forward", act.gm["forward"])
            else:
                a = act.backward_args()
                key = ("backward", act.gm["backward"])
            acts, args = groups.setdefault(key, ([], []))
            acts.append(act)
            args.append(a)
        for q, (key, (acts, args)) in enumerate(sorted(groups.items())):
            self._launch(key[0], key[1], acts, args, self.streams[q])
        for s in self.streams:
            s.synchronize()
        self.ticks += 1
        keep = []
        for act in self.active:
            if act.phase == "fwd":
                k = steps[id(act)]
                act.t += k
                self.comp_steps += k * len(act.req.problem.comp_inds) * act.low.batch
                if act.t >= act.T:
                    act.phase = "bwd" if act.req.grad else "done"
            else:
                act.seg -= 1
                if act.seg < 0:
                    act.phase = "done"
            if act.phase == "done":
                act.finish()
                act.req.finished = self.clock()
                self.done.append(act.req)
                self.used -= act.bytes
            else:
                keep.append(act)
        self.active = keep

    def run(self, requests: Sequence[Request], time_limit: float = 600.0) -> Dict[str, float]:
        """Serves `requests` (arrival times in seconds from now) to completion and
        returns latency and throughput statistics."""
        self.queue = sorted(requests, key=lambda r: r.arrival)
        for i, r in enumerate(self.queue):
            if r.rid < 0:
                r.rid = i
        self.done = []
        self.comp_steps = 0
        torch.cuda.synchronize(self.device)
        self._t0 = time.perf_counter()
        while (self.queue or self.active) and self.clock() < time_limit:
            if not self.active and self.queue and self.queue[0].arrival > self.clock():
                time.sleep(min(0.001, self.queue[0].arrival - self.clock()))
                continue
            self.tick()
        makespan = self.clock()
        return summarize(self.done, makespan, self.comp_steps, ticks=self.ticks, launches=self.launches)


def request_bytes_estimate(req: Request, checkpoint: int) -> int:
    """Admission estimate from the problem's sizes (before lowering)."""
    p = req.problem
    n, B = p.n_nodes, p.batch
    slots = n * 8
    b = n * 80 + B * slots * 4 + (req.n_steps + 1) * B * max(len(p.recordings), 1) * 4
    if req.grad:
        K = min(checkpoint, req.n_steps)
        b += ((req.n_steps + K - 1) // K) * B * slots * 4 + K * B * (slots + n) * 4 + 2 * B * slots * 4
        b += (req.n_steps + 1) * B * max(len(p.recordings), 1) * 4
    return int(b)


def summarize(done: Sequence[Request], makespan: float, comp_steps: int, **extra) -> Dict[str, float]:
    lat = np.asarray([r.latency for r in done]) if done else np.zeros(1)
    out = {"requests": len(done), "makespan_s": makespan,
           "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
           "mean_ms": float(lat.mean() * 1e3), "compartment_steps": int(comp_steps),
           "throughput": comp_steps / makespan if makespan > 0 else 0.0}
    out["p99_over_p50"] = out["p99_ms"] / out["p50_ms"] if out["p50_ms"] > 0 else float("nan")
    slow = np.asarray([r.slowdown for r in done if np.isfinite(r.service) and r.service > 0])
    if len(slow):
        out["slowdown_p50"] = float(np.percentile(slow, 50))
        out["slowdown_p99"] = float(np.percentile(slow, 99))
    out.update(extra)
    return out


def fifo_latencies(arrivals: Sequence[float], service: Sequence[float]) -> np.ndarray:
    """Latencies of one server that takes requests one at a time in arrival order
    (the per-request path), from their arrival and service times."""
    done, out = 0.0, []
    for a, s in sorted(zip(arrivals, service)):
        done = max(done, a) + s
        out.append(done - a)
    return np.asarray(out)


def serve_plain(requests: Sequence[Request], device="cuda", dtype=torch.float32, threads: int = 256,
                checkpoint: int = 100, time_limit: float = 600.0) -> Dict[str, float]:
    """The per-request path on the same kernels: requests in arrival order, one at a
    time, each with its own persistent forward launch and adjoint launches."""
    queue = sorted(requests, key=lambda r: r.arrival)
    done, comp_steps = [], 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for r in queue:
        now = time.perf_counter() - t0
        if now > time_limit:
            break
        if r.arrival > now:
            time.sleep(r.arrival - now)
        sim = Simulation(r.problem, dtype=dtype, device=device, threads=threads,
                         checkpoint=min(checkpoint, r.n_steps), keep_currents=False)
        if r.grad:
            ps = sim.model.pscale.clone().requires_grad_(True)
            rec = sim.run(n_steps=r.n_steps, pscale=ps)
            (g,) = torch.autograd.grad(rec.sum(), ps)
            r.gradient = g.detach().cpu().numpy()
        else:
            with torch.no_grad():
                rec = sim.run(n_steps=r.n_steps)
        r.recordings = rec.detach().cpu().numpy()
        r.finished = time.perf_counter() - t0
        r.service = r.finished - max(now, r.arrival)
        comp_steps += r.n_steps * len(r.problem.comp_inds) * r.problem.batch
        done.append(r)
    return summarize(done, time.perf_counter() - t0, comp_steps)


def make_stream(n: int, seed: int = 0, rate: float = 100.0, grad_fraction: float = 0.3,
                min_comp: int = 8, max_comp: int = 3000, t_range=(5.0, 200.0), dt: float = 0.025):
    """Seeded request stream: one cell per request from the uneven-batch generator
    (log-uniform min_comp..max_comp compartments), horizon U[t_range] ms, a gradient
    for `grad_fraction` of them, Poisson arrivals at `rate` per second."""
    from . import synth

    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=n)
    arrivals = np.cumsum(gaps) - gaps[0]
    reqs = []
    for i in range(n):
        T = int(round(rng.uniform(*t_range) / dt))
        prob = synth.config_uneven(n_cells=1, seed=int(rng.integers(1 << 30)), n_steps=T,
                                   min_comp=min_comp, max_comp=max_comp)
        reqs.append(Request(problem=prob, n_steps=T, grad=bool(rng.random() < grad_fraction),
                            arrival=float(arrivals[i]), rid=i))
    return reqs
