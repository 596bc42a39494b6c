"""Autotuner of the fused simulation launch.

The choices: nodes per block (how trees are packed into CTAs: `max_block_nodes`),
threads per CTA (warps per block of trees), batch rows per work item, and the
checkpoint interval of the adjoint (steps recomputed per backward launch, traded
against the memory of the stored states and trajectories). Each candidate is timed
on a short horizon of the actual problem with CUDA events (forward + adjoint when
`grad`, forward only otherwise), each timed run separately after a warm-up run, the
shortest run counting (a run that host work or another process slowed down does not
decide); the fastest candidate wins. `sim_kwargs` (for example the forward's own
launch shape) go to every probe `Simulation`, so that a probe runs what the tuned run
will. Candidates that the launcher rejects (sizes) or that exceed the memory budget
are skipped. Results are cached per problem signature in-process and, with
`cache_path`, in a JSON file.
"""
from __future__ import annotations

import hashlib
import json
import os
from dataclasses import asdict, dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np
import torch

from .lower import Lowered, lower
from .problem import Problem
from .sim import Simulation


@dataclass
class Choice:
    max_block_nodes: int
    threads: int
    rows_per_item: int
    checkpoint: int
    ms_per_step: float  # fwd (+ adjoint) per simulated step of the probe horizon


_CACHE: Dict[str, Choice] = {}


def signature(problem: Problem, dtype: torch.dtype, grad: bool) -> str:
    """Shape of the problem that the launch choices depend on."""
    parent, _, _ = problem.solve_order_system()
    h = hashlib.sha1()
    h.update(np.asarray(parent, dtype=np.int64).tobytes())
    for ch in problem.channels:
        h.update(ch.type_name.encode())
        h.update(np.asarray(ch.inds, dtype=np.int64).tobytes())
    h.update(f"{problem.batch}|{dtype}|{grad}".encode())
    return h.hexdigest()


def run_bytes(low: Lowered, itemsize: int, T: int, K: int, grad: bool) -> int:
    """Device memory of one run: state, recordings, and for the adjoint the stored
    states (one per K steps), the trajectory and pivots of one segment, the adjoint."""
    B = low.batch
    b = B * low.n_slots * itemsize * 2 + (T + 1) * B * max(low.n_rec, 1) * itemsize * 2
    if grad:
        b += ((T + K - 1) // K) * B * low.n_slots * itemsize
        b += min(K, T) * B * (low.n_slots + low.n_nodes) * itemsize
        b += B * low.n_slots * itemsize + B * low.n_cols * 8
    return int(b)


def _time(sim: Simulation, T: int, grad: bool, reps: int) -> float:
    ps0 = sim.model.pscale

    def once():
        if grad:
            ps = ps0.clone().requires_grad_(True)
            rec = sim.run(n_steps=T, pscale=ps)
            torch.autograd.grad(rec.square().mean(), ps)
        else:
            with torch.no_grad():
                sim.run(n_steps=T, pscale=ps0)

    once()
    torch.cuda.synchronize(sim.model.device)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    best = float("inf")
    for _ in range(max(1, reps)):
        e0.record()
        once()
        e1.record()
        torch.cuda.synchronize(sim.model.device)
        best = min(best, e0.elapsed_time(e1))
    return best / T


def autotune(problem: Problem, dtype: torch.dtype = torch.float32, device="cuda", grad: bool = True,
             probe_steps: int = 40, block_nodes: Sequence[int] = (1024, 2048, 4096),
             threads: Sequence[int] = (256, 512), rows: Sequence[int] = (1, 2, 4),
             checkpoints: Sequence[int] = (50, 100, 200), horizon: Optional[int] = None,
             memory_budget: Optional[int] = None, keep_currents: bool = False,
             cache_path: Optional[str] = None, reps: int = 2,
             sim_kwargs: Optional[dict] = None,
             verbose: bool = False) -> Tuple[Choice, Lowered, List[dict]]:
    """Returns `(choice, lowered model of the chosen block size, table of timings)`."""
    key = signature(problem, dtype, grad)
    if sim_kwargs:  # a choice holds for the launch options it was timed with
        key += "|" + json.dumps(sim_kwargs, sort_keys=True, default=str)
    table: List[dict] = []
    cached = _CACHE.get(key)
    if cached is None and cache_path and os.path.exists(cache_path):
        with open(cache_path) as f:
            d = json.load(f).get(key)
        if d:
            cached = Choice(**d)
    if cached is not None:
        return cached, lower(problem, max_block_nodes=cached.max_block_nodes,
                             keep_currents=keep_currents), table
    T_full = int(horizon if horizon is not None else problem.n_steps)
    itemsize = torch.empty((), dtype=dtype).element_size()
    if memory_budget is None and torch.cuda.is_available():
        free, _ = torch.cuda.mem_get_info(torch.device(device))
        memory_budget = int(free * 0.8)
    lows: Dict[int, Lowered] = {}
    best: Optional[Tuple[float, int, int, int]] = None
    B = problem.batch
    Kp = min(probe_steps, T_full)
    for mbn in block_nodes:
        lows[mbn] = low = lower(problem, max_block_nodes=mbn, keep_currents=keep_currents)
        for th in threads:
            for r in sorted({min(r, B) for r in rows}):
                try:
                    sim = Simulation(problem, low=low, dtype=dtype, device=device, threads=th,
                                     rows_per_item=r, checkpoint=Kp, **(sim_kwargs or {}))
                    ms = _time(sim, Kp, grad, reps)
                except RuntimeError as e:  # sizes the launcher rejects
                    table.append({"max_block_nodes": mbn, "threads": th, "rows": r, "error": str(e)})
                    continue
                table.append({"max_block_nodes": mbn, "threads": th, "rows": r, "ms_per_step": ms})
                if verbose:
                    print("tune", table[-1], flush=True)
                if best is None or ms < best[0]:
                    best = (ms, mbn, th, r)
                del sim
    if best is None:
        raise RuntimeError("no launch configuration ran: " + json.dumps(table))
    ms, mbn, th, r = best
    low = lows[mbn]
    K_best, ms_best = Kp, ms
    if grad:
        Tk = min(T_full, 2 * max(checkpoints))
        cands = [K for K in checkpoints if K <= Tk
                 and (memory_budget is None or run_bytes(low, itemsize, T_full, K, True) <= memory_budget)]
        timed = []
        for K in cands:
            sim = Simulation(problem, low=low, dtype=dtype, device=device, threads=th, rows_per_item=r,
                             checkpoint=K, **(sim_kwargs or {}))
            msk = _time(sim, Tk, True, reps)
            table.append({"checkpoint": K, "horizon": Tk, "ms_per_step": msk})
            if verbose:
                print("tune", table[-1], flush=True)
            timed.append((msk, K))
            del sim
        if timed:
            ms_best, K_best = min(timed)
    choice = Choice(mbn, th, r, K_best, ms_best)
    _CACHE[key] = choice
    if cache_path:
        d = {}
        if os.path.exists(cache_path):
            with open(cache_path) as f:
                d = json.load(f)
        d[key] = asdict(choice)
        with open(cache_path, "w") as f:
            json.dump(d, f, indent=1)
    return choice, low, table
