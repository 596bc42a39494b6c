#!/usr/bin/env python
"""Benchmark of the per-timestep hot path: compartment-steps/s, forward + adjoint.

Workload (per GPU): the synthetic L5PC-like tree (300 branches x 4 compartments, 1200
compartments + branchpoints, near-balanced, height 35-45), 256 parameter sets with
every conductance scaled by U[0.5, 1.5], float32, dt = 0.025 ms, 4000 steps; one
bench step = the simulation of all 256 rows, the MSE to a seeded target trace and its
gradient with respect to the 256 x 10 conductance scales through the adjoint (the
forward stores the trajectory, 36 GB, and the adjoint sweeps it back in launches of
100 steps; `recompute` in the line is the same iteration with a checkpoint every 100
steps recomputed in the adjoint). Compartment-steps count compartments x rows x steps
(branchpoints excluded, every simulated step once).

The same JSON line carries `uneven`: the uneven batch of 4096 seeded cells
(log-uniform 4-3000 compartments, depth 1-60, HH or L5PC, 2000 steps, forward +
adjoint), persistent (autotuned launches, whole iteration in one CUDA graph) against
the plain per-step form (one launch per step and adjoint step), in compartment-steps/s.

`network`: a training step (simulation, MSE, adjoint, capturable Adam on the synaptic
weights, one CUDA graph) of 2048 4-compartment HH cells with in-degree 64 of two
synapse types, 32 rows of Poisson input, 2000 steps; and `serving`: a Poisson stream of single-cell simulation and gradient requests
(8-3000 compartments, 5-200 ms, 30 % gradients) at 80 % of the server's measured
capacity, served with continuous batching: p50/p99 latency and throughput, beside the
plain one-request-at-a-time path on the same arrivals.

`--impl reference` times the reference's own torch path (its `jx.integrate` from the
copy installed under `baseline/_ref`, eager autograd, float32) on the host cores, on a
bounded sample of the same workload (the CPU port of that path when the reference is
not installed); `cpu_baseline` in the line is the same measurement, with the forward
alone beside it.

Multi-GPU (torchrun): every rank simulates its own 256 parameter sets (weak scaling,
no collective in the data path); the timing is the maximum over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from datetime import timedelta

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "compartment-steps/s fwd+bwd on 1 B200 vs plain kernels; p50/p99 request latency"
UNIT = "compartment-steps/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=256)
    ap.add_argument("--tsteps", type=int, default=4000)
    ap.add_argument("--checkpoint", type=int, default=100)
    ap.add_argument("--threads", type=int, default=512)
    ap.add_argument("--forward-threads", type=int, default=256,
                    help="CTA size of the forward launches (wide register budget up to 256)")
    ap.add_argument("--rows", type=int, default=1)
    ap.add_argument("--cpu-batch", type=int, default=16)
    ap.add_argument("--cpu-tsteps", type=int, default=200)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-uneven", action="store_true",
                    help="skip the uneven-batch persistent vs per-step measurement")
    ap.add_argument("--uneven-cells", type=int, default=4096)
    ap.add_argument("--uneven-tsteps", type=int, default=2000)
    ap.add_argument("--uneven-plain-tsteps", type=int, default=2000)
    ap.add_argument("--no-serving", action="store_true", help="skip the serving-stream measurement")
    ap.add_argument("--no-network", action="store_true", help="skip the network training-step measurement")
    ap.add_argument("--no-recompute", action="store_true",
                    help="skip the checkpoint/recompute comparison of the main iteration")
    ap.add_argument("--net-tsteps", type=int, default=2000)
    ap.add_argument("--no-lm", action="store_true",
                    help="skip the language-model network shape (1024 and 2048 HH neurons x 100 synapses)")
    ap.add_argument("--lm-tokens", type=int, default=10, help="tokens of 200 solver steps per training step")
    ap.add_argument("--no-fp32-error", action="store_true",
                    help="skip the float32-against-float64 error of the sampled configurations")
    ap.add_argument("--no-kernel-compare", action="store_true",
                    help="skip the standalone drop-in ops against the reference's Triton kernels")
    ap.add_argument("--kernel-compare-only", action="store_true",
                    help="print only the drop-in comparison as JSON (run as a child of the bench)")
    ap.add_argument("--local-device", type=int, default=0, help=argparse.SUPPRESS)
    ap.add_argument("--serve-requests", type=int, default=240)
    ap.add_argument("--serve-capacity-requests", type=int, default=160)
    return ap.parse_args()


class ClockSampler:
    """Samples SM clocks and throttle reasons with nvidia-smi during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_hbm():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def traffic_from_profiles(kernel: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if any."""
    path = os.path.join(REPO, "profiles", "dram_traffic.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d.get(kernel)
    return None


def max_over_ranks(x: float, world: int, device) -> float:
    """The largest of every rank's `x` (the timing of a multi-GPU run is its slowest rank)."""
    if world == 1:
        return x
    import torch

    t = torch.tensor([x], device=device, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def workload(rank: int, batch: int, tsteps: int):
    from jaxley_pytorch_b200 import synth

    prob = synth.config_l5pc_tree(batch=batch, n_steps=tsteps, seed=0, scale_seed=1 + rank)
    held_out = synth.config_l5pc_tree(batch=1, n_steps=tsteps, seed=0, scale_seed=10_000)
    return prob, held_out


def algorithmic_bytes(low, itemsize: int, stored: bool):
    """Per compartment-step, in units of s = itemsize: S = state slots per
    compartment, P = batch-varying parameters per compartment (conductances),
    N = tree nodes per compartment (one reciprocal pivot each). Forward: state read
    and write and the parameters, s(2S+P), plus with a stored trajectory the state
    and pivot of every step, s(3S+P+N). Adjoint launch: with a stored trajectory,
    trajectory and pivot read, adjoint state read and write, parameters, s(3S+P+N);
    with recompute, the forward's traffic, the trajectory and pivot write, then the
    reverse pass, s(6S+2P+2N)."""
    comps = [i for i in range(low.n_nodes) if low.cls_comp[low.node_class[i]]]
    S = float(np.mean([low.soff[i + 1] - low.soff[i] for i in comps]))
    cls_np = {}
    P_list = []
    for i in comps:
        po = low.poff[i]
        cls = low.node_class[i]
        n_par = 0
        for e in low.entries[low.cls_ptr[cls]:low.cls_ptr[cls + 1]]:
            n_par += int(e[2])
        P_list.append(int(np.count_nonzero(low.pcol[po:po + n_par])))
    P = float(np.mean(P_list))
    N = low.n_nodes / len(comps)
    if stored:
        return S, P, itemsize * (3 * S + P + N), itemsize * (3 * S + P + N)
    return S, P, itemsize * (2 * S + P), itemsize * (6 * S + 2 * P + 2 * N)


def run_ours(args, rank, world, device):
    import torch

    from jaxley_pytorch_b200.sim import Simulation

    torch.cuda.set_device(device)
    prob, held = workload(rank, args.batch, args.tsteps)
    T = prob.n_steps
    kw = dict(dtype=torch.float32, device=device, checkpoint=args.checkpoint, init_steady=True,
              keep_currents=False, threads=args.threads, rows_per_item=args.rows,
              forward_threads=args.forward_threads, forward_wide=args.forward_threads <= 256)
    sim = Simulation(prob, **kw)
    tsim = Simulation(held, **kw)
    with torch.no_grad():
        target = tsim.run()[0, 0].detach()
    low = sim.low
    n_comp = int(len(prob.comp_inds))
    B = low.batch
    ps0 = sim.model.pscale.clone()

    def train_step(ps):
        rec = sim.run(pscale=ps)
        loss = ((rec[:, 0, :] - target) ** 2).mean()
        (g,) = torch.autograd.grad(loss, ps)
        return loss, g

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    def loss_fn(rec):
        return ((rec[:, 0, :] - target) ** 2).mean()

    # The iteration (forward launches, loss, adjoint launches) captured once as a CUDA
    # graph after W eager warm-up iterations, and replayed: no host work per launch.
    from jaxley_pytorch_b200.graphs import GraphedIteration

    git = GraphedIteration(sim, loss_fn, ps0.clone().requires_grad_(True), warmup=args.warmup)
    git.replay()
    torch.cuda.synchronize()
    # Timed region: device timing with CUDA events; inputs resident in HBM.
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(torch.cuda.current_device()) as clocks:
        e0.record()
        for _ in range(args.steps):
            loss, g = git.replay()
        e1.record()
        torch.cuda.synchronize()
    barrier()
    launches = git.launches_per_replay * args.steps
    ms = max_over_ranks(e0.elapsed_time(e1), world, device)
    loss = loss.clone()
    del git
    torch.cuda.empty_cache()
    # Launch durations of each kind (extra eager passes, outside the timed region).
    ps = ps0.clone().requires_grad_(True)
    sim.model.events = []
    sim.model.timed_kind = "backward"
    train_step(ps)
    torch.cuda.synchronize()
    bwd = [(a.elapsed_time(b), k) for a, b, k in sim.model.events]
    sim.model.events = []
    sim.model.timed_kind = "forward"
    train_step(ps)
    torch.cuda.synchronize()
    fwd = [(a.elapsed_time(b), k) for a, b, k in sim.model.events if k > 0]
    sim.model.timed_kind = None

    comp_steps = n_comp * B * T * args.steps * world
    value = comp_steps / (ms / 1e3)

    # End to end through the public API: pinned host inputs in, loss and gradient out.
    ps_host = ps0.detach().cpu().pin_memory()
    loss_host = torch.empty((), dtype=torch.float32).pin_memory()
    g_host = torch.empty_like(ps_host).pin_memory()
    barrier()
    torch.cuda.synchronize()
    f0 = torch.cuda.Event(enable_timing=True)
    f1 = torch.cuda.Event(enable_timing=True)
    f0.record()
    for _ in range(args.steps):
        psd = ps_host.to(device, non_blocking=True).requires_grad_(True)
        loss, g = train_step(psd)
        loss_host.copy_(loss.detach(), non_blocking=True)
        g_host.copy_(g, non_blocking=True)
    f1.record()
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(f0.elapsed_time(f1), world, device)
    e2e = {"value": comp_steps / (e2e_ms / 1e3), "unit": UNIT,
           "h2d_bytes_per_step": int(ps_host.numel() * ps_host.element_size()),
           "d2h_bytes_per_step": int(loss_host.element_size() + g_host.numel() * g_host.element_size())}

    stored = sim.stores_trajectory(T)
    stored_mode = ("reverse sweep over the trajectory stored by the forward" if stored
                   else "recompute of each segment from its checkpoint")
    S, P, fwd_b, bwd_b = algorithmic_bytes(low, 4, stored)
    peak, peak_kind = measured_peak_hbm()
    bwd_ms = float(np.mean([t for t, _ in bwd])) if bwd else None
    fwd_ms = float(np.mean([t for t, _ in fwd])) if fwd else None
    bwd_total = sum(t for t, _ in bwd)  # one iteration each
    fwd_total = sum(t for t, _ in fwd)
    if bwd_total >= fwd_total and bwd:
        kern, k_steps, dur, per = "sim_backward_kernel", bwd[0][1], bwd_ms, bwd_b
    else:
        kern, k_steps, dur, per = "sim_forward_kernel", fwd[0][1], fwd_ms, fwd_b
    bytes_launch = per * n_comp * B * k_steps
    achieved = bytes_launch / (dur / 1e3) / 1e9
    traffic = traffic_from_profiles(kern)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "traffic": traffic, "kernel": kern,
                "peak_source": peak_kind, "avg_launch_ms": dur,
                "algorithmic_bytes_per_comp_step": per, "state_slots_per_comp": S,
                "batched_params_per_comp": P, "fwd_launch_ms": fwd_ms, "bwd_launch_ms": bwd_ms}
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "l5pc_tree_300x4_b256_t4000_fwd_adjoint", "compartments": n_comp,
                   "nodes": prob.n_nodes, "tree_height": prob.meta["height"], "batch": B,
                   "time_steps": T, "checkpoint": args.checkpoint,
                   "threads_per_cta": args.threads, "forward_threads_per_cta": args.forward_threads,
                   "rows_per_cta": args.rows,
                   "adjoint": stored_mode,
                   "l2": "working set larger than L2 (%s %d MB)" % (
                       ("stored trajectory", sim.trajectory_bytes(T) // 2**20) if stored
                       else ("trajectory buffer", args.checkpoint * B * low.n_slots * 4 // 2**20)),
                   "loss": "MSE of the somatic voltage to a held-out parameter set's trace"},
        "roofline": roofline, "e2e": e2e, "gpu_launches": int(launches),
        "clocks": clocks.summary(), "loss": float(loss.detach()),
    }
    if stored and not args.no_recompute:
        # The same iteration with the checkpoint/recompute adjoint (a checkpoint every
        # `checkpoint` steps, each segment recomputed in its adjoint launch).
        del sim
        rsim = Simulation(prob, store_trajectory=False, **kw)

        def recompute_step(ps):
            rec = rsim.run(pscale=ps)
            loss = ((rec[:, 0, :] - target) ** 2).mean()
            return torch.autograd.grad(loss, ps)[0]

        for _ in range(2):
            recompute_step(ps)
        barrier()
        torch.cuda.synchronize()
        r0 = torch.cuda.Event(enable_timing=True)
        r1 = torch.cuda.Event(enable_timing=True)
        r0.record()
        for _ in range(args.steps):
            recompute_step(ps)
        r1.record()
        torch.cuda.synchronize()
        rms = max_over_ranks(r0.elapsed_time(r1), world, device)
        out["recompute"] = {"value": comp_steps / (rms / 1e3), "unit": UNIT,
                            "ms_per_step": rms / args.steps, "checkpoint": args.checkpoint}
    return out


def run_uneven(args, device):
    """Uneven batch: 4096 seeded cells (log-uniform 4-3000 compartments, depth 1-60,
    HH or L5PC, own step current and trainable conductances), float32, 2000 steps,
    forward + adjoint of an MSE loss. The persistent form (autotuned block size,
    threads and checkpoint interval; the whole iteration replayed as one CUDA graph)
    against the plain per-step form (one launch per step and per adjoint step,
    checkpoint every step) on the same cells and horizon; the time of every size group
    of the persistent form (shared-memory classes and global work areas)."""
    import torch

    from jaxley_pytorch_b200 import synth
    from jaxley_pytorch_b200.graphs import GraphedIteration
    from jaxley_pytorch_b200.sim import Simulation
    from jaxley_pytorch_b200.tune import autotune

    torch.cuda.empty_cache()
    T = args.uneven_tsteps
    prob = synth.config_uneven(n_cells=args.uneven_cells, n_steps=T)
    n_comp = int(len(prob.comp_inds))
    wide = dict(forward_threads=args.forward_threads, forward_wide=args.forward_threads <= 256)
    # the probes run the forward at its own launch shape, as the tuned run does, so
    # that `threads` decides the adjoint's CTA size only
    choice, low, table = autotune(prob, dtype=torch.float32, device=device, probe_steps=40,
                                  block_nodes=(1024, 2048), threads=(256, 512), rows=(1,),
                                  checkpoints=(50, 100, 200), horizon=T, reps=2,
                                  sim_kwargs=dict(wide, store_fraction=0.6))

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    def loss_of(target):
        return lambda rec: ((rec - target) ** 2).mean()

    sim = Simulation(prob, low=low, dtype=torch.float32, device=device, threads=choice.threads,
                     rows_per_item=choice.rows_per_item, checkpoint=choice.checkpoint,
                     store_fraction=0.6, **wide)
    stored = sim.stores_trajectory(T)
    ps0 = sim.model.pscale.clone()
    with torch.no_grad():
        target = sim.run(pscale=ps0 * 1.05).detach()
    it = GraphedIteration(sim, loss_of(target), ps0.clone().requires_grad_(True), warmup=1)
    ms = timed(it.replay, 2)
    loss = float(it.loss)
    launches = it.launches_per_replay
    del it
    # the plain per-step form: one launch per step, checkpoint every step
    Tp = args.uneven_plain_tsteps
    torch.cuda.empty_cache()
    plain = Simulation(prob, low=low, dtype=torch.float32, device=device, threads=choice.threads,
                       rows_per_item=choice.rows_per_item, checkpoint=1, segment=1, **wide)
    with torch.no_grad():
        tp = plain.run(n_steps=Tp, pscale=ps0 * 1.05).detach()

    def plain_step():
        ps = ps0.clone().requires_grad_(True)
        rec = plain.run(n_steps=Tp, pscale=ps)
        torch.autograd.grad(((rec - tp) ** 2).mean(), ps)

    ms_plain_eager = timed(plain_step, 1)
    # The same per-step launches captured as one CUDA graph (no host work per launch).
    git = GraphedIteration(plain, loss_of(tp), ps0.clone().requires_grad_(True), n_steps=Tp, warmup=1)
    ms_plain = timed(git.replay, 2)
    plain_launches = git.launches_per_replay
    del git
    rate = n_comp * T / (ms / 1e3)
    rate_plain = n_comp * Tp / (ms_plain / 1e3)
    rate_plain_eager = n_comp * Tp / (ms_plain_eager / 1e3)
    del plain
    torch.cuda.empty_cache()
    # Per size group: one eager iteration of the persistent form with an event pair
    # around every group launch (the groups run concurrently on their own streams).
    sim.model.group_timing = True
    sim.model.group_events = []
    ps = ps0.clone().requires_grad_(True)
    torch.autograd.grad(loss_of(target)(sim.run(pscale=ps)), ps)
    torch.cuda.synchronize()
    sim.model.group_timing = False
    per_group = {}
    names = {-1: "global work areas", 0: "up to 1/4 of the shared memory", 1: "up to 1/2", 2: "up to all"}
    for kind, key, n_items, a, b in sim.model.group_events:
        ent = per_group.setdefault(f"{kind}/{names.get(key[1], key[1])}",
                                   {"items": n_items, "launches": 0, "ms": 0.0})
        ent["launches"] += 1
        ent["ms"] += a.elapsed_time(b)
    for g in sim.model.groups["forward"]:
        ent = per_group.get(f"forward/{names.get(g['key'][1], g['key'][1])}")
        if ent is not None:
            items = g["items"].cpu().numpy()
            ent["nodes_largest_block"] = int(sim.low.blocks[items[:, 0], 1].max())
    return {
        "workload": f"uneven_{args.uneven_cells}cells_t{T}_fwd_adjoint", "cells": args.uneven_cells,
        "compartments": n_comp, "nodes": prob.n_nodes, "time_steps": T,
        "persistent": {"value": rate, "unit": UNIT, "ms_per_iteration": ms, "graph_launches": launches,
                       "max_block_nodes": choice.max_block_nodes, "threads_per_cta": choice.threads,
                       "forward_threads_per_cta": args.forward_threads,
                       "checkpoint": choice.checkpoint, "loss": loss,
                       "adjoint": "stored trajectory (%d MB)" % (sim.trajectory_bytes(T) // 2**20) if stored
                       else "recompute from checkpoints"},
        "per_step": {"value": rate_plain, "unit": UNIT, "ms_per_iteration": ms_plain, "time_steps": Tp,
                     "checkpoint": 1, "graph_launches": plain_launches,
                     "form": "one forward launch per step and one adjoint launch per step, replayed as one "
                             "CUDA graph",
                     "eager": {"value": rate_plain_eager, "ms_per_iteration": ms_plain_eager}},
        "persistent_over_per_step": rate / rate_plain,
        "persistent_over_per_step_eager": rate / rate_plain_eager,
        "per_group": per_group,
        "tuning": table,
    }


def run_serving(args, device):
    """Serving stream: seeded single-cell requests from the uneven-batch generator
    (8-3000 compartments), horizons U[5, 200] ms, 30 % with gradients, float32.
    For each scheduling policy (time slice: every request advances per tick by the
    steps that take about 2 ms of GPU time; equal progress: by 1/16 of its work;
    fixed: by 200 steps) the capacity is measured on a closed batch (all requests
    waiting), then Poisson arrivals at 80 % of that capacity give p50/p99 latency,
    compartment-steps/s and every request's slowdown (latency over its latency when
    served alone, measured on the plain per-request path). The plain per-request path
    itself (one request at a time, same kernels) on the same arrivals is the FIFO
    queue of those alone latencies."""
    from jaxley_pytorch_b200.serve import Request, Server, fifo_latencies, make_stream, serve_plain

    def copy(reqs, zero=False):
        return [Request(problem=r.problem, n_steps=r.n_steps, grad=r.grad, arrival=0.0 if zero else r.arrival,
                        rid=r.rid) for r in reqs]

    policies = {"time_slice_2ms": dict(slice_ms=2.0, checkpoint=200, min_chunk=20),
                "equal_progress_16": dict(progress_ticks=16, chunk=200, checkpoint=200),
                "fixed_chunk_200": dict(progress_ticks=0, chunk=200, checkpoint=200)}
    Server(device=device, threads=256, **policies["fixed_chunk_200"]).run(make_stream(8, seed=99, rate=1e6))
    closed = make_stream(args.serve_requests // 3 * 2, seed=7, rate=1e9)
    base = make_stream(args.serve_requests, seed=8, rate=1.0)  # problems and horizons (rate-free)
    # alone latencies: every request on its own, one after the other
    alone = copy(base, zero=True)
    pl = serve_plain(alone, device=device, threads=256, checkpoint=200)
    service = {r.rid: r.service for r in alone}
    out = {"workload": "serving_stream_8_3000comp_5_200ms_30pct_grad", "unit": UNIT, "policies": {}}
    for name, pol in policies.items():
        cap = Server(device=device, threads=256, **pol).run(copy(closed, zero=True))
        capacity = cap["requests"] / cap["makespan_s"]
        stream = make_stream(args.serve_requests, seed=8, rate=0.8 * capacity)
        for r in stream:
            r.service = service[r.rid]
        st = Server(device=device, threads=256, **pol).run(stream)
        plain_lat = fifo_latencies([r.arrival for r in stream], [service[r.rid] for r in stream])
        out["policies"][name] = {
            "capacity_rps": capacity, "closed_batch_throughput": cap["throughput"],
            "arrival_rate_rps": 0.8 * capacity, "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
            "p99_over_p50": st["p99_over_p50"], "slowdown_p50": st.get("slowdown_p50"),
            "slowdown_p99": st.get("slowdown_p99"), "throughput": st["throughput"],
            "requests": st["requests"], "ticks": st["ticks"], "launches": st["launches"],
            "makespan_s": st["makespan_s"],
            "plain_per_request_same_arrivals": {"p50_ms": float(np.percentile(plain_lat, 50) * 1e3),
                                                "p99_ms": float(np.percentile(plain_lat, 99) * 1e3)}}
    first = out["policies"]["time_slice_2ms"]
    out.update({k: first[k] for k in ("p50_ms", "p99_ms", "p99_over_p50", "slowdown_p50", "slowdown_p99",
                                      "throughput", "capacity_rps", "arrival_rate_rps")})
    out["policy"] = "time_slice_2ms"
    out["plain_per_request"] = {"throughput": pl["throughput"], "alone_p50_ms": pl["p50_ms"],
                                "requests": pl["requests"], "wall_s": pl["makespan_s"]}
    out["throughput_over_plain"] = first["throughput"] / pl["throughput"] if pl["throughput"] else None
    return out


def run_network(args, device):
    """Fixed in-degree network: 2048 HH cells of 1 branch x 4 compartments, 64
    KineticSynapse and 64 SigmoidRateSynapse inputs on compartment 0 of every cell
    (131,072 synapses per type, gS ~ U[0, 1e-3] uS), 32 rows of Poisson input (20 Hz,
    0.2 nA one-step pulses), float32, 2000 steps. One training step = the simulation,
    the MSE of all somatic voltages to a target, the adjoint, and Adam
    (capturable) on the synaptic weights of both types, replayed as one CUDA graph."""
    import torch

    from jaxley_pytorch_b200.graphs import GraphedIteration
    from jaxley_pytorch_b200.network import NetworkSimulation, config_network

    T = args.net_tsteps
    prob = config_network(n_cells=2048, ncomp=4, k=64, batch=32, n_steps=T, seed=0)
    net = NetworkSimulation(prob, dtype=torch.float32, device=device, checkpoint=50, threads=256,
                            max_block_nodes=256)
    sizes = [ty.E for ty in net.types]
    with torch.no_grad():
        tgt_params = [[ty.params[0] * 1.2] + ty.params[1:] for ty in net.types]
        target = net.run(net.model.pscale, tgt_params).detach()

    def run(w):
        parts = torch.split(w, sizes)
        return net.run(net.model.pscale, [[parts[t]] + ty.params[1:] for t, ty in enumerate(net.types)])

    def loss_fn(rec):
        return ((rec - target) ** 2).mean()

    w = torch.cat([ty.params[0] for ty in net.types]).clone().requires_grad_(True)
    syn0 = net.syn_launches
    it = GraphedIteration(net, loss_fn, w, optimizer=torch.optim.Adam([w], lr=1e-6, capturable=True),
                          warmup=1, run=run)
    it.replay()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 2
    e0.record()
    for _ in range(reps):
        it.replay()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    n_comp = len(prob.comp_inds)
    return {"workload": f"network_2048x4_k64x2_b32_t{T}_train_step", "compartments": n_comp,
            "synapses": int(sum(sizes)), "batch": 32, "time_steps": T,
            "value": n_comp * 32 * T / (ms / 1e3), "unit": UNIT,
            "synapse_steps_per_s": sum(sizes) * 32 * T / (ms / 1e3),
            "ms_per_training_step": ms, "graph_sim_launches": it.launches_per_replay,
            "graph_synapse_launches": (net.syn_launches - syn0) // 2,  # warm-up + capture
            "loss": float(it.loss)}


def _errors(rec64, rec32, g64, g32, vcols):
    from jaxley_pytorch_b200.accuracy import gradient_error, voltage_errors

    out = voltage_errors(rec64[:, vcols], rec32[:, vcols])
    if g64 is not None:
        out["grad_rel_err"] = gradient_error(g64, g32)
    return out


def fp32_errors(device):
    """float32 against float64 of the same kernels on samples of the benchmarked
    configurations: max |dV| of the voltage recordings over the whole trace and over
    its subthreshold stretches, and the relative error of the adjoint's gradient of
    an MSE loss (largest deviation over the largest gradient entry)."""
    import torch

    from jaxley_pytorch_b200 import synth
    from jaxley_pytorch_b200.network import NetworkSimulation, config_network
    from jaxley_pytorch_b200.sim import Simulation

    def cell_run(prob, dtype, steady, kw):
        sim = Simulation(prob, dtype=dtype, device=device, init_steady=steady, **kw)
        ps = sim.model.pscale.clone().requires_grad_(True)
        rec = sim.run(pscale=ps)
        with torch.no_grad():
            target = rec.detach() * 0 + (-65.0)
        loss = ((rec - target) ** 2).mean()
        (g,) = torch.autograd.grad(loss, ps)
        return rec.detach().double().cpu().numpy(), g.double().cpu().numpy()

    out = {}
    kw = dict(keep_currents=False, checkpoint=100)
    prob = synth.config_l5pc_tree(batch=8, n_steps=4000, seed=0, scale_seed=1)
    r64, g64 = cell_run(prob, torch.float64, True, kw)
    r32, g32 = cell_run(prob, torch.float32, True, kw)
    out["C2"] = dict(_errors(r64, r32, g64, g32, [0]), sample="8 parameter sets, 4000 steps")
    prob = synth.config_uneven(n_cells=64, n_steps=2000)
    r64, g64 = cell_run(prob, torch.float64, False, kw)
    r32, g32 = cell_run(prob, torch.float32, False, kw)
    out["C3"] = dict(_errors(r64, r32, g64, g32, list(range(64))), sample="64 cells, 2000 steps")
    prob = config_network(n_cells=256, ncomp=4, k=64, batch=4, n_steps=2000, seed=0)

    def net_run(dtype):
        net = NetworkSimulation(prob, dtype=dtype, device=device, checkpoint=50, threads=256,
                                max_block_nodes=256)
        params = [[p.clone().requires_grad_(True)] + p_[1:] for p, p_ in
                  ((ty.params[0], ty.params) for ty in net.types)]
        rec = net.run(net.model.pscale, params)
        loss = ((rec + 65.0) ** 2).mean()
        grads = torch.autograd.grad(loss, [p[0] for p in params])
        return rec.detach().double().cpu().numpy(), torch.cat(grads).double().cpu().numpy()

    r64, g64 = net_run(torch.float64)
    r32, g32 = net_run(torch.float32)
    out["C4"] = dict(_errors(r64, r32, g64, g32, list(range(256))),
                     sample="256 cells, k = 64 of each type, 4 rows, 2000 steps; gradient of gS")
    return out


def import_reference():
    """The reference package (jaxley-pytorch) installed under `baseline/_ref`, or
    None. Its module-level matplotlib import (plotting only) is served by the
    stand-in package under `tests/golden/_mpl_stub`."""
    import importlib

    path = os.path.join(REPO, "baseline", "_ref")
    if not os.path.isdir(os.path.join(path, "jaxley_pytorch")):
        return None
    for p in (os.path.join(REPO, "tests", "golden", "_mpl_stub"), path):
        if p not in sys.path:
            sys.path.insert(0, p)
    try:
        return importlib.import_module("jaxley_pytorch")
    except Exception:
        return None


class ReferenceSample:
    """The reference's own torch path on the host cores: its `jx.integrate`
    (`voltage_solver="jaxley.dhs"`, float32) on `batch` of the workload's parameter
    sets and `tsteps` of its steps, the cell rebuilt with the reference's module API
    from the generator's morphology; `step()` is one forward + `loss.backward()` of
    the MSE of the somatic voltage to a held-out parameter set's trace, `forward()`
    the forward alone. Returns seconds."""

    def __init__(self, jx, batch: int, tsteps: int):
        import torch

        from jaxley_pytorch_b200 import synth

        self.jx, self.torch = jx, torch
        self.cores = os.cpu_count() or 1
        torch.set_num_threads(self.cores)
        prob = synth.config_l5pc_tree(batch=batch, n_steps=tsteps, seed=0, scale_seed=1)
        held = synth.config_l5pc_tree(batch=1, n_steps=tsteps, seed=0, scale_seed=10_000)
        m = prob.meta
        self.cell = synth.reference_l5pc_cell(jx, m["parents"], m["ncomp"], m["radius"], m["lengths"])
        self.cell.init_states()
        self.cell.branch(0).loc(0.0).record(verbose=False)
        delay, dur, amp = m["stim"]
        self.cell.branch(0).loc(0.0).stimulate(jx.step_current(delay, dur, amp, 0.025, tsteps * 0.025),
                                               verbose=False)
        self.t_max = (tsteps - 0.5) * 0.025  # tsteps steps (integrate.py:521)
        self.nb = len(m["parents"])
        base = {k: v for _, _, d in synth.L5PC_SOMA + synth.L5PC_DEND for k, v in d.items()}
        base["Leak_gLeak"] = 3e-05
        self.soma = {k for _, _, d in synth.L5PC_SOMA for k in d}
        self.dend = {k for _, _, d in synth.L5PC_DEND for k in d}
        self.values = {k: np.asarray(m["scales"][k])[:, None] * base[k] for k in synth.L5PC_SCALED}
        hv = {k: np.asarray(held.meta["scales"][k])[:, None] * base[k] for k in synth.L5PC_SCALED}
        with torch.no_grad():
            self.target = self._run(hv, grad=False)[0][..., 0, :]
        self.comp_steps = len(prob.comp_inds) * batch * tsteps

    def _run(self, values, grad: bool):
        torch = self.torch
        ps, leaves = None, []
        for k, v in values.items():
            val = torch.tensor(v, dtype=torch.float32, requires_grad=grad)
            view = (self.cell.branch(0) if k in self.soma
                    else self.cell.branch(list(range(1, self.nb))) if k in self.dend else self.cell)
            ps = view.data_set(k, val, ps)
            leaves.append(val)
        rec = self.jx.integrate(self.cell, param_state=ps, delta_t=0.025, t_max=self.t_max,
                                voltage_solver="jaxley.dhs")
        return rec, leaves

    def step(self) -> float:
        t0 = time.perf_counter()
        rec, leaves = self._run(self.values, grad=True)
        loss = ((rec[..., 0, :] - self.target) ** 2).mean()
        loss.backward()
        return time.perf_counter() - t0

    def forward(self) -> float:
        t0 = time.perf_counter()
        with self.torch.no_grad():
            self._run(self.values, grad=False)
        return time.perf_counter() - t0


def reference_baseline(batch: int, tsteps: int, warmup: int = 1, reps: int = 3):
    """`cpu_baseline` from the reference's own code: one warm-up, then the median of
    `reps` forward + backward and of `reps` forward-only runs. None without the
    reference installed."""
    jx = import_reference()
    if jx is None:
        return None
    smp = ReferenceSample(jx, batch, tsteps)
    for _ in range(warmup):
        smp.step()
    fb = float(np.median([smp.step() for _ in range(reps)]))
    smp.forward()
    fw = float(np.median([smp.forward() for _ in range(reps)]))
    return {"value": smp.comp_steps / fb, "unit": UNIT, "cores": smp.cores, "kind": "reference",
            "sample": f"{batch} of 256 rows x {tsteps} of 4000 steps, fwd+bwd (MSE), float32, "
                      f"jx.integrate voltage_solver=jaxley.dhs, median of {reps} after {warmup} warm-up",
            "seconds_fwd_bwd": fb, "forward": {"value": smp.comp_steps / fw, "unit": UNIT, "seconds": fw}}


# Published H100 figures of the reference's language-model HH networks (float32,
# 100 KineticSynapse inputs per neuron, 32 streams): ms per solver step, forward,
# recomputation and backward together (examples/language_modeling/README.md:115-116).
H100_MS_PER_SOLVER_STEP = {1024: 0.21, 2048: 0.33}


def run_lm(args, device, n_cells: int):
    """The reference's language-model Hodgkin-Huxley network shape (`n_cells` point
    neurons, 100 KineticSynapse inputs each, 80 % excitatory, 32 streams, float32,
    dt 0.025 ms): one training step = the simulation of 10 tokens x 200 solver steps,
    the MSE of the voltages to a target, the adjoint, and Adam (capturable) on the
    synaptic weights, replayed as one CUDA graph; reported per solver step beside
    the published H100 figure."""
    import torch

    from jaxley_pytorch_b200.graphs import GraphedIteration
    from jaxley_pytorch_b200.network import NetworkSimulation, config_lm

    prob = config_lm(n_cells=n_cells, n_tokens=args.lm_tokens)
    T = prob.n_steps
    net = NetworkSimulation(prob, dtype=torch.float32, device=device, checkpoint=50, threads=256,
                            max_block_nodes=256, init_steady=True)
    (ty,) = net.types
    with torch.no_grad():
        target = net.run(net.model.pscale, [[ty.params[0] * 1.2] + ty.params[1:]]).detach()

    def run(w):
        return net.run(net.model.pscale, [[w] + ty.params[1:]])

    def loss_fn(rec):
        return ((rec - target) ** 2).mean()

    w = ty.params[0].clone().requires_grad_(True)
    it = GraphedIteration(net, loss_fn, w, optimizer=torch.optim.Adam([w], lr=1e-6, capturable=True),
                          warmup=1, run=run)
    it.replay()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    reps = 2
    e0.record()
    for _ in range(reps):
        it.replay()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / reps
    per_step = ms / T
    h100 = H100_MS_PER_SOLVER_STEP.get(n_cells)
    return {"workload": f"lm_hh_{n_cells}x100_b32_t{T}_train_step", "neurons": n_cells,
            "synapses": int(ty.E), "batch": 32, "time_steps": T,
            "ms_per_training_step": ms, "ms_per_solver_step": per_step,
            "h100_ms_per_solver_step": h100, "speedup_over_h100": h100 / per_step if h100 else None,
            "synapse_steps_per_s": ty.E * 32 * T / (ms / 1e3),
            "value": n_cells * 32 * T / (ms / 1e3), "unit": UNIT, "loss": float(it.loss)}


def _device_us(fn, reps: int, calls: int = 20) -> float:
    """Device time of one call of `fn` in microseconds: `calls` calls captured in a
    CUDA graph (so that host-side dispatch does not pace the GPU), replayed `reps`
    times between CUDA events, after warm-up calls on a side stream."""
    import torch

    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(side):
        for _ in range(3):
            fn()
    torch.cuda.current_stream().wait_stream(side)
    torch.cuda.synchronize()
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph):
        for _ in range(calls):
            fn()
    graph.replay()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        graph.replay()
    e1.record()
    torch.cuda.synchronize()
    us = e0.elapsed_time(e1) * 1e3 / (reps * calls)
    del graph
    return us


def run_kernel_compare(device, reps: int = 20):
    """The standalone drop-in ops against the reference's Triton kernels, both on this
    GPU with the same inputs: the tree solve (`kernels/tree_solve.py`, registers and
    levels variants) on the 300 x 4 L5PC tree with 256 rows and on a forest of 512
    small trees with 32 rows, and the synapse step (`kernels/synapse_step.py`,
    KineticSynapse forward and backward with the gS gradient) at the language-model
    shapes (1024 and 2048 targets x 100 inputs, 32 rows), float32. Inputs stay in L2
    between calls, as in the reference's step loop. `fraction_of_hbm` counts one read
    of the operands and one write of the results."""
    import torch

    jx = import_reference()
    if jx is None:
        return {"unavailable": "the reference is not installed under baseline/_ref"}
    try:
        import triton  # noqa: F401
        from jaxley_pytorch.kernels import synapse_step as rss
        from jaxley_pytorch.kernels import tree_solve as rts
    except Exception as e:  # noqa: BLE001
        return {"unavailable": f"the reference's Triton kernels do not import: {e!r}"[:300]}
    if not (rts.HAS_TRITON and rss.HAS_TRITON):
        return {"unavailable": "triton is not importable for the reference's kernels"}
    from jaxley_pytorch.synapses import KineticSynapse

    from jaxley_pytorch_b200 import synth
    from jaxley_pytorch_b200.kernels import synapse_step as ss
    from jaxley_pytorch_b200.kernels import tree_solve as ts
    from jaxley_pytorch_b200.lower import lower

    peak = measured_peak_hbm()[0]
    gen = torch.Generator(device=device).manual_seed(3)
    out = {"tree_solve": [], "synapse_step": []}

    def systems(parent, B):
        n = len(parent)
        par = torch.as_tensor(parent, device=device)
        l = -0.05 - 0.35 * torch.rand(B, n, generator=gen, device=device)
        u = -0.05 - 0.35 * torch.rand(B, n, generator=gen, device=device)
        root = par < 0
        l[:, root] = 0
        u[:, root] = 0
        d = 1.5 + torch.rand(B, n, generator=gen, device=device) + l.abs()
        d.index_add_(1, par.clamp_min(0)[~root], u[:, ~root].abs())
        s = torch.randn(B, n, generator=gen, device=device)
        return d, l, u, s

    c2 = lower(synth.config_l5pc_tree(batch=1, n_steps=1, seed=0))
    rng = np.random.default_rng(5)
    small = []
    for _ in range(512):
        b = len(small)
        small += [-1] + [b + int(rng.integers(0, j)) for j in range(1, 40)]
    for name, parent, B in (("l5pc_tree_300x4", np.asarray(c2.parent), 256),
                            ("forest_512x40", np.asarray(small), 32)):
        d, l, u, s = systems(parent, B)
        n = len(parent)
        for mode in ("registers", "levels"):
            rk = rts.make_tree_solve_kernel(parent, device, mode=mode)
            ok = ts.make_tree_solve_kernel(parent, device, mode=mode)
            if rk is None or ok is None:
                continue
            err = float(((ok.solve(d, l, u, s) - rk.solve(d, l, u, s)).abs().max()
                         / rk.solve(d, l, u, s).abs().max()).item())
            t_ref = _device_us(lambda: rk.solve(d, l, u, s), reps)
            t_ours = _device_us(lambda: ok.solve(d, l, u, s), reps)
            nbytes = 5 * n * B * 4
            out["tree_solve"].append({
                "shape": f"{name}_b{B}", "nodes": n, "rows": B, "variant": mode,
                "us_reference_triton": t_ref, "us_ours": t_ours, "speedup": t_ref / t_ours,
                "fraction_of_hbm_ours": nbytes / (t_ours * 1e-6) / 1e9 / peak,
                "max_rel_diff": err})

    syn = KineticSynapse()
    names = list(syn.synapse_params)
    B, k = 32, 100
    for T in (1024, 2048):
        E = T * k
        n = T
        pre = np.concatenate([rng.choice(np.delete(np.arange(n), t), size=k, replace=False) for t in range(T)])
        targets = np.arange(T)
        v = -40.0 + 40.0 * torch.rand(B, n, generator=gen, device=device)  # around v_th: both voltage gradients
        st = torch.rand(B, E, generator=gen, device=device)
        params = []
        for q, nm in enumerate(names):
            base = float(syn.synapse_params[nm])
            p = torch.full((E,), base, device=device)
            if q == 0:
                p = p * (0.5 + torch.rand(E, generator=gen, device=device))
            if q == 1:  # e_syn: excitatory 0 mV, inhibitory -80 mV (one in five)
                p = torch.where(torch.rand(E, generator=gen, device=device) < 0.8, 0.0, -80.0)
            params.append(p)
        params += [params[0]] * (6 - len(params))
        area = torch.full((E,), 100.0, device=device)
        g_sn = torch.randn(B, E, generator=gen, device=device)
        g_lin = torch.randn(B, T, generator=gen, device=device)
        g_const = torch.randn(B, T, generator=gen, device=device)
        none = v.new_empty(0)
        row = {"shape": f"kinetic_{T}x{k}_b{B}", "synapses": E, "rows": B}
        for tag, mod in (("reference_triton", rss), ("ours", ss)):
            plan = mod.kernel_plan(syn, pre, targets, n, device)
            if tag == "ours":
                ss._ensure_ops()
            sc = mod.kernel_scalars(0.025, 1e-3, torch.float32, device)
            fargs = (v, st, plan["kernel_pre"], plan["kernel_targets"], *params, area, sc, plan["kernel_inv"],
                     plan["kernel_pre_nodes"], k, rss.KINETIC, True, False)
            bargs = (v, st, plan["kernel_pre"], plan["kernel_targets"], *params, area, sc, plan["kernel_inv"],
                     plan["kernel_pre_nodes"], g_sn, none, g_lin, g_const, k, rss.KINETIC, True, True, False, 1)
            row[f"us_forward_{tag}"] = _device_us(lambda: mod.synapse_step_op(*fargs), reps)
            row[f"us_backward_{tag}"] = _device_us(lambda: mod.synapse_step_backward_op(*bargs), reps)
            row[f"outputs_{tag}"] = (mod.synapse_step_op(*fargs), mod.synapse_step_backward_op(*bargs))
        fo, bo = row.pop("outputs_ours")
        fr, br = row.pop("outputs_reference_triton")
        outs = ("s_new", "lin", "const", "g_v", "g_s", "g_gS")
        f32_ours = (fo[0], fo[2], fo[3], bo[0], bo[1], bo[2])
        f32_ref = (fr[0], fr[2], fr[3], br[0], br[1], br[2])
        # The same calls in float64: the float32 differences in g_s and g_gS are the
        # cancellation in the adjoint of the finite-difference slope (1e-3 mV), which
        # both implementations evaluate in their own order.
        d64 = []
        for mod in (ss, rss):
            plan = mod.kernel_plan(syn, pre, targets, n, device)
            sc = mod.kernel_scalars(0.025, 1e-3, torch.float64, device)
            dd = lambda x: x.double()  # noqa: E731
            fa = (dd(v), dd(st), plan["kernel_pre"], plan["kernel_targets"], *[dd(p) for p in params], dd(area), sc,
                  plan["kernel_inv"], plan["kernel_pre_nodes"], k, rss.KINETIC, True, False)
            ba = fa[:14] + (dd(g_sn), none.double(), dd(g_lin), dd(g_const), k, rss.KINETIC, True, True, False, 1)
            fo64, bo64 = mod.synapse_step_op(*fa), mod.synapse_step_backward_op(*ba)
            d64.append((fo64[0], fo64[2], fo64[3], bo64[0], bo64[1], bo64[2]))
        def rel(a, b):
            return float(((a.double() - b.double()).abs().max() / b.double().abs().max().clamp_min(1e-300)).item())

        # float64: the two implementations against each other; float32: each against
        # the reference's float64 result
        row["max_rel_diff_f64"] = {nm: rel(a, b) for nm, a, b in zip(outs, d64[0], d64[1])}
        row["f32_error_ours"] = {nm: rel(a, b) for nm, a, b in zip(outs, f32_ours, d64[1])}
        row["f32_error_reference_triton"] = {nm: rel(a, b) for nm, a, b in zip(outs, f32_ref, d64[1])}
        row["speedup_forward"] = row["us_forward_reference_triton"] / row["us_forward_ours"]
        row["speedup_backward"] = row["us_backward_reference_triton"] / row["us_backward_ours"]
        out["synapse_step"].append(row)
    out["note"] = ("device time per call: 20 calls captured in a CUDA graph, replayed %d times; float32, "
                   "same inputs for both; operands resident in L2 between calls" % reps)
    return out


def kernel_compare_child(local: int, timeout_s: int = 600):
    """`run_kernel_compare` in a child process (the reference's Triton kernels are
    compiled and run there), so that a failure of that path leaves the rest of the
    line intact; its stderr tail is kept when it fails."""
    cmd = [sys.executable, "-X", "faulthandler", os.path.abspath(__file__), "--kernel-compare-only",
           "--local-device", str(local)]
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout_s)
    except subprocess.TimeoutExpired:
        return {"unavailable": f"the comparison did not finish within {timeout_s} s"}
    if r.returncode == 0 and r.stdout.strip():
        return json.loads(r.stdout.strip().splitlines()[-1])
    return {"unavailable": f"the comparison process ended with status {r.returncode}",
            "stderr_tail": r.stderr[-1500:]}


def cpu_sample(batch: int, tsteps: int, reps: int = 1):
    """Times the torch CPU restatement of the reference path (forward + autograd
    backward) on `batch` rows x `tsteps` steps of the workload."""
    import torch

    from jaxley_pytorch_b200 import synth
    from oracle import torch_port

    cores = os.cpu_count() or 1
    torch.set_num_threads(cores)
    prob = synth.config_l5pc_tree(batch=batch, n_steps=tsteps, seed=0, scale_seed=1)
    held = synth.config_l5pc_tree(batch=1, n_steps=tsteps, seed=0, scale_seed=10_000)
    with torch.no_grad():
        target = torch_port.integrate(held, {}, dtype=torch.float32, init_steady=True)[0, 0]
    names = synth.L5PC_SCALED
    params = {k: torch.as_tensor(np.asarray(prob.params[k]), dtype=torch.float32).requires_grad_(True)
              for k in names}
    n_comp = len(prob.comp_inds)
    times = []
    for r in range(reps + 1):
        t0 = time.perf_counter()
        rec = torch_port.integrate(prob, params, dtype=torch.float32, init_steady=True)
        loss = ((rec[:, 0, :] - target) ** 2).mean()
        loss.backward()
        times.append(time.perf_counter() - t0)
    t = float(np.median(times[1:])) if reps > 0 else times[0]
    return n_comp * batch * tsteps / t, cores, t


def main():
    args = parse()
    if args.kernel_compare_only:
        import torch

        print(json.dumps(run_kernel_compare(torch.device("cuda", args.local_device))))
        return 0
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank != 0:
            return 0
        jx = import_reference()
        sample = (f"{args.cpu_batch} of 256 rows x {args.cpu_tsteps} of 4000 steps per step, fwd+bwd "
                  f"(MSE), float32")
        if jx is not None:  # the reference's own jx.integrate on the host cores
            smp = ReferenceSample(jx, args.cpu_batch, args.cpu_tsteps)
            for _ in range(args.warmup):
                smp.step()
            secs = [smp.step() for _ in range(args.steps)]
            value = smp.comp_steps / float(np.median(secs))
            cores, kind = smp.cores, "reference"
            sample += ", jx.integrate voltage_solver=jaxley.dhs from baseline/_ref"
        else:  # the CPU port of the reference's path
            for _ in range(args.warmup):
                cpu_sample(args.cpu_batch, args.cpu_tsteps, reps=0)
            vals, secs = [], []
            for _ in range(args.steps):
                v, cores, t = cpu_sample(args.cpu_batch, args.cpu_tsteps, reps=0)
                vals.append(v)
                secs.append(t)
            value, kind = float(np.median(vals)), "port"
            sample += ", CPU port of the reference path (reference not installed)"
        out = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
               "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
               "ms_per_step": float(np.median(secs)) * 1e3, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f32", "data": "synthetic",
               "config": {"workload": "l5pc_tree_300x4_b256_t4000_fwd_adjoint"},
               "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind,
                                "sample": sample},
               "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                       "d2h_bytes_per_step": 0}}
        print(json.dumps(out))
        return 0
    import torch

    if world > 1:
        torch.distributed.init_process_group("nccl", timeout=timedelta(seconds=300),
                                             device_id=torch.device("cuda", local))
    device = torch.device("cuda", local)
    t_start = time.perf_counter()

    def section(name, fn):
        t0 = time.perf_counter()
        res = fn()
        print(f"[bench] {name}: {time.perf_counter() - t0:.1f} s (total {time.perf_counter() - t_start:.1f} s)",
              file=sys.stderr, flush=True)
        return res

    out = section("main iteration", lambda: run_ours(args, rank, world, device))
    if world == 1 and not args.no_uneven:
        out["uneven"] = section("uneven batch", lambda: run_uneven(args, device))
    if world == 1 and not args.no_serving:
        out["serving"] = section("serving", lambda: run_serving(args, device))
    if world == 1 and not args.no_network:
        out["network"] = section("network", lambda: run_network(args, device))
    if world == 1 and not args.no_lm:
        out["lm_network"] = section("lm networks", lambda: [run_lm(args, device, n) for n in (1024, 2048)])
    if world == 1 and not args.no_fp32_error:
        out["fp32_error"] = section("fp32 errors", lambda: fp32_errors(device))
    if world == 1 and not args.no_kernel_compare:
        out["dropin_vs_triton"] = section("drop-in ops vs the reference's Triton kernels",
                                          lambda: kernel_compare_child(local))
    if rank == 0:
        if world == 1 and not args.no_cpu_baseline:
            ref = section("cpu baseline", lambda: reference_baseline(args.cpu_batch, args.cpu_tsteps))
            if ref is not None:
                out["cpu_baseline"] = ref
            else:
                v, cores, t = cpu_sample(args.cpu_batch, args.cpu_tsteps, reps=0)
                out["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                                       "sample": f"{args.cpu_batch} of 256 rows x {args.cpu_tsteps} of "
                                                 f"4000 steps, fwd+bwd, {t:.1f} s (reference not installed)"}
        print(json.dumps(out))
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
