"""A whole gradient (or training) iteration captured once as a CUDA graph.

The iteration — the forward launches, the loss, the adjoint launches in reverse
segment order and, optionally, a capturable optimizer step — is captured once with
`torch.cuda.graph` and replayed with one call, so the host issues no per-launch work
(the reference's step loop issues its kernels from Python every step,
`integrate.py:396-666`). The simulation's launches go on the current stream (the
capture stream); the fork onto the side stream for oversized blocks is joined back
inside the capture.
"""
from __future__ import annotations

from typing import Callable, Optional

import torch

from .sim import Simulation


class GraphedIteration:
    """`loss_fn(recordings) -> scalar` on `sim.run(pscale=params)` (or on `run(params)`
    when given, e.g. a network's simulation with `params` as its synapse weights), its gradient with
    respect to `params` (a leaf tensor on the device) and an optional optimizer step
    over `[params]` (it must be capturable, e.g. `torch.optim.Adam(..., capturable=True)`).

    `replay()` runs the iteration and returns the static `(loss, grad)` tensors, which
    the next replay overwrites. Inputs that change between iterations (targets,
    stimuli) must be written in place into the tensors the capture used.
    """

    def __init__(self, sim: Simulation, loss_fn: Callable[[torch.Tensor], torch.Tensor],
                 params: torch.Tensor, n_steps: Optional[int] = None,
                 optimizer: Optional[torch.optim.Optimizer] = None, warmup: int = 2,
                 run: Optional[Callable[[torch.Tensor], torch.Tensor]] = None):
        if not params.is_leaf or not params.requires_grad:
            raise ValueError("params must be a leaf tensor that requires grad")
        self.sim, self.loss_fn, self.params = sim, loss_fn, params
        self.n_steps, self.optimizer = n_steps, optimizer
        self.run_fn = run
        dev = sim.model.device
        side = torch.cuda.Stream(dev)
        side.wait_stream(torch.cuda.current_stream(dev))
        with torch.cuda.stream(side):  # warm-up: allocations, optimizer state
            for _ in range(max(1, warmup)):
                self._body()
        torch.cuda.current_stream(dev).wait_stream(side)
        torch.cuda.synchronize(dev)
        # The warm-up's buffers (a stored trajectory can take tens of GB) go back to the
        # device before the capture allocates its own from the graph's pool.
        torch.cuda.empty_cache()
        self.graph = torch.cuda.CUDAGraph()
        n0 = sim.model.launches
        with torch.cuda.graph(self.graph):
            self.loss, self.grad = self._body()
        self.launches_per_replay = sim.model.launches - n0

    def _body(self):
        if self.run_fn is not None:
            rec = self.run_fn(self.params)
        else:
            rec = self.sim.run(n_steps=self.n_steps, pscale=self.params)
        loss = self.loss_fn(rec)
        (g,) = torch.autograd.grad(loss, self.params)
        if self.optimizer is not None:
            self.params.grad = g
            self.optimizer.step()
        return loss.detach(), g

    def replay(self):
        self.graph.replay()
        return self.loss, self.grad
