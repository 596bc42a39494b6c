"""Shared-parameter gradients over several ranks (`network.shard_rows`,
`network.allreduce_gradients`): two `gloo` ranks on the CPU each simulate half of a
network's batch rows (the torch restatement of the reference step) and all-reduce the
gradient of the synaptic weights shared by all rows; the sum must equal the gradient
of one rank simulating the whole batch (float64, 1e-12 relative)."""
import os

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from jaxley_pytorch_b200.network import allreduce_gradients, config_network, shard_rows


def _problem():
    return config_network(n_cells=10, ncomp=2, k=3, batch=4, n_steps=60, seed=2, rate_hz=400.0, amp=0.3)


def _grads(prob, n_rows_total):
    """Gradient of the rows' share of the batch loss with respect to every synapse
    type's gS (shared by all rows)."""
    from oracle import torch_port

    gs = [torch.as_tensor(np.asarray(s.params[0]), dtype=torch.float64).requires_grad_(True)
          for s in prob.synapses]
    syn = [[g] + [torch.as_tensor(np.asarray(x), dtype=torch.float64) for x in s.params[1:]]
           for g, s in zip(gs, prob.synapses)]
    rec = torch_port.integrate(prob, {}, dtype=torch.float64, syn_params=syn)
    loss = ((rec + 65.0) ** 2).sum() / n_rows_total
    return [g.detach() for g in torch.autograd.grad(loss, gs)]


def _worker(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        prob = _problem()
        shard = shard_rows(prob, rank, world)
        grads = _grads(shard, prob.batch)
        allreduce_gradients(grads)
        torch.save(grads, os.path.join(out_dir, f"g{rank}.pt"))
    finally:
        dist.destroy_process_group()


def test_sharded_rows_allreduce_equals_one_rank(tmp_path):
    prob = _problem()
    assert shard_rows(prob, 0, 2).batch == 2 and shard_rows(prob, 1, 2).stim.shape[0] == 2
    ref = _grads(prob, prob.batch)
    port = 29500 + os.getpid() % 1000
    mp.start_processes(_worker, args=(2, port, str(tmp_path)), nprocs=2, start_method="spawn")
    for rank in range(2):
        got = torch.load(tmp_path / f"g{rank}.pt")
        for a, b in zip(got, ref):
            assert (a - b).abs().max().item() <= 1e-12 * b.abs().max().item()
