"""The multi-GPU bench path on CPU with the gloo backend (world size 2): the timing
is the maximum over ranks, and every rank simulates its own parameter sets of the
same shape (weak scaling, no collective in the data path)."""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

from conftest import REPO


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, out):
    import torch.distributed as dist

    sys.path.insert(0, REPO)
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        t = bench.max_over_ranks(10.0 + 5.0 * rank, world, "cpu")
        prob, held = bench.workload(rank, batch=4, tsteps=10)
        scale = np.asarray(prob.params[sorted(k for k in prob.params if k.endswith("_gNaTs2T"))[0]])
        out[rank] = (t, prob.n_nodes, prob.batch, float(scale.sum()))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_per_rank_workloads():
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    port = _free_port()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, start_method="spawn", join=True)
    (t0, n0, b0, s0), (t1, n1, b1, s1) = out[0], out[1]
    assert t0 == t1 == 15.0  # both ranks report the slowest
    assert n0 == n1 and b0 == b1 == 4  # same shapes on every rank
    assert s0 != s1  # different parameter sets per rank
