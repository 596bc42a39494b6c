"""Serving loop host logic (CPU): launch sizing over requests, the CTA pair list,
admission estimates and the latency summary."""
import numpy as np

from jaxley_pytorch_b200 import _lib, synth
from jaxley_pytorch_b200.lower import lower
from jaxley_pytorch_b200.serve import (Request, launch_sizes, pair_list, request_bytes,
                                       request_bytes_estimate, summarize)


def test_launch_sizes_are_the_maxima_over_requests():
    args = []
    for k in range(3):
        a = _lib.JxbSimArgs()
        a.max_rows, a.max_nodes, a.max_slots = 1, 100 * (k + 1), 700 - 100 * k
        a.max_chains, a.max_child, a.max_levels, a.max_pslots = 10 + k, 5, 3 * k + 1, 40
        a.max_gslots, a.n_entries, a.n_classes = 7, 5 + k, 3
        args.append(a)
    sz = launch_sizes(args)
    assert sz["max_nodes"] == 300 and sz["max_slots"] == 700 and sz["max_levels"] == 7
    assert sz["n_entries"] == 7 and sz["max_chains"] == 12 and sz["max_rows"] == 1


def test_pair_list_covers_items_largest_first():
    nodes = [np.array([5, 300]), np.array([120]), np.array([7, 7, 900])]
    pairs = pair_list(nodes)
    assert sorted(map(tuple, pairs.tolist())) == [(0, 0), (0, 1), (1, 0), (2, 0), (2, 1), (2, 2)]
    sizes = [nodes[r][i] for r, i in pairs]
    assert sizes == sorted(sizes, reverse=True)
    assert pairs.dtype == np.int32 and pairs.flags["C_CONTIGUOUS"]


def test_admission_estimate_bounds_the_request_memory():
    for seed, grad in [(1, False), (2, True), (3, True)]:
        prob = synth.config_uneven(n_cells=1, seed=seed, n_steps=800, min_comp=8, max_comp=3000)
        req = Request(problem=prob, n_steps=800, grad=grad)
        low = lower(prob, keep_currents=False)
        exact = request_bytes(low, 800, grad, 100)
        est = request_bytes_estimate(req, 100)
        assert est > 0 and exact > 0
        assert 0.25 * exact <= est <= 8 * exact
        if grad:
            assert request_bytes(low, 800, True, 100) > request_bytes(low, 800, False, 100)


def test_summary_percentiles():
    reqs = []
    for i in range(100):
        r = Request(problem=None, n_steps=1, arrival=0.0)
        r.finished = (i + 1) * 1e-3
        reqs.append(r)
    s = summarize(reqs, 0.1, 1000)
    assert abs(s["p50_ms"] - 50.5) < 1e-6 and abs(s["p99_ms"] - 99.01) < 1e-6
    assert s["throughput"] == 1000 / 0.1 and s["requests"] == 100


def test_fifo_latencies_and_slowdown():
    from jaxley_pytorch_b200.serve import fifo_latencies

    # arrivals 0, 1, 1.5; service 2, 1, 1: done at 2, 3, 4
    lat = fifo_latencies([0.0, 1.0, 1.5], [2.0, 1.0, 1.0])
    assert np.allclose(lat, [2.0, 2.0, 2.5])
    r = Request(problem=None, n_steps=1, arrival=1.0)
    r.finished, r.service = 4.0, 1.5
    assert r.slowdown == 2.0
    s = summarize([r], 1.0, 10)
    assert s["slowdown_p50"] == 2.0


def test_step_cost_grows_with_levels_and_nodes():
    from jaxley_pytorch_b200.serve import step_cost_us

    small = lower(synth.config_uneven(n_cells=1, seed=1, n_steps=10, min_comp=8, max_comp=9), keep_currents=False)
    big = lower(synth.config_l5pc_tree(batch=1, n_steps=10), keep_currents=False)
    assert 2.0 < step_cost_us(small) < step_cost_us(big) < 60.0
