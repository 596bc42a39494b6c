"""Continuous batching: every served request's recordings equal those of the same
problem simulated alone through the per-request path (bit for bit: the same
arithmetic per work item), and its gradient agrees to 1e-12 relative (float64 column
sums accumulated with atomics in a different order). The same request gives the same
result alone in the server and in a mix."""
import numpy as np
import pytest
import torch

from jaxley_pytorch_b200.serve import Request, Server, make_stream, serve_plain

pytestmark = pytest.mark.gpu


def _copy(reqs, arrival=None):
    return [Request(problem=r.problem, n_steps=r.n_steps, grad=r.grad,
                    arrival=r.arrival if arrival is None else arrival, rid=r.rid) for r in reqs]


def _check_same(a, b, rtol=1e-12):
    assert a.recordings.shape == b.recordings.shape
    assert np.array_equal(a.recordings, b.recordings), np.abs(a.recordings - b.recordings).max()
    if a.grad:
        s = np.abs(b.gradient).max()
        assert s > 0
        assert np.abs(a.gradient - b.gradient).max() <= rtol * s


@pytest.mark.parametrize("force_global,policy", [(False, "fixed"), (True, "fixed"), (False, "slice")])
def test_served_results_equal_the_per_request_path(cuda_device, force_global, policy):
    reqs = make_stream(10, seed=3, rate=2000.0, grad_fraction=0.4, min_comp=8, max_comp=600,
                       t_range=(2.0, 12.0))
    assert any(r.grad for r in reqs) and not all(r.grad for r in reqs)
    kw = dict(chunk=64, checkpoint=50) if policy == "fixed" else dict(slice_ms=0.3, min_chunk=8)
    server = Server(device=cuda_device, threads=256, **kw)
    if force_global:
        server.smem_limit = 1  # every request's items run with global work areas
    stats = server.run(_copy(reqs))
    assert stats["requests"] == len(reqs) and stats["ticks"] >= 2
    served = {r.rid: r for r in server.done}
    plain = _copy(reqs, arrival=0.0)
    serve_plain(plain, device=cuda_device, threads=256, checkpoint=50)
    for p in plain:
        _check_same(served[p.rid], p, rtol=1e-6)


def test_same_result_alone_and_in_a_mix(cuda_device):
    reqs = make_stream(8, seed=11, rate=5000.0, grad_fraction=0.5, min_comp=8, max_comp=800,
                       t_range=(2.0, 10.0))
    probe = next(r for r in reqs if r.grad)
    alone = Server(device=cuda_device, chunk=50, threads=256, checkpoint=40)
    alone.run(_copy([probe], arrival=0.0))
    mix = Server(device=cuda_device, chunk=50, threads=256, checkpoint=40)
    mix.run(_copy(reqs))
    in_mix = next(r for r in mix.done if r.rid == probe.rid)
    _check_same(in_mix, alone.done[0])


def test_admission_respects_the_hbm_budget(cuda_device):
    reqs = make_stream(6, seed=5, rate=1e6, grad_fraction=1.0, min_comp=200, max_comp=400,
                       t_range=(2.0, 4.0))
    from jaxley_pytorch_b200.serve import request_bytes_estimate

    one = max(request_bytes_estimate(r, 40) for r in reqs)
    server = Server(device=cuda_device, chunk=40, threads=256, checkpoint=40, hbm_budget=int(2.5 * one))
    peak = []
    orig = server.tick

    def tick():
        orig()
        peak.append(len(server.active))

    server.tick = tick
    stats = server.run(_copy(reqs, arrival=0.0))
    assert stats["requests"] == 6
    assert max(peak) <= 2  # never more than the budget holds
