"""The drop-in boundary inside the reference itself.

1. The reference's own `jx.integrate`, run on CUDA with this package's
   `make_tree_solve_kernel` / `fused_tree_solve` installed at the call sites of
   `DHSSolver.__init__` and `dhs_solve` (`solver_voltage.py:69-76, 237-240`) and its
   `kernel_plan` / `kernel_scalars` / `fused_step` at those of the network step
   (`modules/network.py:343-346, 402-407`, `integrate.py:600-611`), must give the
   recordings (1e-9 relative) and the autograd gradients (1e-8 relative) of the
   reference's own run on the CPU, float64, for HH and L5PC cells, a cell with clamps
   and a synapse network. The call sites import these names from
   `jaxley_pytorch.kernels.*` when they run, so replacing the module attributes is
   exactly the binding a maintainer would add.
2. This package's `integrate` (the reference's signature, fused kernels and
   hand-written adjoint) on the same models: recordings 1e-9, gradients 1e-6.

The reference is imported from `baseline/_ref` (or `JXB_REFERENCE`); the tests skip
where it is not installed.
"""
import numpy as np
import pytest
import torch

import reference_models as rm
from conftest import import_reference

pytestmark = pytest.mark.gpu

CELLS = ["hh_tree", "l5pc_cell", "clamped_cell", "hh_tree_cn", "pospischil_cell"]


def _build(jx, name):
    f = getattr(rm, name)
    return f(jx, torch) if name == "clamped_cell" else f(jx)


def _to(x, device):
    if isinstance(x, torch.Tensor):
        return x.to(device)
    if isinstance(x, dict):
        return {k: _to(v, device) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return type(x)(_to(v, device) for v in x)
    return x


def _run(fn, module, kw, device):
    """Recordings and gradients of `sum(w * recordings)` (w seeded) with respect to
    every trainable of `module`, run by `fn` (an `integrate`) on `device` in float64."""
    params = [{k: v.detach().to(device=device, dtype=torch.float64).requires_grad_(True)
               for k, v in p.items()} for p in module.get_parameters()]
    rec = fn(module, params=params, **_to(kw, device))
    w = torch.as_tensor(np.random.default_rng(5).normal(size=tuple(rec.shape)), device=rec.device)
    (rec * w).sum().backward()
    grads = [list(p.values())[0].grad.detach().cpu().numpy() for p in params]
    return rec.detach().cpu().numpy(), grads


def _rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


@pytest.fixture(scope="module")
def jx_with_dropin(cuda_device):
    jx = import_reference()
    import jaxley_pytorch.kernels.synapse_step as ref_ss
    import jaxley_pytorch.kernels.tree_solve as ref_ts

    from jaxley_pytorch_b200.kernels import synapse_step as ss
    from jaxley_pytorch_b200.kernels import tree_solve as ts

    mp = pytest.MonkeyPatch()
    mp.setattr(ref_ts, "HAS_TRITON", True)
    mp.setattr(ref_ts, "make_tree_solve_kernel", ts.make_tree_solve_kernel)
    mp.setattr(ref_ts, "fused_tree_solve", ts.fused_tree_solve)
    mp.setattr(ref_ss, "HAS_TRITON", True)
    mp.setattr(ref_ss, "kernel_plan", ss.kernel_plan)
    mp.setattr(ref_ss, "kernel_scalars", ss.kernel_scalars)
    mp.setattr(ref_ss, "fused_step", ss.fused_step)
    yield jx
    mp.undo()


@pytest.mark.parametrize("name", CELLS + ["synapse_net"])
def test_reference_integrate_runs_the_dropin_kernels(jx_with_dropin, cuda_device, name):
    jx = jx_with_dropin
    from jaxley_pytorch_b200.kernels import tree_solve as ts

    module, kw = _build(jx, name)
    rec_cpu, g_cpu = _run(jx.integrate, module, kw, "cpu")
    calls = {"n": 0}
    orig = ts.fused_tree_solve

    def counting(*a):
        calls["n"] += 1
        return orig(*a)

    import jaxley_pytorch.kernels.tree_solve as ref_ts
    with pytest.MonkeyPatch.context() as mp:
        mp.setattr(ref_ts, "fused_tree_solve", counting)
        rec_gpu, g_gpu = _run(jx.integrate, module, kw, cuda_device)
    assert calls["n"] > 0  # the voltage solve went through this package's kernel
    assert _rel(rec_gpu, rec_cpu) <= 1e-9
    for a, b in zip(g_gpu, g_cpu):
        assert _rel(a, b) <= 1e-8


@pytest.mark.parametrize("name", CELLS)
def test_integrate_entry_matches_reference(cuda_device, name):
    jx = import_reference()
    from jaxley_pytorch_b200.integrate import integrate

    module, kw = _build(jx, name)
    rec_ref, g_ref = _run(jx.integrate, module, kw, "cpu")
    rec, g = _run(integrate, module, kw, cuda_device)
    assert rec.shape == rec_ref.shape
    assert _rel(rec, rec_ref) <= 1e-9
    for a, b in zip(g, g_ref):
        assert a.shape == b.shape
        assert _rel(a, b) <= 1e-6


def test_integrate_return_states_and_all_states(cuda_device):
    """`return_states` gives the reference's final states, and a run that starts from
    them (`all_states`) gives the reference's recordings from the same states."""
    jx = import_reference()
    from jaxley_pytorch_b200.integrate import integrate

    module, kw = rm.hh_tree(jx)
    gna = torch.tensor([0.12], dtype=torch.float64)
    ps_gpu = module.data_set("HH_gNa", gna.to(cuda_device), None)
    ps_cpu = module.data_set("HH_gNa", gna, None)
    rec, states = integrate(module, param_state=ps_gpu, t_max=3.0, return_states=True, **kw)
    ref_rec, ref_states = jx.integrate(module, param_state=ps_cpu, t_max=3.0, return_states=True, **kw)
    assert _rel(rec.cpu().numpy(), ref_rec.detach().numpy()) <= 1e-9
    for k in ("v", "HH_m", "HH_h", "HH_n"):
        assert _rel(states[k].cpu().numpy(), ref_states[k].detach().numpy()) <= 1e-9
    again = integrate(module, param_state=ps_gpu, t_max=3.0, all_states=states, **kw)
    ref_again = jx.integrate(module, param_state=ps_cpu, t_max=3.0,
                             all_states={k: v.detach() for k, v in ref_states.items()}, **kw)
    assert _rel(again.cpu().numpy(), ref_again.detach().numpy()) <= 1e-9
