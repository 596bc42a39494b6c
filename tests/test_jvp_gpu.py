"""Forward-mode derivatives: the fused forward kernel in dual numbers (`jxb_sim_tangent`,
`Simulation.jvp`) against the reference's `torch.func.jvp` through its `jx.integrate`
(the tree solve's forward-mode rule `_DHSSolveForwardAD`, solver_voltage.py:190-224).

The fixtures hold the reference's tangent of the recordings along seeded directions of
the trainable parameters, in float64 (`tests/golden/make_fixtures.py`); the entry-level
tests run the reference itself on the CPU beside the package's `integrate` under
`torch.func.jvp` and `torch.autograd.forward_ad`, as the reference's own
`test_jvp_through_simulation_matches_vjp` (tests/test_solver.py:198-232) does.
"""
import numpy as np
import pytest
import torch

from conftest import import_reference, load_fixture
from jaxley_pytorch_b200.lower import lower
from jaxley_pytorch_b200.sim import Simulation

pytestmark = pytest.mark.gpu

JVP_FIXTURES = ["hh_clamp_7x3", "pospischil_7x3", "cn_hh_7x3"]


def _rel(got, ref):
    got, ref = np.asarray(got, dtype=np.float64), np.asarray(ref, dtype=np.float64)
    return np.abs(got - ref).max() / max(np.abs(ref).max(), 1e-300)


def _direction(low, extra):
    """The tangent of the parameter-scale columns `(B, n_cols)` for the fixture's
    directions of its trainables (column value = trainable value / base scale)."""
    cols, base = low.group_scale()
    src = extra["trainable_source"]
    d = np.zeros((low.batch, low.n_cols))
    for g, (q, k) in enumerate(src):
        assert cols[g] > 0, (q, k)
        d[:, cols[g]] += extra[f"jvp_dir_{q}"].reshape(-1)[k] / base[g]
    return d


@pytest.mark.parametrize("name", JVP_FIXTURES)
def test_tangent_matches_reference_jvp(cuda_device, name):
    prob, extra = load_fixture(name)
    low = lower(prob)
    sim = Simulation(prob, low=low, dtype=torch.float64, device=cuda_device)
    d = torch.as_tensor(_direction(low, extra), device=cuda_device)
    rec, tan = sim.jvp(sim.model.pscale, d)
    ref = extra["ref"].reshape(rec.shape)
    assert _rel(rec.cpu().numpy(), ref) <= 1e-9
    err = _rel(tan.cpu().numpy(), extra["jvp"].reshape(tan.shape))
    assert err <= 1e-7, err
    # The values of the dual launch are the plain forward's (to round-off: the dual
    # arithmetic contracts some products differently).
    plain = sim.run(pscale=sim.model.pscale)
    assert _rel(rec.cpu(), plain.cpu()) <= 1e-12


@pytest.mark.parametrize("name", ["hh_clamp_7x3", "cn_hh_7x3"])
def test_tangent_float32(cuda_device, name):
    """Dual<float>: the tangent within 1e-3 of its largest value (float64 reference),
    on these cells whose recordings stay below the spike threshold for most of the run
    (the tangent of a spike time is sensitive to the rounding of the state)."""
    prob, extra = load_fixture(name)
    low = lower(prob)
    sim = Simulation(prob, low=low, dtype=torch.float32, device=cuda_device)
    d = torch.as_tensor(_direction(low, extra), device=cuda_device, dtype=torch.float32)
    _, tan = sim.jvp(sim.model.pscale, d)
    err = _rel(tan.cpu().numpy(), extra["jvp"].reshape(tan.shape))
    assert err <= 1e-3, err


def test_tangent_linear_and_adjoint_consistent(cuda_device):
    """w^T (J q) equals (J^T w)^T q between the forward-mode kernel and the adjoint
    kernel, and the tangent is linear in the direction. Column 0 (the unit scale of
    the parameters without a column of their own, which are not trainable and get no
    gradient slots in the adjoint) is left out of the directions."""
    prob, extra = load_fixture("pospischil_7x3")
    low = lower(prob)
    sim = Simulation(prob, low=low, dtype=torch.float64, device=cuda_device)
    gen = torch.Generator(device="cpu").manual_seed(5)
    q1 = torch.randn(low.batch, low.n_cols, generator=gen, dtype=torch.float64).to(cuda_device)
    q2 = torch.randn(low.batch, low.n_cols, generator=gen, dtype=torch.float64).to(cuda_device)
    q1[:, 0] = 0.0
    q2[:, 0] = 0.0
    _, t1 = sim.jvp(sim.model.pscale, q1)
    _, t2 = sim.jvp(sim.model.pscale, q2)
    _, t12 = sim.jvp(sim.model.pscale, 2.0 * q1 - 0.5 * q2)
    assert _rel((2.0 * t1 - 0.5 * t2).cpu(), t12.cpu()) <= 1e-6
    ps = sim.model.pscale.clone().requires_grad_(True)
    rec = sim.run(pscale=ps)
    w = torch.randn(rec.shape, generator=gen, dtype=torch.float64).to(cuda_device)
    (g,) = torch.autograd.grad((w * rec).sum(), ps)
    lhs, rhs = float((w * t1).sum()), float((g * q1).sum())
    assert abs(lhs - rhs) <= 1e-7 * max(abs(lhs), abs(rhs), 1.0)


def test_state_tangent(cuda_device):
    """A tangent of the initial state (as a Lyapunov-exponent computation advances it,
    examples/paper/fig4_lyapunov.py): against central differences of the float64
    forward."""
    prob, _ = load_fixture("cn_hh_7x3")
    low = lower(prob)
    sim = Simulation(prob, low=low, dtype=torch.float64, device=cuda_device, check_finite=False)
    T = 120
    gen = torch.Generator(device="cpu").manual_seed(9)
    s0 = sim.model.initial_state()
    ds = torch.zeros_like(s0)
    v_slots = [int(s) for s in np.asarray(low.soff)[:low.n_nodes]] if hasattr(low, "soff") else []
    ds[:, v_slots] = torch.randn(low.batch, len(v_slots), generator=gen, dtype=torch.float64).to(cuda_device)
    _, tan = sim.jvp(sim.model.pscale, torch.zeros_like(sim.model.pscale), n_steps=T, state_tangent=ds)

    def run_from(state0):
        m = sim.model
        m._state0 = state0.contiguous()
        try:
            return sim.run(n_steps=T, pscale=m.pscale)
        finally:
            m._state0 = None

    h = 1e-4
    fd = (run_from(s0 + h * ds) - run_from(s0 - h * ds)) / (2 * h)
    assert _rel(tan.cpu(), fd.cpu()) <= 1e-4


def _hh_cell(jx):
    from jaxley_pytorch.channels import HH

    cell = jx.Cell([jx.Branch(jx.Compartment(), 3)] * 3, parents=[-1, 0, 0])
    cell.insert(HH())
    cell.branch(1).comp(2).stimulate(jx.step_current(0.5, 1.0, 0.3, 0.025, 4.0), verbose=False)
    cell.branch(0).comp(0).record(verbose=False)
    cell.branch(2).comp(1).record(verbose=False)
    return cell


@pytest.mark.parametrize("api", ["func", "forward_ad"])
def test_integrate_entry_jvp_matches_reference(cuda_device, api):
    """The package's `integrate` under `torch.func.jvp` / `forward_ad` with per-branch
    `data_set` sodium conductances: the tangent is the reference's (CPU, float64), and
    agrees with the reverse mode through the same entry."""
    jx = import_reference()
    from jaxley_pytorch_b200.integrate import integrate

    cell = _hh_cell(jx)
    theta = torch.tensor([0.12, 0.10, 0.14], dtype=torch.float64)
    q = torch.randn(3, generator=torch.Generator().manual_seed(1), dtype=torch.float64)

    def simulate(fn, gna):
        pstate = None
        for b in range(3):
            pstate = cell.branch(b).data_set("HH_gNa", gna[b], pstate)
        return fn(cell, param_state=pstate, delta_t=0.025)

    ref_v, ref_t = torch.func.jvp(lambda g: simulate(jx.integrate, g), (theta,), (q,))
    th = theta.to(cuda_device)
    qd = q.to(cuda_device)
    if api == "func":
        v, t = torch.func.jvp(lambda g: simulate(integrate, g), (th,), (qd,))
    else:
        import torch.autograd.forward_ad as fwAD

        with fwAD.dual_level():
            v, t = fwAD.unpack_dual(simulate(integrate, fwAD.make_dual(th, qd)))
    assert v.shape == ref_v.shape and t.shape == ref_t.shape
    assert _rel(v.cpu(), ref_v.detach()) <= 1e-9
    assert _rel(t.cpu(), ref_t.detach()) <= 1e-7
    w = torch.randn(v.shape, generator=torch.Generator().manual_seed(2), dtype=torch.float64).to(cuda_device)
    leaf = th.clone().requires_grad_(True)
    (g,) = torch.autograd.grad((w * simulate(integrate, leaf)).sum(), leaf)
    np.testing.assert_allclose(float((w * t).sum()), float((g * qd).sum()), rtol=1e-9)
