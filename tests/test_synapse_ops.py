"""The synapse-step drop-in (jaxley_pytorch_b200.kernels.synapse_step) against the
oracle's restatement of the reference ops (kernels/synapse_step.py:121-330), as the
reference's tests/test_synapse_kernels.py:124-220 check its Triton kernels (float64
1e-9), including k = 150 (more synapses per target than one reference chunk), both
models, targets that are all nodes or a subset, and gradcheck of the custom op."""
import numpy as np
import pytest
import torch

import oracle
from jaxley_pytorch_b200.kernels import synapse_step as ss
from jaxley_pytorch_b200.lower import presynaptic_lists

pytestmark = pytest.mark.gpu

def close(got, ref, rel):
    """|got - ref| <= rel * max|ref| elementwise: the gradient terms carry a 1 / diff =
    1e3 scale with cancellation, so near-zero entries are compared at the scale of
    the array."""
    got, ref = np.asarray(got), np.asarray(ref)
    assert np.max(np.abs(got - ref)) <= rel * max(np.max(np.abs(ref)), 1e-300)


RANGES = {  # tests/test_synapse_kernels.py:25-29 style parameter ranges
    0: [(1e-4, 1e-3), (-80.0, 0.0), (0.5, 2.0), (0.05, 0.5), (-40.0, 0.0), (1.0, 4.0)],
    1: [(-1e-3, 1e-3), (-70.0, -40.0), (0.05, 0.5)],
}


def make(model, k, B, targets_are_nodes, seed=0):
    rng = np.random.default_rng(seed)
    n = 40 if not targets_are_nodes else 30
    T = n if targets_are_nodes else 17
    targets = np.arange(n) if targets_are_nodes else np.sort(rng.choice(n, T, replace=False))
    E = T * k
    pre = rng.integers(0, n, E)
    params = [rng.uniform(lo, hi, E) for lo, hi in RANGES[model]]
    area = rng.uniform(100.0, 500.0, E)
    v = rng.uniform(-80, 20, (B, n))
    s = rng.uniform(0, 1, (B, E)) if model == 0 else None
    return dict(n=n, T=T, E=E, k=k, targets=targets, pre=pre, params=params, area=area, v=v, s=s)


def torch_args(c, model, dev, dtype=torch.float64):
    t = lambda a: torch.as_tensor(a, dtype=dtype, device=dev)  # noqa: E731
    nodes, inv = presynaptic_lists(c["pre"])
    params = [t(p) for p in c["params"]] + [t(c["params"][0])] * (6 - len(c["params"]))
    return dict(
        v=t(c["v"]), s=t(c["s"]) if model == 0 else torch.empty(0, dtype=dtype, device=dev),
        pre=torch.as_tensor(c["pre"], dtype=torch.int32, device=dev),
        targets=torch.as_tensor(c["targets"], dtype=torch.int32, device=dev), params=params,
        area=t(c["area"]), scalars=ss.kernel_scalars(0.025, 1e-3, dtype, dev),
        inv=torch.as_tensor(inv, device=dev), nodes=torch.as_tensor(nodes, device=dev))


@pytest.mark.parametrize("model", [0, 1])
@pytest.mark.parametrize("k", [3, 64, 150])
@pytest.mark.parametrize("tan", [False, True])
def test_synapse_ops_match_oracle(cuda_device, model, k, tan):
    ss._ensure_ops()
    c = make(model, k, 5, tan, seed=k + model)
    a = torch_args(c, model, cuda_device)
    s_new, cur, lin, const = ss.synapse_step_op(a["v"], a["s"], a["pre"], a["targets"], *a["params"],
                                                a["area"], a["scalars"], a["inv"], a["nodes"], k,
                                                model, tan, True)
    r_s, r_i, r_lin, r_const = oracle.synapse_step(model, c["v"], c["s"], c["pre"], c["targets"], k,
                                                   c["params"], c["area"], 0.025, targets_are_nodes=tan)
    np.testing.assert_allclose(lin.cpu().numpy(), r_lin, rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(const.cpu().numpy(), r_const, rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(cur.cpu().numpy(), r_i, rtol=1e-12, atol=1e-15)
    if model == 0:
        np.testing.assert_allclose(s_new.cpu().numpy(), r_s, rtol=1e-12, atol=1e-15)
    # Backward op against the oracle's restatement of the reference backward kernel.
    rng = np.random.default_rng(1)
    B, T, E = 5, c["T"], c["E"]
    g_lin, g_const = rng.normal(size=(B, T)), rng.normal(size=(B, T))
    g_sn = rng.normal(size=(B, E)) if model == 0 else None
    g_cur = rng.normal(size=(B, E))
    need = (1 << len(c["params"])) - 1
    t = lambda x: torch.as_tensor(x, dtype=torch.float64, device=cuda_device)  # noqa: E731
    g_v, g_s, g_p = ss.synapse_step_backward_op(
        a["v"], a["s"], a["pre"], a["targets"], *a["params"], a["area"], a["scalars"], a["inv"],
        a["nodes"], t(g_sn) if model == 0 else t([]), t(g_cur), t(g_lin), t(g_const), k, model, tan,
        model == 0, True, need)
    r_gv, r_gs, r_gp = oracle.synapse_step_backward(model, c["v"], c["s"], c["pre"], c["targets"], k,
                                                    c["params"], c["area"], 0.025, g_sn, g_cur, g_lin,
                                                    g_const, targets_are_nodes=tan)
    # float64 rounding of terms amplified by 1 / diff = 1e3 with cancellation: 1e-8.
    close(g_v.cpu().numpy(), r_gv, 1e-8)
    for q in range(len(c["params"])):
        close(g_p[q].cpu().numpy(), r_gp[q], 1e-8)
    if model == 0:
        close(g_s.cpu().numpy(), r_gs, 1e-8)


def _reference_step_torch(model, v, s, pre, targets, k, params, area, dt, diff, tan):
    """Autograd restatement of the op's forward (modules/network.py:434-478 with the
    fused kernel's output convention), as tests/test_synapse_kernels.py:155-180."""
    vpre = v[:, pre]
    node = torch.arange(len(targets)) if tan else targets
    vp = torch.repeat_interleave(v[:, node], k, dim=1)
    gs = params[0]
    if model == 0:
        e_syn, alpha, beta, v_th, delta = params[1:6]
        tr = torch.sigmoid((vpre - v_th) / delta)
        a = alpha * tr
        rate = a + beta
        s_inf = a / rate
        s_new = s_inf + (s - s_inf) * torch.exp(-dt * rate)
        i0 = gs * s_new * (vp - e_syn)
        i1 = gs * s_new * ((vp + diff) - e_syn)
    else:
        x_off, slope = params[1:3]
        s_new = None
        i0 = -gs * torch.sigmoid((vpre - x_off) * slope)
        i1 = -gs * torch.sigmoid(((vpre + diff) - x_off) * slope)
    d0 = i0 / area * 100000.0
    d1 = i1 / area * 100000.0
    vt = (d1 - d0) / diff
    ct = d0 - vt * vp
    B = v.shape[0]
    return s_new, i0, vt.reshape(B, -1, k).sum(-1), ct.reshape(B, -1, k).sum(-1)


@pytest.mark.parametrize("model", [0, 1])
def test_synapse_op_autograd_matches_restatement(cuda_device, model):
    """Gradients through the custom op's autograd equal those of an autograd
    restatement of its forward (float64, 1e-8 at the scale of every gradient)."""
    ss._ensure_ops()
    c = make(model, 64, 4, False, seed=12)
    a = torch_args(c, model, cuda_device)
    npar = len(c["params"])
    rng = np.random.default_rng(2)
    B, T, E = 4, c["T"], c["E"]
    w = [torch.as_tensor(rng.normal(size=sh)) for sh in [(B, E), (B, E), (B, T), (B, T)]]

    def run(dev, use_op):
        t = lambda x: torch.as_tensor(x, dtype=torch.float64, device=dev)  # noqa: E731
        v = t(c["v"]).requires_grad_(True)
        s = t(c["s"]).requires_grad_(True) if model == 0 else t([])
        ps = [t(p).requires_grad_(True) for p in c["params"]]
        if use_op:
            full = ps + [ps[0].detach()] * (6 - npar)
            outs = ss.synapse_step_op(v, s, a["pre"], a["targets"], *full, a["area"], a["scalars"],
                                      a["inv"], a["nodes"], 64, model, False, True)
        else:
            outs = _reference_step_torch(model, v, s, torch.as_tensor(c["pre"]),
                                         torch.as_tensor(c["targets"]), 64, ps, t(c["area"]), 0.025,
                                         1e-3, False)
        loss = sum((o * wi.to(dev)).sum() for o, wi in zip(outs, w) if o is not None and o.numel())
        ins = [v] + ([s] if model == 0 else []) + ps
        return [g.detach().cpu().numpy() for g in torch.autograd.grad(loss, ins)]

    for g_op, g_ref in zip(run(cuda_device, True), run("cpu", False)):
        close(g_op, g_ref, 1e-8)
