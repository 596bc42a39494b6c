"""Generate the parity fixtures under tests/golden/ by running the reference.

Run with the path of a jaxley-pytorch source tree in JXB_REFERENCE:

    JXB_REFERENCE=<path to jaxley-pytorch> python tests/golden/make_fixtures.py [which ...]

The reference imports matplotlib at module level for plotting only; a stand-in
package (`tests/golden/_mpl_stub`) takes its place. Every fixture is an npz written by
`jaxley_pytorch_b200.problem.save_problem`: the lowered problem (reference node order)
plus `extra/ref` (the reference's `jx.integrate` output, float64), and for the golden
cases `extra/golden` (the values held by the reference's own tests).
"""
import ast
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REFERENCE = os.environ.get("JXB_REFERENCE")
if not REFERENCE:
    raise SystemExit("set JXB_REFERENCE to the path of a jaxley-pytorch source tree")
sys.path.insert(0, os.path.join(HERE, "_mpl_stub"))
sys.path.insert(0, REFERENCE)
sys.path.insert(0, REPO)

import numpy as np  # noqa: E402
import torch  # noqa: E402

torch.set_default_dtype(torch.float64)

import jaxley_pytorch as jx  # noqa: E402
from jaxley_pytorch.channels import HH  # noqa: E402
from jaxley_pytorch.channels.pospischil import Leak  # noqa: E402
from jaxley_pytorch.mech.channels.l5pc import (  # noqa: E402
    H, M, CaHVA, CaLVA, CaNernstReversal, CaPump, KPst, KTst, NapEt2, NaTaT, NaTs2T, SKE2, SKv3_1,
)
from jaxley_pytorch.synapses import KineticSynapse, SigmoidRateSynapse  # noqa: E402

from jaxley_pytorch_b200.problem import load_problem, problem_from_module, save_problem  # noqa: E402


def golden_arrays(test_file: str, func: str, var: str = "voltages_081123", index: int = 0) -> np.ndarray:
    """The `index`-th `var = np.asarray(<literal>)` of a test function of the
    reference (its golden trace), read from the source text."""
    tree = ast.parse(open(test_file).read())
    for node in ast.walk(tree):
        if isinstance(node, ast.FunctionDef) and node.name == func:
            found = [sub for sub in ast.walk(node)
                     if isinstance(sub, ast.Assign) and isinstance(sub.targets[0], ast.Name)
                     and sub.targets[0].id == var]
            found.sort(key=lambda sub: sub.lineno)
            call = found[index].value
            return np.asarray(ast.literal_eval(call.args[0]), dtype=np.float64)
    raise KeyError(func)


def save(name, module, **kw):
    extra = kw.pop("extra", {})
    ref = jx.integrate(module, **kw).detach().numpy()
    prob = problem_from_module(module, param_state=kw.get("param_state"),
                               t_max=kw.get("t_max"), delta_t=kw.get("delta_t", 0.025))
    path = os.path.join(HERE, f"{name}.npz")
    save_problem(prob, path, ref=ref, **extra)
    print(name, ref.shape, prob.n_nodes, "nodes", prob.batch, "rows")
    return prob, ref


def loss_weights(shape, seed):
    """Weights of the linear loss `sum(w * recordings)` whose gradient the fixtures
    hold (seeded; scaled so that the loss is of order one)."""
    rng = np.random.default_rng(seed)
    return rng.normal(size=shape) / np.sqrt(np.prod(shape))


def reference_grads(module, tensors, loss_w, **kw):
    """`(recordings, [d loss / d t for t in tensors])` of the reference's `jx.integrate`
    (autograd through its step and `_DHSSolve.backward`, solver_voltage.py:143-187)
    for the loss `sum(loss_w * recordings)`."""
    for t in tensors:
        t.requires_grad_(True)
    rec = jx.integrate(module, **kw)
    (rec * torch.as_tensor(loss_w)).sum().backward()
    return rec.detach().numpy(), [t.grad.detach().numpy().copy() for t in tensors]


def reference_jvp(module, params, seed, **kw):
    """`(directions, tangent)`: seeded directions for the trainable `params` and the
    reference's forward-mode derivative of its `jx.integrate` recordings along them
    (`torch.func.jvp`, through `_DHSSolveForwardAD`, solver_voltage.py:190-224)."""
    keys = [list(p.keys())[0] for p in params]
    vals = tuple(list(p.values())[0].detach().clone() for p in params)
    rng = np.random.default_rng(seed)
    dirs = tuple(torch.as_tensor(rng.normal(size=v.shape)) * v.abs().clamp_min(1e-3) for v in vals)

    def run(*xs):
        return jx.integrate(module, params=[{k: x} for k, x in zip(keys, xs)], **kw)

    _, tangent = torch.func.jvp(run, vals, dirs)
    return [d.numpy() for d in dirs], tangent.detach().numpy()


def save_with_grads(name, module, params, seed, extra=None, jvp=False, **kw):
    """A fixture of `module` with the reference's gradients with respect to the
    trainable `params` (entry q, group g -> `extra/grad_q`) of a linear loss, and with
    `jvp` its forward-mode derivative along seeded directions (`extra/jvp_dir_q`,
    `extra/jvp`)."""
    extra = dict(extra or {})
    probe = jx.integrate(module, params=params, **kw).detach().numpy()
    w = loss_weights(probe.shape, seed)
    if jvp:
        dirs, tangent = reference_jvp(module, params, seed + 1, **kw)
        for q, d in enumerate(dirs):
            extra[f"jvp_dir_{q}"] = d
        extra["jvp"] = tangent
    tensors = [list(p.values())[0] for p in params]
    ref, grads = reference_grads(module, tensors, w, params=params, **kw)
    prob = problem_from_module(module, params=params, param_state=kw.get("param_state"),
                               t_max=kw.get("t_max"), delta_t=kw.get("delta_t", 0.025),
                               data_clamps=kw.get("data_clamps"), data_stimuli=kw.get("data_stimuli"),
                               solver=kw.get("solver", "bwd_euler"))
    extra["loss_w"] = w
    extra["trainable_source"] = np.asarray(prob.trainable_source, dtype=np.int64).reshape(-1, 2)
    for q, g in enumerate(grads):
        extra[f"grad_{q}"] = g
    path = os.path.join(HERE, f"{name}.npz")
    save_problem(prob, path, ref=ref, **extra)
    print(name, ref.shape, prob.n_nodes, "nodes", prob.batch, "rows", len(params), "trainables")
    return prob, ref


def binary_parents(nbranches):
    """Branch parents of the reference's `SimpleCell` fixture (tests/conftest.py:24-31)."""
    parents = [-1]
    depth = 0
    while nbranches > len(parents):
        parents = [-1] + [b // 2 for b in range(0, 2**depth - 2)]
        depth += 1
    return parents[:nbranches]


def golden_cases():
    test_file = os.path.join(REFERENCE, "tests", "jaxley_identical", "test_basic_modules.py")
    current = jx.step_current(i_delay=0.5, i_dur=1.0, i_amp=0.02, delta_t=0.025, t_max=5.0)
    g = golden_arrays(test_file, "test_compartment")
    comp = jx.Compartment()
    comp.insert(HH())
    comp.record()
    comp.stimulate(current)
    save("golden_compartment", comp, delta_t=0.025, extra={"golden": g, "every": 20})
    cell = jx.Cell([jx.Branch([jx.Compartment()], )], parents=[-1])
    cell.insert(HH())
    cell.record()
    cell.stimulate(current)
    save("golden_cell_1comp", cell, delta_t=0.025, extra={"golden": g, "every": 20})
    net = jx.Network([jx.Cell([jx.Branch([jx.Compartment()])], parents=[-1])])
    net.insert(HH())
    net.record()
    net.stimulate(current)
    save("golden_net_1comp", net, delta_t=0.025, extra={"golden": g, "every": 20})
    g = golden_arrays(test_file, "test_branch")
    branch = jx.Branch([jx.Compartment()] * 2)
    branch.insert(HH())
    branch.loc(0.0).record()
    branch.loc(0.0).stimulate(current)
    save("golden_branch", branch, delta_t=0.025, extra={"golden": g, "every": 20})
    # test_cell: SimpleCell(3, 2) (branch parents of tests/conftest.py:24-31), HH
    g = golden_arrays(test_file, "test_cell", "voltages_300724")
    cell = jx.Cell([jx.Branch([jx.Compartment()] * 2)] * 3, parents=binary_parents(3))
    cell.insert(HH())
    cell.branch(1).loc(0.0).record()
    cell.branch(1).loc(0.0).stimulate(current)
    save("golden_cell_3x2", cell, delta_t=0.025, extra={"golden": g, "every": 20})
    # test_branch_uneven_radiuses, backward Euler (its second trace; tolerance 1e-5)
    g = golden_arrays(test_file, "test_branch_uneven_radiuses", "voltages_240920", index=1)
    current2 = jx.step_current(i_delay=0.5, i_dur=1.0, i_amp=2.0, delta_t=0.025, t_max=10.0)
    branch = jx.Branch([jx.Compartment()] * 8)
    branch.set("axial_resistivity", 500.0)
    branch.set("length", np.linspace(20, 300, 8))
    branch.set("radius", np.linspace(1, 5, 8))
    branch.insert(HH())
    branch.loc(1.0).stimulate(current2)
    branch.loc(0.0).record()
    save("golden_branch_uneven_radiuses", branch, delta_t=0.025,
         extra={"golden": g[None] if g.ndim == 1 else g, "every": 50, "tol": 1e-5})
    # tests/jaxley_identical/test_radius_and_length.py: the same inputs (numpy's
    # generator seeded with 1, as there) and its golden traces
    rl_file = os.path.join(REFERENCE, "tests", "jaxley_identical", "test_radius_and_length.py")
    g = golden_arrays(rl_file, "test_radius_and_length_compartment")
    comp = jx.Compartment()
    np.random.seed(1)
    comp.set("length", 5 * np.random.rand(1))
    comp.set("radius", np.random.rand(1))
    comp.insert(HH())
    comp.record()
    comp.stimulate(current)
    save("golden_radius_length_comp", comp, delta_t=0.025, extra={"golden": g, "every": 20})
    g = golden_arrays(rl_file, "test_radius_and_length_branch", "voltages_300724")
    branch = jx.Branch([jx.Compartment()] * 2)
    np.random.seed(1)
    branch.set("length", np.flip(5 * np.random.rand(2)))
    branch.set("radius", np.flip(np.random.rand(2)))
    branch.insert(HH())
    branch.loc(0.0).record()
    branch.loc(0.0).stimulate(current)
    save("golden_radius_length_branch", branch, delta_t=0.025, extra={"golden": g, "every": 20})
    g = golden_arrays(rl_file, "test_radius_and_length_cell", "voltages_300724")
    cell = jx.Cell([jx.Branch([jx.Compartment()] * 2)] * 3, parents=binary_parents(3))
    np.random.seed(1)
    rands1 = 5 * np.random.rand(6)
    rands2 = np.random.rand(6)
    for b in range(3):
        cell.branch(b).set("length", np.flip(rands1[2 * b:2 * b + 2]))
        cell.branch(b).set("radius", np.flip(rands2[2 * b:2 * b + 2]))
    cell.insert(HH())
    cell.branch(1).loc(0.0).record()
    cell.branch(1).loc(0.0).stimulate(current)
    save("golden_radius_length_cell", cell, delta_t=0.025, extra={"golden": g, "every": 20})


def config_small():
    """The plain-method small case: 1 branch x 8 compartments, HH, fp64."""
    cell = jx.Cell([jx.Branch(jx.Compartment(), 8)], parents=[-1])
    cell.set("length", 10.0)
    cell.set("radius", 1.0)
    cell.insert(HH())
    cell.branch(0).comp(0).record()
    cell.branch(0).comp(0).stimulate(jx.step_current(1.0, 1.0, 0.1, 0.025, 10.0))
    save("cell_8comp_hh", cell, delta_t=0.025)


def hh_tree():
    """A branched HH cell (15 branches x 3 compartments) with several recordings."""
    cell = jx.Cell([jx.Branch(jx.Compartment(), 3)] * 15, parents=binary_parents(15))
    cell.insert(HH())
    rng = np.random.default_rng(3)
    for b in range(15):
        cell.branch(b).set("radius", float(rng.uniform(0.5, 2.0)))
        cell.branch(b).set("length", float(rng.uniform(5.0, 40.0)))
    cell.branch(0).comp(0).record()
    cell.branch(7).comp(2).record()
    cell.branch(12).comp(1).record("HH_m")
    cell.branch(3).comp(0).record("i_HH")
    cell.branch(0).comp(0).stimulate(jx.step_current(1.0, 2.0, 0.3, 0.025, 15.0))
    cell.branch(9).comp(2).stimulate(jx.step_current(4.0, 2.0, 0.2, 0.025, 15.0))
    save("hh_tree_15x3", cell, delta_t=0.025)


def l5pc_cell():
    cell = jx.Cell([jx.Branch(jx.Compartment(), 4)] * 7, parents=[-1, 0, 0, 1, 1, 2, 2])
    b0 = lambda: cell.branch(0)  # noqa: E731 - views are rebuilt after every insert
    b0().insert(NaTs2T().change_name("somatic_NaTs2T"))
    b0().insert(SKv3_1().change_name("somatic_SKv3_1"))
    b0().insert(SKE2().change_name("somatic_SKE2"))
    ca = CaNernstReversal()
    ca.channel_constants["T"] = 307.15
    b0().insert(ca)
    b0().insert(CaPump().change_name("somatic_CaPump"))
    b0().insert(CaHVA().change_name("somatic_CaHVA"))
    b0().insert(CaLVA().change_name("somatic_CaLVA"))
    b0().set("CaCon_i", 5e-05)
    b0().set("CaCon_e", 2.0)
    for b in range(1, 7):
        cell.branch(b).insert(NaTs2T().change_name("apical_NaTs2T"))
        cell.branch(b).insert(SKv3_1().change_name("apical_SKv3_1"))
        cell.branch(b).insert(M().change_name("apical_M"))
        cell.branch(b).insert(H().change_name("apical_H"))
    for b in (5, 6):
        cell.branch(b).insert(NaTaT().change_name("axonal_NaTaT"))
        cell.branch(b).insert(KTst().change_name("axonal_KTst"))
        cell.branch(b).insert(KPst().change_name("axonal_KPst"))
        cell.branch(b).insert(NapEt2().change_name("axonal_NapEt2"))
    cell.insert(Leak())
    cell.set("Leak_gLeak", 3e-05)
    cell.set("Leak_eLeak", -75.0)
    cell.set("eNa", 50.0)
    cell.set("eK", -85.0)
    cell.set("v", -65.0)
    for key, val in [
        ("somatic_NaTs2T_gNaTs2T", 0.983955), ("somatic_SKv3_1_gSKv3_1", 0.303472),
        ("somatic_SKE2_gSKE2", 0.008407), ("somatic_CaHVA_gCaHVA", 0.000994),
        ("somatic_CaLVA_gCaLVA", 0.000333), ("somatic_CaPump_gamma", 0.000609),
        ("somatic_CaPump_decay", 210.485291), ("apical_NaTs2T_gNaTs2T", 0.026145),
        ("apical_SKv3_1_gSKv3_1", 0.004226), ("apical_M_gM", 0.000143), ("apical_H_gH", 8e-5),
        ("axonal_NaTaT_gNaTaT", 0.01), ("axonal_KTst_gKTst", 0.01), ("axonal_KPst_gKPst", 0.01),
        ("axonal_NapEt2_gNapEt2", 0.001),
    ]:
        cell.set(key, val)
    cell.branch(0).loc(0.0).record()
    cell.branch(0).loc(0.0).record("CaCon_i")
    cell.branch(0).loc(0.0).record("eCa")
    cell.branch(4).loc(1.0).record()
    cell.branch(0).loc(0.0).record("i_Ca")
    cell.branch(6).loc(0.5).record("axonal_NapEt2_h")
    cell.branch(0).loc(0.0).stimulate(jx.step_current(2.0, 20.0, 1.0, 0.025, 30.0))
    cell.init_states()
    save("l5pc_7x4", cell, delta_t=0.025)
    # Batched conductances (data_set with a batch dimension).
    pstate = cell.branch(0).data_set("somatic_NaTs2T_gNaTs2T", torch.tensor([[0.9], [1.1], [0.5]]), None)
    pstate = cell.branch(1).data_set("apical_M_gM", torch.tensor([[1e-4], [2e-4], [3e-4]]), pstate)
    pstate = cell.branch(2).data_set("apical_H_gH", torch.tensor([[5e-5], [8e-5], [1.2e-4]]), pstate)
    # Trainables (shared over the batch): the reference's gradients pin the adjoint.
    cell.branch(0).make_trainable("somatic_SKv3_1_gSKv3_1", verbose=False)
    cell.branch(0).make_trainable("somatic_CaHVA_gCaHVA", verbose=False)
    cell.make_trainable("apical_NaTs2T_gNaTs2T", verbose=False)
    cell.make_trainable("Leak_gLeak", verbose=False)
    cell.branch(5).make_trainable("axonal_KTst_gKTst", verbose=False)
    cell.branch("all").make_trainable("apical_SKv3_1_gSKv3_1", verbose=False)
    save_with_grads("l5pc_7x4_batch3", cell, cell.get_parameters(), seed=21, param_state=pstate,
                    delta_t=0.025, t_max=15.0)


def hh_forest():
    """A network of unconnected cells of uneven size and depth."""
    rng = np.random.default_rng(5)
    cells = []
    for c in range(6):
        nb = int(rng.integers(1, 12))
        parents = [-1] + [int(rng.integers(0, b)) for b in range(1, nb)]
        ncomp = int(rng.integers(1, 5))
        cells.append(jx.Cell([jx.Branch(jx.Compartment(), ncomp)] * nb, parents=parents))
    net = jx.Network(cells)
    net.insert(HH())
    for c in range(6):
        net.cell(c).branch(0).comp(0).record()
        net.cell(c).branch(0).comp(0).stimulate(
            jx.step_current(float(rng.uniform(1, 3)), 2.0, float(rng.uniform(0.05, 0.5)), 0.025, 12.0)
        )
    save("hh_forest_6", net, delta_t=0.025)


def synapse_net():
    """HH point-like cells coupled by Kinetic and SigmoidRate synapses in the regular
    layout (sorted by target, equal in-degree)."""
    rng = np.random.default_rng(7)
    n = 8
    cells = [jx.Cell([jx.Branch(jx.Compartment(), 2)], parents=[-1]) for _ in range(n)]
    net = jx.Network(cells)
    net.insert(HH())
    k = 3
    for post in range(n):
        pres = rng.choice([c for c in range(n) if c != post], size=k, replace=False)
        for pre in sorted(pres):
            jx.connect(net.cell(int(pre)).branch(0).comp(0), net.cell(post).branch(0).comp(0),
                       KineticSynapse())
    for post in range(n):
        pres = rng.choice([c for c in range(n) if c != post], size=k, replace=False)
        for pre in sorted(pres):
            jx.connect(net.cell(int(pre)).branch(0).comp(1), net.cell(post).branch(0).comp(0),
                       SigmoidRateSynapse())
    net.set("KineticSynapse_gS", rng.uniform(0, 1e-3, size=n * k))
    net.set("SigmoidRateSynapse_gS", rng.uniform(0, 1e-3, size=n * k))
    for c in range(n):
        net.cell(c).branch(0).comp(0).record()
    for c in range(0, n, 2):
        net.cell(c).branch(0).comp(1).stimulate(jx.step_current(1.0, 3.0, 0.3, 0.025, 15.0))
    save("synapse_net_8", net, delta_t=0.025)
    # The reference's gradients of a linear loss with respect to every synapse's gS
    # (per synapse, `edges` order) and the shared HH_gNa of all cells.
    probe = jx.integrate(net, delta_t=0.025).detach().numpy()
    w = loss_weights(probe.shape, 31)
    edges = net.edges
    gs = {}
    for syn in ("KineticSynapse", "SigmoidRateSynapse"):
        sel = edges[edges.type == syn]
        gs[syn] = torch.tensor(sel[f"{syn}_gS"].to_numpy(), dtype=torch.float64, requires_grad=True)
    # (data_set broadcasts its value: the leaves must require gradients before it)
    gna = torch.tensor([float(net.nodes["HH_gNa"].iloc[0])], dtype=torch.float64, requires_grad=True)
    pstate = None
    for syn, vals in gs.items():
        pstate = net.select(edges=edges.index[edges.type == syn].to_numpy()).data_set(f"{syn}_gS", vals, pstate)
    pstate = net.data_set("HH_gNa", gna, pstate)
    _, grads = reference_grads(net, [gs["KineticSynapse"], gs["SigmoidRateSynapse"], gna], w,
                               param_state=pstate, delta_t=0.025)
    prob, extra = load_problem(os.path.join(HERE, "synapse_net_8.npz"))
    extra = {k: v for k, v in extra.items() if not k.startswith("grad_")}
    extra.update(loss_w=w, grad_0=grads[0], grad_1=grads[1], grad_2=grads[2])
    save_problem(prob, os.path.join(HERE, "synapse_net_8.npz"), **extra)
    print("synapse_net_8 gradients", [g.shape for g in grads])


def clamp_cell():
    """A branched HH cell with a voltage clamp on one compartment and a gate clamp
    on another (Module.clamp, modules/base.py:2607), with the reference's gradients."""
    cell = jx.Cell([jx.Branch(jx.Compartment(), 3)] * 7, parents=binary_parents(7))
    cell.insert(HH())
    rng = np.random.default_rng(13)
    for b in range(7):
        cell.branch(b).set("radius", float(rng.uniform(0.5, 2.0)))
        cell.branch(b).set("length", float(rng.uniform(5.0, 40.0)))
    T = 401
    t = np.arange(T) * 0.025
    vc = np.where((t >= 2.0) & (t < 6.0), -20.0, -70.0)
    cell.branch(3).comp(1).clamp("v", vc, verbose=False)
    cell.branch(5).comp(0).clamp("HH_m", np.full(T, 0.3), verbose=False)
    cell.branch(0).comp(0).record()
    cell.branch(3).comp(1).record()
    cell.branch(3).comp(2).record()
    cell.branch(5).comp(0).record("HH_m")
    cell.branch(6).comp(2).record()
    cell.branch(0).comp(0).stimulate(jx.step_current(1.0, 2.0, 0.05, 0.025, 10.0))
    cell.make_trainable("HH_gNa", verbose=False)
    cell.branch(3).make_trainable("HH_gK", verbose=False)
    cell.branch("all").make_trainable("HH_gLeak", verbose=False)
    save_with_grads("hh_clamp_7x3", cell, cell.get_parameters(), seed=41, delta_t=0.025, jvp=True)


def pospischil_cell():
    """A branched cell with the Pospischil channels (channels/pospischil.py: Na, K, Km,
    CaL, CaT, Leak), a regular-spiking and a fast-spiking region, two stimuli, and
    the reference's gradients with respect to conductances, the shared threshold vt,
    Km's taumax and CaT's vx."""
    from jaxley_pytorch.channels.pospischil import CaL, CaT, K, Km, Na

    cell = jx.Cell([jx.Branch(jx.Compartment(), 3)] * 7, parents=binary_parents(7))
    rng = np.random.default_rng(17)
    for b in range(7):
        cell.branch(b).set("radius", float(rng.uniform(0.5, 2.0)))
        cell.branch(b).set("length", float(rng.uniform(5.0, 40.0)))
    cell.insert(Na())
    cell.insert(K())
    cell.insert(Leak())
    rs = cell.branch([0, 1, 3, 4])
    rs.insert(Km())
    cell.branch([0, 2, 5]).insert(CaL())
    cell.branch([0, 2, 6]).insert(CaT())
    cell.set("Na_gNa", 5e-2)
    cell.set("vt", -60.0)
    cell.set("Leak_eLeak", -70.0)
    cell.branch([0, 1, 3, 4]).set("K_gK", 5e-3)
    cell.branch([2, 5, 6]).set("K_gK", 1e-2)
    cell.branch([0, 1, 3, 4]).set("Km_gKm", 7e-5)
    cell.branch([0, 1, 3, 4]).set("Km_taumax", 1000.0)
    cell.branch([0, 2, 5]).set("CaL_gCaL", 2e-4)
    cell.branch([0, 2, 6]).set("CaT_gCaT", 4e-4)
    cell.set("v", -70.0)
    cell.init_states()
    cell.branch(0).comp(0).record(verbose=False)
    cell.branch(4).comp(2).record(verbose=False)
    cell.branch(6).comp(1).record(verbose=False)
    cell.branch(0).comp(0).record("Na_m", verbose=False)
    cell.branch(2).comp(1).record("i_Ca", verbose=False)
    cell.branch(6).comp(0).record("CaT_u", verbose=False)
    cell.branch(0).comp(0).stimulate(jx.step_current(1.0, 4.0, 0.15, 0.025, 12.0), verbose=False)
    cell.branch(5).comp(2).stimulate(jx.step_current(3.0, 3.0, 0.1, 0.025, 12.0), verbose=False)
    cell.make_trainable("Na_gNa", verbose=False)
    cell.make_trainable("vt", verbose=False)
    cell.branch([0, 1, 3, 4]).make_trainable("Km_taumax", verbose=False)
    cell.branch("all").make_trainable("K_gK", verbose=False)
    cell.make_trainable("CaT_vx", verbose=False)
    cell.make_trainable("CaT_gCaT", verbose=False)
    cell.make_trainable("CaL_gCaL", verbose=False)
    save_with_grads("pospischil_7x3", cell, cell.get_parameters(), seed=81, delta_t=0.025, jvp=True)


def crank_nicolson():
    """A branched HH cell with a voltage clamp, stepped with Crank-Nicolson
    (`solver="crank_nicolson"`, modules/base.py:3327-3365), with the reference's
    gradients."""
    cell = jx.Cell([jx.Branch(jx.Compartment(), 3)] * 7, parents=binary_parents(7))
    cell.insert(HH())
    rng = np.random.default_rng(23)
    for b in range(7):
        cell.branch(b).set("radius", float(rng.uniform(0.5, 2.0)))
        cell.branch(b).set("length", float(rng.uniform(5.0, 40.0)))
    T = 321
    t = np.arange(T) * 0.025
    cell.branch(4).comp(1).clamp("v", np.where((t >= 2.0) & (t < 5.0), -30.0, -70.0), verbose=False)
    cell.branch(0).comp(0).record(verbose=False)
    cell.branch(4).comp(2).record(verbose=False)
    cell.branch(6).comp(2).record("HH_n", verbose=False)
    cell.branch(0).comp(0).stimulate(jx.step_current(1.0, 2.0, 0.3, 0.025, 8.0), verbose=False)
    cell.make_trainable("HH_gNa", verbose=False)
    cell.branch("all").make_trainable("HH_gK", verbose=False)
    save_with_grads("cn_hh_7x3", cell, cell.get_parameters(), seed=91, delta_t=0.025, jvp=True,
                    solver="crank_nicolson")


def reference_l5pc_cell(parents, ncomp, radius, lengths):
    from jaxley_pytorch_b200 import synth

    return synth.reference_l5pc_cell(jx, parents, ncomp, radius, lengths)


def c2_sample():
    """The large-batch L5PC tree (300 branches x 4 compartments, height 35-45) at 2
    parameter sets and 400 steps, stimulus from 1 ms, rebuilt with the reference from
    the generator's morphology; gradients with respect to the per-row conductances."""
    from jaxley_pytorch_b200 import synth

    B, T = 2, 400
    prob = synth.config_l5pc_tree(batch=B, n_steps=T, stim_delay=1.0)
    m = prob.meta
    cell = reference_l5pc_cell(m["parents"], m["ncomp"], m["radius"], m["lengths"])
    cell.init_states()
    cell.branch(0).loc(0.0).record()
    delay, dur, amp = m["stim"]
    t_max = (T - 1) * 0.025
    cell.branch(0).loc(0.0).stimulate(jx.step_current(delay, dur, amp, 0.025, T * 0.025))
    soma_vals = {k: v for _, _, d in synth.L5PC_SOMA for k, v in d.items() if k != "__constants__"}
    dend_vals = {k: v for _, _, d in synth.L5PC_DEND for k, v in d.items()}
    nb = len(m["parents"])
    pstate, tensors = None, []
    for k in synth.L5PC_SCALED:
        vals = torch.tensor(m["scales"][k])[:, None]
        # (data_set broadcasts its value: the leaf must require gradients before it)
        if k in soma_vals:
            val = (vals * soma_vals[k]).requires_grad_(True)
            pstate = cell.branch(0).data_set(k, val, pstate)
        elif k in dend_vals:
            val = (vals * dend_vals[k]).requires_grad_(True)
            pstate = cell.branch(list(range(1, nb))).data_set(k, val, pstate)
        else:
            val = (vals * 3e-05).requires_grad_(True)
            pstate = cell.data_set(k, val, pstate)
        tensors.append(val)
    probe = jx.integrate(cell, param_state=pstate, delta_t=0.025, t_max=t_max).detach().numpy()
    assert probe.shape[-1] == T + 1, probe.shape
    w = loss_weights(probe.shape, 51)
    ref, grads = reference_grads(cell, tensors, w, param_state=pstate, delta_t=0.025, t_max=t_max)
    extra = {"init_steady": 1, "loss_w": w, "height": m["height"],
             "grad_names": np.frombuffer(",".join(synth.L5PC_SCALED).encode(), dtype=np.uint8)}
    for q, g in enumerate(grads):
        extra[f"grad_{q}"] = g
    save_problem(prob, os.path.join(HERE, "c2_l5pc_tree_b2.npz"), ref=ref, **extra)
    print("c2_l5pc_tree_b2", ref.shape, prob.n_nodes, "nodes, height", m["height"])


def c3_sample():
    """The first 8 cells of the uneven batch (HH or L5PC, 4-3000 compartments, depth
    1-60, own step currents), 200 steps, as one reference network; gradients with
    respect to every cell's trainable conductances."""
    from jaxley_pytorch_b200 import synth

    T = 200
    prob = synth.config_uneven(n_cells=8, n_steps=T, seed=0)
    cells = []
    for spec in prob.meta["cells"]:
        if spec["kind"] == "L5PC":
            c = reference_l5pc_cell(spec["parents"], spec["ncomp"], spec["radius"], spec["lengths"])
        else:
            nb = len(spec["parents"])
            c = jx.Cell([jx.Branch(jx.Compartment(), spec["ncomp"])] * nb, parents=list(spec["parents"]))
            for b in range(nb):
                c.branch(b).set("radius", float(spec["radius"][b]))
                c.branch(b).set("length", float(spec["lengths"][b] / spec["ncomp"]))
            c.set("axial_resistivity", 100.0)
            c.insert(HH())
            c.set("v", -65.0)
        cells.append(c)
    net = jx.Network(cells)
    net.init_states()
    for ci, spec in enumerate(prob.meta["cells"]):
        net.cell(ci).branch(0).comp(0).record()
        delay, dur, amp = spec["stim"]
        net.cell(ci).branch(0).comp(0).stimulate(jx.step_current(delay, dur, amp, 0.025, T * 0.025))
    for ci, spec in enumerate(prob.meta["cells"]):
        for k in spec["train"]:
            net.cell(ci).make_trainable(k, verbose=False)
    params = net.get_parameters()
    assert len(params) == len(prob.trainable)
    t_max = (T - 1) * 0.025
    probe = jx.integrate(net, params=params, delta_t=0.025, t_max=t_max).detach().numpy()
    assert probe.shape[-1] == T + 1, probe.shape
    w = loss_weights(probe.shape, 61)
    tensors = [list(p.values())[0] for p in params]
    ref, grads = reference_grads(net, tensors, w, params=params, delta_t=0.025, t_max=t_max)
    extra = {"init_steady": 1, "loss_w": w}
    for q, g in enumerate(grads):
        extra[f"grad_{q}"] = g
    save_problem(prob, os.path.join(HERE, "c3_uneven_8.npz"), ref=ref, **extra)
    print("c3_uneven_8", ref.shape, prob.n_nodes, "nodes", [s["kind"] for s in prob.meta["cells"]])


def c4_sample():
    """The fixed in-degree network (HH cells of 4 compartments, 64 KineticSynapse and
    64 SigmoidRateSynapse inputs on compartment 0 of every cell, Poisson input) at 72
    cells, 4 batch rows and 200 steps, built with the reference; gradients with respect
    to every synapse's gS and the shared HH_gNa."""
    from jaxley_pytorch.synapses import KineticSynapse, SigmoidRateSynapse
    from jaxley_pytorch_b200.network import config_network

    n, k, B, T = 72, 64, 4, 200
    prob = config_network(n_cells=n, k=k, batch=B, n_steps=T, seed=3)
    cells = [jx.Cell([jx.Branch(jx.Compartment(), 4)], parents=[-1]) for _ in range(n)]
    net = jx.Network(cells)
    net.insert(HH())
    net.set("v", -65.0)
    nodes = net.nodes
    for syn, cls in zip(prob.synapses, (KineticSynapse, SigmoidRateSynapse)):
        net._append_multiple_synapses(nodes.loc[syn.pre], nodes.loc[syn.post], cls())
    edges = net.edges
    for syn in prob.synapses:
        sel = edges.index[edges.type == syn.name].to_numpy()
        assert np.array_equal(edges.loc[sel, "pre_index"].to_numpy(), syn.pre)
        assert np.array_equal(edges.loc[sel, "post_index"].to_numpy(), syn.post)
        net.select(edges=sel).set(f"{syn.name}_gS", syn.params[0])
    for c in range(n):
        net.cell(c).branch(0).comp(0).record()
    t_max = (T - 1) * 0.025
    stim = torch.as_tensor(prob.stim)  # (B, n, L)
    data_stimuli = net.cell(list(range(n))).branch(0).comp(0).data_stimulate(stim)
    gs = [torch.tensor(s.params[0], dtype=torch.float64, requires_grad=True) for s in prob.synapses]
    gna = torch.tensor([0.12], dtype=torch.float64, requires_grad=True)
    pstate = None
    for syn, vals in zip(prob.synapses, gs):
        sel = edges.index[edges.type == syn.name].to_numpy()
        pstate = net.select(edges=sel).data_set(f"{syn.name}_gS", vals, pstate)
    pstate = net.data_set("HH_gNa", gna, pstate)
    kw = dict(param_state=pstate, data_stimuli=data_stimuli, delta_t=0.025, t_max=t_max)
    probe = jx.integrate(net, **kw).detach().numpy()
    assert probe.shape == (B, n, T + 1), probe.shape
    w = loss_weights(probe.shape, 71)
    ref, grads = reference_grads(net, gs + [gna], w, **kw)
    prob.trainable = [("HH_gNa", np.arange(prob.n_nodes))]
    extra = {"loss_w": w, "grad_0": grads[0], "grad_1": grads[1], "grad_2": grads[2]}
    save_problem(prob, os.path.join(HERE, "c4_network_72.npz"), ref=ref, **extra)
    print("c4_network_72", ref.shape, prob.n_nodes, "nodes", sum(len(s.pre) for s in prob.synapses), "synapses")


if __name__ == "__main__":
    which = [w for w in sys.argv[1:] if w != "synth"] if sys.argv[1:] else [
        "golden", "small", "tree", "l5pc", "forest", "synapse", "clamp", "pospischil", "cn", "c2", "c3", "c4",
        "synth"]
    fns = {"golden": golden_cases, "small": config_small, "tree": hh_tree, "l5pc": l5pc_cell,
           "forest": hh_forest, "synapse": synapse_net, "clamp": clamp_cell, "pospischil": pospischil_cell, "cn": crank_nicolson,
           "c2": c2_sample,
           "c3": c3_sample, "c4": c4_sample}
    for w in which:
        if w in fns:
            fns[w]()


def synth_check():
    """A small tree from `jaxley_pytorch_b200.synth` rebuilt with the reference's own
    `jx.Cell`: checks the synthetic morphology, conductances and channel setup."""
    from jaxley_pytorch_b200 import synth

    nb, ncomp, B = 15, 4, 2
    rng = np.random.default_rng(11)
    parents = synth.balanced_random_tree(nb, rng)
    lengths = rng.lognormal(np.log(30.0), 0.5, size=nb)
    depth = np.zeros(nb, dtype=np.int64)
    for b in range(1, nb):
        depth[b] = depth[parents[b]] + 1
    radius = 2.0 - (2.0 - 0.3) * depth / max(int(depth.max()), 1)
    cellm = synth.morphology(parents, [ncomp] * nb, [np.full(ncomp, r) for r in radius],
                             [np.full(ncomp, L / ncomp) for L in lengths], r_a=100.0)
    scales = {k: np.linspace(0.6, 1.4, B) for k in synth.L5PC_SCALED}
    chans = synth.l5pc_channels(cellm, scales, ncomp_soma=ncomp)
    n_steps = 600
    prob = synth.assemble([cellm], [chans], batch=B, dt=0.025, n_steps=n_steps, v0=-65.0,
                          stim=[(0, (0, 0), synth.step_current(2.0, 10.0, 0.3, 0.025, n_steps * 0.025))],
                          recordings=[("v", 0, (0, 0)), ("v", 0, (nb - 1, 3))])
    for k in ["eNa", "eK"]:
        prob.params[k] = np.full(prob.n_nodes, 50.0 if k == "eNa" else -85.0)

    cell = jx.Cell([jx.Branch(jx.Compartment(), ncomp)] * nb, parents=parents)
    for b in range(nb):
        cell.branch(b).set("radius", float(radius[b]))
        cell.branch(b).set("length", float(lengths[b] / ncomp))
    cell.set("axial_resistivity", 100.0)
    classes = {"NaTs2T": NaTs2T, "SKv3_1": SKv3_1, "SKE2": SKE2, "CaPump": CaPump, "CaHVA": CaHVA,
               "CaLVA": CaLVA, "M": M, "H": H}
    for t, name, vals in synth.L5PC_SOMA:
        if t == "CaNernstReversal":
            ch = CaNernstReversal()
            ch.channel_constants["T"] = 307.15
        else:
            ch = classes[t]().change_name(name)
        cell.branch(0).insert(ch)
    cell.branch(0).set("CaCon_i", 5e-05)
    cell.branch(0).set("CaCon_e", 2.0)
    for b in range(1, nb):
        for t, name, vals in synth.L5PC_DEND:
            cell.branch(b).insert(classes[t]().change_name(name))
    cell.insert(Leak())
    for t, name, vals in synth.L5PC_SOMA + synth.L5PC_DEND + [("Leak", "Leak", {"Leak_gLeak": 3e-05, "Leak_eLeak": -75.0})]:
        for k, v in vals.items():
            if k != "__constants__":
                cell.set(k, v)
    cell.set("eNa", 50.0)
    cell.set("eK", -85.0)
    cell.set("v", -65.0)
    cell.init_states()
    cell.branch(0).loc(0.0).record()
    cell.branch(nb - 1).comp(3).record()
    cell.branch(0).loc(0.0).stimulate(jx.step_current(2.0, 10.0, 0.3, 0.025, n_steps * 0.025))
    pstate = None
    soma_vals = {k: v for _, _, d in synth.L5PC_SOMA for k, v in d.items() if k != "__constants__"}
    dend_vals = {k: v for _, _, d in synth.L5PC_DEND for k, v in d.items()}
    for k in synth.L5PC_SCALED:
        vals = torch.tensor(scales[k])[:, None]
        if k in soma_vals:
            pstate = cell.branch(0).data_set(k, vals * soma_vals[k], pstate)
        elif k in dend_vals:
            view = cell.branch(list(range(1, nb)))
            pstate = view.data_set(k, vals * dend_vals[k], pstate)
        else:
            pstate = cell.data_set(k, vals * 3e-05, pstate)
    ref = jx.integrate(cell, param_state=pstate, delta_t=0.025, t_max=(n_steps - 1) * 0.025).detach().numpy()
    path = os.path.join(HERE, "synth_l5pc_15x4.npz")
    save_problem(prob, path, ref=ref, init_steady=1)
    print("synth_l5pc_15x4", ref.shape, prob.n_nodes)


if __name__ == "__main__" and "synth" in sys.argv[1:]:
    synth_check()
