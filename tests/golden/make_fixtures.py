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

from jaxley_pytorch_b200.problem import problem_from_module, save_problem  # noqa: E402


def golden_arrays(test_file: str, func: str) -> np.ndarray:
    """The `voltages_081123` literal of a test function of the reference."""
    tree = ast.parse(open(test_file).read())
    for node in ast.walk(tree):
        if isinstance(node, ast.FunctionDef) and node.name == func:
            for sub in ast.walk(node):
                if (isinstance(sub, ast.Assign) and isinstance(sub.targets[0], ast.Name)
                        and sub.targets[0].id == "voltages_081123"):
                    call = sub.value
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
    save("l5pc_7x4_batch3", cell, param_state=pstate, delta_t=0.025, t_max=15.0)


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


if __name__ == "__main__":
    which = [w for w in sys.argv[1:] if w != "synth"] if sys.argv[1:] else ["golden", "small", "tree", "l5pc", "forest", "synapse", "synth"]
    fns = {"golden": golden_cases, "small": config_small, "tree": hh_tree, "l5pc": l5pc_cell,
           "forest": hh_forest, "synapse": synapse_net}
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
