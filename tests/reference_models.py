"""Small models built with the reference's own module API (jaxley-pytorch), for the
drop-in tests. Each builder takes the imported `jaxley_pytorch` package and returns
`(module, kwargs of integrate)`; trainables are made with `make_trainable` and
returned by `module.get_parameters()`."""
import numpy as np


def hh_tree(jx):
    """A branched HH cell (15 branches x 3 compartments) with two stimuli and
    trainable sodium (one value) and potassium (one per branch) conductances."""
    from jaxley_pytorch.channels import HH

    parents = [-1, 0, 0, 1, 1, 2, 2, 3, 3, 4, 4, 5, 5, 6, 6]
    cell = jx.Cell([jx.Branch(jx.Compartment(), 3)] * 15, parents=parents)
    cell.insert(HH())
    rng = np.random.default_rng(3)
    for b in range(15):
        cell.branch(b).set("radius", float(rng.uniform(0.5, 2.0)))
        cell.branch(b).set("length", float(rng.uniform(5.0, 40.0)))
    cell.branch(0).comp(0).record(verbose=False)
    cell.branch(7).comp(2).record(verbose=False)
    cell.branch(12).comp(1).record("HH_m", verbose=False)
    cell.branch(0).comp(0).stimulate(jx.step_current(1.0, 2.0, 0.3, 0.025, 8.0), verbose=False)
    cell.branch(9).comp(2).stimulate(jx.step_current(4.0, 2.0, 0.2, 0.025, 8.0), verbose=False)
    cell.make_trainable("HH_gNa", verbose=False)
    cell.branch("all").make_trainable("HH_gK", verbose=False)
    return cell, {"delta_t": 0.025}


def l5pc_cell(jx):
    """Seven branches of four compartments with the somatic, apical and axonal L5PC
    channel sets (every mechanism of mech/channels/l5pc.py), a trainable somatic and
    a trainable apical conductance."""
    from jaxley_pytorch.channels.pospischil import Leak
    from jaxley_pytorch.mech.channels.l5pc import (
        H, M, CaHVA, CaLVA, CaNernstReversal, CaPump, KPst, KTst, NapEt2, NaTaT, NaTs2T, SKE2, SKv3_1,
    )

    cell = jx.Cell([jx.Branch(jx.Compartment(), 4)] * 7, parents=[-1, 0, 0, 1, 1, 2, 2])
    for ch in [NaTs2T().change_name("somatic_NaTs2T"), SKv3_1().change_name("somatic_SKv3_1"),
               SKE2().change_name("somatic_SKE2")]:
        cell.branch(0).insert(ch)
    ca = CaNernstReversal()
    ca.channel_constants["T"] = 307.15
    cell.branch(0).insert(ca)
    cell.branch(0).insert(CaPump().change_name("somatic_CaPump"))
    cell.branch(0).insert(CaHVA().change_name("somatic_CaHVA"))
    cell.branch(0).insert(CaLVA().change_name("somatic_CaLVA"))
    cell.branch(0).set("CaCon_i", 5e-05)
    cell.branch(0).set("CaCon_e", 2.0)
    for b in range(1, 7):
        for ch in [NaTs2T().change_name("apical_NaTs2T"), SKv3_1().change_name("apical_SKv3_1"),
                   M().change_name("apical_M"), H().change_name("apical_H")]:
            cell.branch(b).insert(ch)
    for b in (5, 6):
        for ch in [NaTaT().change_name("axonal_NaTaT"), KTst().change_name("axonal_KTst"),
                   KPst().change_name("axonal_KPst"), NapEt2().change_name("axonal_NapEt2")]:
            cell.branch(b).insert(ch)
    cell.insert(Leak())
    for key, val in [("Leak_gLeak", 3e-05), ("Leak_eLeak", -75.0), ("eNa", 50.0), ("eK", -85.0),
                     ("v", -65.0), ("somatic_NaTs2T_gNaTs2T", 0.983955),
                     ("somatic_SKv3_1_gSKv3_1", 0.303472), ("somatic_SKE2_gSKE2", 0.008407),
                     ("somatic_CaHVA_gCaHVA", 0.000994), ("somatic_CaLVA_gCaLVA", 0.000333),
                     ("somatic_CaPump_gamma", 0.000609), ("somatic_CaPump_decay", 210.485291),
                     ("apical_NaTs2T_gNaTs2T", 0.026145), ("apical_SKv3_1_gSKv3_1", 0.004226),
                     ("apical_M_gM", 0.000143), ("apical_H_gH", 8e-5), ("axonal_NaTaT_gNaTaT", 0.01),
                     ("axonal_KTst_gKTst", 0.01), ("axonal_KPst_gKPst", 0.01),
                     ("axonal_NapEt2_gNapEt2", 0.001)]:
        cell.set(key, val)
    cell.init_states()
    cell.branch(0).loc(0.0).record(verbose=False)
    cell.branch(0).loc(0.0).record("CaCon_i", verbose=False)
    cell.branch(4).loc(1.0).record(verbose=False)
    cell.branch(0).loc(0.0).stimulate(jx.step_current(2.0, 5.0, 1.0, 0.025, 10.0), verbose=False)
    cell.branch(0).make_trainable("somatic_SKv3_1_gSKv3_1", verbose=False)
    cell.make_trainable("apical_NaTs2T_gNaTs2T", verbose=False)
    return cell, {"delta_t": 0.025}


def clamped_cell(jx, torch):
    """An HH cell of 7 x 3 compartments with a voltage clamp and a gate clamp given as
    `data_clamps` (integrate.py:345-375), and a trainable sodium conductance."""
    from jaxley_pytorch.channels import HH

    cell = jx.Cell([jx.Branch(jx.Compartment(), 3)] * 7, parents=[-1, 0, 0, 1, 1, 2, 2])
    cell.insert(HH())
    cell.branch(0).comp(0).record(verbose=False)
    cell.branch(3).comp(1).record(verbose=False)
    cell.branch(3).comp(2).record(verbose=False)
    cell.branch(0).comp(0).stimulate(jx.step_current(1.0, 2.0, 0.05, 0.025, 6.0), verbose=False)
    t = np.arange(241) * 0.025
    vc = torch.as_tensor(np.where((t >= 1.0) & (t < 4.0), -20.0, -70.0))
    clamps = cell.branch(3).comp(1).data_clamp("v", vc, None)
    clamps = cell.branch(5).comp(0).data_clamp("HH_m", torch.full((241,), 0.3), clamps)
    cell.make_trainable("HH_gNa", verbose=False)
    return cell, {"delta_t": 0.025, "data_clamps": clamps}


def synapse_net(jx):
    """Eight HH cells of two compartments coupled by KineticSynapse and
    SigmoidRateSynapse in the regular layout (3 inputs of each type per cell), with a
    trainable sodium conductance shared by all cells."""
    from jaxley_pytorch.channels import HH
    from jaxley_pytorch.synapses import KineticSynapse, SigmoidRateSynapse

    rng = np.random.default_rng(7)
    n, k = 8, 3
    net = jx.Network([jx.Cell([jx.Branch(jx.Compartment(), 2)], parents=[-1]) for _ in range(n)])
    net.insert(HH())
    for cls, comp in ((KineticSynapse, 0), (SigmoidRateSynapse, 1)):
        for post in range(n):
            pres = rng.choice([c for c in range(n) if c != post], size=k, replace=False)
            for pre in sorted(pres):
                jx.connect(net.cell(int(pre)).branch(0).comp(comp), net.cell(post).branch(0).comp(0), cls())
    net.set("KineticSynapse_gS", rng.uniform(0, 1e-3, size=n * k))
    net.set("SigmoidRateSynapse_gS", rng.uniform(0, 1e-3, size=n * k))
    for c in range(n):
        net.cell(c).branch(0).comp(0).record(verbose=False)
    for c in range(0, n, 2):
        net.cell(c).branch(0).comp(1).stimulate(jx.step_current(1.0, 3.0, 0.3, 0.025, 8.0), verbose=False)
    net.make_trainable("HH_gNa", verbose=False)
    return net, {"delta_t": 0.025}


def hh_tree_cn(jx):
    """`hh_tree` stepped with Crank-Nicolson (modules/base.py:3327-3365)."""
    cell, kw = hh_tree(jx)
    return cell, dict(kw, solver="crank_nicolson")


def pospischil_cell(jx):
    """A branched cell with the Pospischil channels (Na, K, Km, CaT, Leak) and
    trainable conductances, threshold vt and CaT's vx."""
    from jaxley_pytorch.channels.pospischil import CaT, K, Km, Leak, Na

    cell = jx.Cell([jx.Branch(jx.Compartment(), 2)] * 5, parents=[-1, 0, 0, 1, 1])
    for ch in (Na(), K(), Leak()):
        cell.insert(ch)
    cell.branch([0, 1]).insert(Km())
    cell.branch([0, 3]).insert(CaT())
    cell.set("v", -70.0)
    cell.init_states()
    cell.branch(0).comp(0).record(verbose=False)
    cell.branch(4).comp(1).record(verbose=False)
    cell.branch(0).comp(0).stimulate(jx.step_current(1.0, 3.0, 0.1, 0.025, 8.0), verbose=False)
    cell.make_trainable("Na_gNa", verbose=False)
    cell.make_trainable("vt", verbose=False)
    cell.make_trainable("CaT_vx", verbose=False)
    return cell, {"delta_t": 0.025}
