"""Registry of the ion-channel models that the CUDA step kernels implement.

Every entry restates the interface of one reference channel class: the order of its
parameters and states (the order of the class's ``channel_params`` /
``channel_states`` dicts), its ``current_name``, its default values and the integer
type id under which ``csrc/channels.cuh`` implements its ``update_states`` and
``compute_current``. The lowering (``lower.py``) maps each channel instance of a
problem onto a kernel entry through this table.

Reference classes (file:line in jaxley-pytorch):

====================  =======================================  ====
type                  reference class                           id
====================  =======================================  ====
HH                    ``channels/hh.py:14``                      0
Leak                  ``channels/pospischil.py:39``              1
NaTaT                 ``mech/channels/l5pc.py:38``               2
NaTs2T                ``mech/channels/l5pc.py:118``              3
NapEt2                ``mech/channels/l5pc.py:200``              4
KPst                  ``mech/channels/l5pc.py:294``              5
KTst                  ``mech/channels/l5pc.py:384``              6
SKE2                  ``mech/channels/l5pc.py:463``              7
SKv3_1                ``mech/channels/l5pc.py:533``              8
M                     ``mech/channels/l5pc.py:593``              9
CaHVA                 ``mech/channels/l5pc.py:664``             10
CaLVA                 ``mech/channels/l5pc.py:737``             11
CaPump                ``mech/channels/l5pc.py:814``             12
CaNernstReversal      ``mech/channels/l5pc.py:872``             13
H                     ``mech/channels/l5pc.py:919``             14
Na                    ``channels/pospischil.py:74``              15
K                     ``channels/pospischil.py:143``             16
Km                    ``channels/pospischil.py:197``             17
CaL                   ``channels/pospischil.py:252``             18
CaT                   ``channels/pospischil.py:318``             19
====================  =======================================  ====
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Dict, List, Tuple


@dataclass(frozen=True)
class ChannelSpec:
    """Kernel-facing description of one channel model.

    ``params`` and ``states`` hold ``(suffix, default)`` pairs in the reference's dict
    order. A suffix that starts with ``"/"`` is a global (unprefixed) name such as
    ``eNa`` or ``CaCon_i``; otherwise the name is ``f"{instance}_{suffix}"``.
    ``constants`` are the reference's ``channel_constants`` (passed to the kernel
    as parameters that never carry gradients). ``current`` is the ``current_name``;
    ``"{name}"`` is replaced by the instance name (``Leak`` uses ``i_{name}``).
    """

    type_id: int
    params: Tuple[Tuple[str, float], ...]
    states: Tuple[Tuple[str, float], ...]
    current: str
    constants: Tuple[Tuple[str, float], ...] = ()
    ohmic_g: Tuple[int, ...] = ()  # Indices of the conductance parameters.


def _p(*pairs):
    return tuple(pairs)


SPECS: Dict[str, ChannelSpec] = {
    "HH": ChannelSpec(
        0,
        _p(("gNa", 0.12), ("gK", 0.036), ("gLeak", 0.0003), ("eNa", 50.0),
           ("eK", -77.0), ("eLeak", -54.3)),
        _p(("m", 0.2), ("h", 0.2), ("n", 0.2)),
        "i_HH",
        ohmic_g=(0, 1, 2),
    ),
    "Leak": ChannelSpec(1, _p(("gLeak", 1e-4), ("eLeak", -70.0)), (), "i_{name}",
                        ohmic_g=(0,)),
    "NaTaT": ChannelSpec(2, _p(("gNaTaT", 1e-5), ("/eNa", 50.0)),
                         _p(("m", 0.1), ("h", 0.1)), "i_Na", ohmic_g=(0,)),
    "NaTs2T": ChannelSpec(3, _p(("gNaTs2T", 1e-5), ("/eNa", 50.0)),
                          _p(("m", 0.1), ("h", 0.1)), "i_Na", ohmic_g=(0,)),
    "NapEt2": ChannelSpec(4, _p(("gNapEt2", 1e-5), ("/eNa", 50.0)),
                          _p(("m", 0.1), ("h", 0.1)), "i_Na", ohmic_g=(0,)),
    "KPst": ChannelSpec(5, _p(("gKPst", 1e-5), ("/eK", -77.0)),
                        _p(("m", 0.1), ("h", 0.1)), "i_K", ohmic_g=(0,)),
    "KTst": ChannelSpec(6, _p(("gKTst", 1e-5), ("/eK", -77.0)),
                        _p(("m", 0.1), ("h", 0.1)), "i_K", ohmic_g=(0,)),
    "SKE2": ChannelSpec(7, _p(("gSKE2", 1e-6), ("/eK", -77.0)),
                        _p(("z", 0.0), ("/CaCon_i", 5e-5)), "i_K", ohmic_g=(0,)),
    "SKv3_1": ChannelSpec(8, _p(("gSKv3_1", 1e-5), ("/eK", -77.0)),
                          _p(("m", 0.1),), "i_K", ohmic_g=(0,)),
    "M": ChannelSpec(9, _p(("gM", 1e-5), ("/eK", -77.0)), _p(("m", 0.0),), "i_K",
                     ohmic_g=(0,)),
    "CaHVA": ChannelSpec(10, _p(("gCaHVA", 1e-5),),
                         _p(("m", 0.1), ("h", 0.1), ("/eCa", 0.0)), "i_Ca",
                         ohmic_g=(0,)),
    "CaLVA": ChannelSpec(11, _p(("gCaLVA", 1e-5),),
                         _p(("m", 0.0), ("h", 0.0), ("/eCa", 0.0)), "i_Ca",
                         ohmic_g=(0,)),
    "CaPump": ChannelSpec(12, _p(("gamma", 0.05), ("decay", 80.0), ("depth", 0.1),
                                 ("minCai", 1e-4)),
                          _p(("/CaCon_i", 5e-5),), "i_Ca"),
    "CaNernstReversal": ChannelSpec(
        13, (), _p(("/eCa", 0.0), ("/CaCon_i", 5e-5), ("/CaCon_e", 2.0)), "i_Ca",
        constants=_p(("F", 96485.3329), ("T", 279.45), ("R", 8.314)),
    ),
    "H": ChannelSpec(14, _p(("gH", 1e-5), ("/eH", -45.0)), _p(("m", 0.0),), "i_H",
                     ohmic_g=(0,)),
    "Na": ChannelSpec(15, _p(("gNa", 50e-3), ("/eNa", 50.0), ("/vt", -60.0)),
                      _p(("m", 0.2), ("h", 0.2)), "i_Na", ohmic_g=(0,)),
    "K": ChannelSpec(16, _p(("gK", 5e-3), ("/eK", -90.0), ("/vt", -60.0)),
                     _p(("n", 0.2),), "i_K", ohmic_g=(0,)),
    "Km": ChannelSpec(17, _p(("gKm", 0.004e-3), ("taumax", 4000.0), ("/eK", -90.0)),
                      _p(("p", 0.2),), "i_K", ohmic_g=(0,)),
    "CaL": ChannelSpec(18, _p(("gCaL", 0.1e-3), ("/eCa", 120.0)),
                       _p(("q", 0.2), ("r", 0.2)), "i_Ca", ohmic_g=(0,)),
    "CaT": ChannelSpec(19, _p(("gCaT", 0.4e-4), ("vx", 2.0), ("/eCa", 120.0)),
                       _p(("u", 0.2),), "i_Ca"),
}

# Reference modules whose classes of the same name are the ones restated here (the
# `pumps/` package has different classes called `CaPump` and `CaNernstReversal`).
_REFERENCE_MODULES = {
    "HH": "jaxley_pytorch.channels.hh",
    **{k: "jaxley_pytorch.channels.pospischil" for k in ("Leak", "Na", "K", "Km", "CaL", "CaT")},
}
_L5PC_MODULE = "jaxley_pytorch.mech.channels.l5pc"


def full_name(instance: str, suffix: str) -> str:
    """The reference's name of a parameter or state of a channel instance."""
    if suffix.startswith("/"):
        return suffix[1:]
    return f"{instance}_{suffix}"


def current_name(type_name: str, instance: str) -> str:
    return SPECS[type_name].current.replace("{name}", instance)


def spec_for_reference_channel(channel) -> Tuple[str, ChannelSpec]:
    """Return `(type_name, spec)` for an instance of a reference channel class.

    Raises `NotImplementedError` for channels that have no CUDA implementation.
    """
    cls = type(channel)
    name = cls.__name__
    module = cls.__module__
    expected = _REFERENCE_MODULES.get(name, _L5PC_MODULE)
    if name not in SPECS or module != expected:
        raise NotImplementedError(
            f"channel {module}.{name} has no sm_100a implementation in this package"
        )
    return name, SPECS[name]


@dataclass
class ChannelInstance:
    """One inserted channel of a problem (reference node order).

    ``params``/``states`` are the full reference names in kernel role order;
    ``constants`` are values (channel constants such as the Nernst temperature).
    """

    type_name: str
    name: str
    inds: "object"  # np.ndarray of node indices (reference node order)
    params: List[str]
    states: List[str]
    current: str
    constants: List[float] = field(default_factory=list)

    @property
    def spec(self) -> ChannelSpec:
        return SPECS[self.type_name]


def make_instance(type_name: str, inds, name: str | None = None,
                  constants: Dict[str, float] | None = None) -> ChannelInstance:
    """A channel instance with the reference's naming conventions."""
    spec = SPECS[type_name]
    name = name or type_name
    consts = dict(spec.constants)
    if constants:
        consts.update(constants)
    return ChannelInstance(
        type_name=type_name,
        name=name,
        inds=inds,
        params=[full_name(name, s) for s, _ in spec.params],
        states=[full_name(name, s) for s, _ in spec.states],
        current=current_name(type_name, name),
        constants=[float(consts[k]) for k, _ in spec.constants],
    )


def default_params(inst: ChannelInstance) -> Dict[str, float]:
    return {n: d for n, (_, d) in zip(inst.params, inst.spec.params)}


def default_states(inst: ChannelInstance) -> Dict[str, float]:
    return {n: d for n, (_, d) in zip(inst.states, inst.spec.states)}
