"""Host-side lowering: the chain schedule replayed on the CPU must solve the same
system as the oracle, and the library must export the C ABI."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle
from conftest import REPO, fixture_names, load_fixture
from jaxley_pytorch_b200.lower import chain_order, emulate_block_solve, lower


@pytest.mark.parametrize("name", fixture_names())
@pytest.mark.parametrize("max_block", [4096, 16])
def test_chain_schedule_solves_the_tree(name, max_block):
    prob, _ = load_fixture(name)
    low = lower(prob, max_block_nodes=max_block)
    n = prob.n_nodes
    parent, gl, gu = prob.solve_order_system()
    rng = np.random.default_rng(1)
    B, dt = 3, 0.025
    d = rng.uniform(1, 3, (B, n))
    s = rng.normal(size=(B, n))
    ref = oracle.tree_solve(d, -dt * gl * np.ones((B, 1)), -dt * gu * np.ones((B, 1)), s, parent)
    solve_of_node = np.empty(n, np.int64)
    solve_of_node[prob.to_solve] = np.arange(n)
    int2solve = solve_of_node[low.int2node]
    got = emulate_block_solve(low, d[:, int2solve], s[:, int2solve], -dt * low.a_low, -dt * low.a_up)
    np.testing.assert_allclose(got, ref[:, int2solve], rtol=1e-12, atol=1e-12)


def test_chain_order_properties():
    rng = np.random.default_rng(2)
    parent = [-1] + [int(rng.integers(0, j)) for j in range(1, 200)]
    parent += [-1] + [200 + int(rng.integers(0, j)) for j in range(1, 50)]
    order, trees, chains = chain_order(np.asarray(parent))
    assert sorted(order.tolist()) == list(range(250))
    assert trees.tolist() == [0, 200, 250]
    pos = np.empty(250, np.int64)
    pos[order] = np.arange(250)
    for top, ln, ptop, kids in chains:
        for j in range(top + 1, top + ln):
            assert parent[order[j]] == order[j - 1]
        if ptop >= 0:
            assert parent[order[top]] == order[ptop]
            assert ptop < top


def test_library_exports_every_declared_symbol():
    from jaxley_pytorch_b200 import _lib

    header = open(os.path.join(REPO, "include", "jxb.h")).read()
    declared = set(re.findall(r"^\s*(?:int|int64_t|const char\*)\s+(jxb_\w+)\s*\(", header, re.M))
    assert declared == set(_lib.EXPORTED)
    if not os.path.exists(_lib.LIB_PATH):
        pytest.skip("libjxb is not built")
    lib = ctypes.CDLL(_lib.LIB_PATH)
    for name in declared:
        assert hasattr(lib, name), name


@pytest.mark.parametrize("name", fixture_names())
def test_every_batched_parameter_has_a_gradient_slot(name):
    prob, _ = load_fixture(name)
    low = lower(prob)
    for i in range(low.n_nodes):
        cls = low.node_class[i]
        npar = sum(int(e[2]) for e in low.entries[low.cls_ptr[cls]:low.cls_ptr[cls + 1]])
        run = slice(low.poff[i], low.poff[i] + npar)
        cols, gk = low.pcol[run], low.gk[run]
        assert np.all((cols != 0) == (gk >= 0))
        if npar:
            assert sorted(gk[gk >= 0].tolist()) == list(range(int(np.count_nonzero(cols))))


def test_float32_expm1_series_bound():
    """The float32 exp(x) - 1 of csrc/jxb_math.cuh: degree-7 Taylor series below
    |x| = 1/4 (evaluated here in float32 Horner form), exp(x) - 1 above; checked
    against float64 expm1 to 1e-6 relative."""
    x = np.concatenate([np.linspace(-0.2499, 0.2499, 20001), -np.logspace(-12, -0.7, 500),
                        np.logspace(-12, -0.7, 500)]).astype(np.float32)
    p = np.float32(1.0 / 5040.0)
    for c in [1.0 / 720.0, 1.0 / 120.0, 1.0 / 24.0, 1.0 / 6.0, 0.5, 1.0]:
        p = (p * x + np.float32(c)).astype(np.float32)
    got = (p * x).astype(np.float64)
    ref = np.expm1(x.astype(np.float64))
    rel = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300)
    assert rel.max() < 1e-6, rel.max()


def test_somatic_program_needs_its_exact_layout():
    # the L5PC soma class runs the compile-time somatic program only with the slot
    # layout it was written for; extra current slots send it back to the interpreter
    from jaxley_pytorch_b200 import synth
    from jaxley_pytorch_b200.lower import PROG_L5PC_SOMA, lower as lower_

    prob = synth.config_l5pc_tree(batch=1, n_steps=10, seed=0, scale_seed=1)
    assert PROG_L5PC_SOMA in set(int(p) for p in lower_(prob, keep_currents=False).cls_prog)
    assert PROG_L5PC_SOMA not in set(int(p) for p in lower_(prob, keep_currents=True).cls_prog)
