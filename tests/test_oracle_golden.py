"""The CPU restatement (oracle/) against the reference's own golden traces and the
reference's outputs stored in the fixtures."""
import numpy as np
import pytest

import oracle
from conftest import fixture_names, load_fixture


@pytest.mark.parametrize("name", fixture_names("golden_"))
def test_oracle_matches_reference_golden_vectors(name):
    # tests/jaxley_identical/test_basic_modules.py:25-122, 125-243: max abs error
    # <= 1e-8 (1e-5 for the uneven radii, as there).
    prob, extra = load_fixture(name)
    out = oracle.integrate(prob)
    every = int(extra["every"])
    tol = float(extra["tol"]) if "tol" in extra else 1e-8
    golden = extra["golden"].reshape(out[0, :, ::every].shape)
    assert np.max(np.abs(out[0, :, ::every] - golden)) <= tol


@pytest.mark.parametrize("name", fixture_names())
def test_oracle_matches_reference_run(name):
    prob, extra = load_fixture(name)
    out = oracle.integrate(prob, init_steady=bool(extra.get("init_steady", 0)))
    ref = extra["ref"].reshape(out.shape)
    scale = max(1.0, np.max(np.abs(ref)))
    assert np.max(np.abs(out - ref)) <= 1e-9 * scale


def test_tree_solve_against_dense():
    # tests/test_solver.py:78-86, 107-130: a ragged tree against np.linalg.solve.
    rng = np.random.default_rng(0)
    parent = np.array([-1, 0, 0, 1, 1, 2, 5, 5, 7])
    n = len(parent)
    B = 4
    d = rng.uniform(2, 4, (B, n))
    l = rng.normal(size=(B, n)) * 0.3
    u = rng.normal(size=(B, n)) * 0.3
    l[:, 0] = u[:, 0] = 0
    s = rng.normal(size=(B, n))
    x = oracle.tree_solve(d, l, u, s, parent)
    for b in range(B):
        A = np.diag(d[b])
        for j in range(1, n):
            A[j, parent[j]] = l[b, j]
            A[parent[j], j] = u[b, j]
        np.testing.assert_allclose(x[b], np.linalg.solve(A, s[b]), rtol=1e-12, atol=1e-12)


def test_x_over_expm1_against_float64_reference():
    # tests/test_float32_safety.py:31-45: the series branch and the limit at 0.
    x = np.array([-1e-7, 0.0, 1e-7, 1e-3, -3.0, 25.0, -50.0])
    y = 10.0
    ref = np.where(np.abs(x / y) < 1e-12, y, x / np.expm1(np.minimum(x / y, 20.0) + 0 * x))
    got = oracle.x_over_expm1(x, y)
    np.testing.assert_allclose(got, ref, rtol=1e-6)
    assert oracle.x_over_expm1(np.array(0.0), 10.0) == 10.0


@pytest.mark.parametrize("name", ["cell_8comp_hh", "hh_tree_15x3", "l5pc_7x4_batch3", "hh_forest_6"])
def test_torch_port_matches_oracle(name):
    """The torch restatement used as the timed CPU baseline computes what the numpy
    oracle computes (float64)."""
    import torch

    from oracle import torch_port

    prob, extra = load_fixture(name)
    prob.n_steps = min(prob.n_steps, 200)
    ref = oracle.integrate(prob)
    out = torch_port.integrate(prob, {}, dtype=torch.float64).numpy()
    np.testing.assert_allclose(out, ref, rtol=1e-10, atol=1e-9)
