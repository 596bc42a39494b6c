"""The standalone tree-solve drop-in (jaxley_pytorch_b200.kernels.tree_solve) against
the oracle and a dense solve, as the reference's tests/test_kernels.py:63-136 and
tests/test_solver.py:78-199 check its Triton kernels (float64 1e-12, float32 1e-4,
gradients 1e-10, gradcheck)."""
import numpy as np
import pytest
import torch

import oracle
from jaxley_pytorch_b200.kernels import tree_solve as ts


def forests():
    rng = np.random.default_rng(0)
    out = {}
    out["chain_12"] = [-1] + list(range(11))
    out["star_8"] = [-1] + [0] * 8  # a node with 8 children (tests/test_kernels.py:25-33)
    out["point_cells_5"] = [-1] * 5
    out["ragged_4"] = [-1, 0, 0, 1]  # tests/test_solver.py:78-86
    rnd = [-1] + [int(rng.integers(0, j)) for j in range(1, 40)]
    out["random_40"] = rnd
    # a forest of uneven trees
    f = []
    for sz in [1, 7, 30, 3, 60, 2]:
        base = len(f)
        f += [-1] + [base + int(rng.integers(0, j)) for j in range(1, sz)]
    out["forest_mixed"] = f
    deep = [-1] + [int(j - 1 if rng.random() < 0.8 else rng.integers(0, j)) for j in range(1, 600)]
    out["deep_600"] = deep
    # blocks beyond one warp's 256 nodes: the CTA form of the registers variant
    wide = [-1] + [int(rng.integers(max(0, j - 40), j)) for j in range(1, 5000)]
    out["tree_5000"] = wide
    f = []
    for sz in [300, 1, 900, 40, 2500]:
        base = len(f)
        f += [-1] + [base + int(rng.integers(max(0, j - 8), j)) for j in range(1, sz)]
    out["forest_large"] = f
    return out


def system(parent, B, dtype, seed=1):
    rng = np.random.default_rng(seed)
    n = len(parent)
    parent = np.asarray(parent)
    l = rng.uniform(-0.4, -0.05, (B, n))
    u = rng.uniform(-0.4, -0.05, (B, n))
    l[:, parent < 0] = 0
    u[:, parent < 0] = 0
    d = 1.0 + rng.uniform(0.5, 1.5, (B, n)) + np.abs(l)
    for j in range(n):
        if parent[j] >= 0:
            d[:, parent[j]] += np.abs(u[:, j])
    s = rng.normal(size=(B, n))
    return d, l, u, s


def test_schedules_on_cpu():
    for name, parent in forests().items():
        lv = ts.build_level_schedule(np.asarray(parent))
        assert sorted(lv["perm"].tolist()) == list(range(len(parent)))
        if max(np.diff(np.append(np.nonzero(np.asarray(parent) < 0)[0], len(parent)))) <= ts.MAX_BLOCK:
            fs = ts.build_forest_schedule(np.asarray(parent))
            assert fs["block_size"] % 32 == 0
    big = [-1] + list(range(ts.MAX_BLOCK))  # one tree of MAX_BLOCK + 1 nodes
    with pytest.raises(ValueError):
        ts.build_forest_schedule(np.asarray(big))
    assert ts.build_forest_schedule(np.asarray(forests()["tree_5000"]))["block_size"] == 8192
    with pytest.raises(ValueError):
        ts.build_level_schedule(np.asarray([0, -1]))


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["registers", "registers_warp", "levels"])
@pytest.mark.parametrize("name", list(forests()))
def test_tree_solve_matches_oracle(cuda_device, mode, name):
    parent = np.asarray(forests()[name])
    if mode == "registers_warp":  # blocks of at most 256 nodes: one warp each
        if max(np.diff(np.append(np.nonzero(parent < 0)[0], len(parent)))) > 256:
            pytest.skip("a tree of more than 256 nodes")
        kern = ts.TreeSolveKernel(ts.build_forest_schedule(parent, max_block=256), cuda_device)
        assert kern.block_size <= 256
    else:
        kern = ts.make_tree_solve_kernel(parent, cuda_device, mode=mode)
    assert isinstance(kern, ts.LevelTreeSolveKernel if mode == "levels" else ts.TreeSolveKernel)
    d, l, u, s = system(parent, 6, np.float64)
    ref = oracle.tree_solve(d, l, u, s, parent)
    for dtype, tol in [(torch.float64, 1e-12), (torch.float32, 1e-4)]:
        args = [torch.as_tensor(a, dtype=dtype, device=cuda_device) for a in (d, l, u, s)]
        x = kern.solve(*args).double().cpu().numpy()
        np.testing.assert_allclose(x, ref, rtol=tol, atol=tol)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["registers", "levels"])
def test_tree_solve_gradients(cuda_device, mode):
    parent = np.asarray(forests()["random_40"])
    kern = ts.make_tree_solve_kernel(parent, cuda_device, mode=mode)
    d, l, u, s = system(parent, 3, np.float64, seed=4)
    args = [torch.as_tensor(a, device=cuda_device).requires_grad_(True) for a in (d, l, u, s)]
    w = torch.randn(3, len(parent), dtype=torch.float64, device=cuda_device)
    (ts.fused_tree_solve(kern, *args) * w).sum().backward()
    # Dense reference: A x = s.
    n = len(parent)
    dn = [torch.as_tensor(a).requires_grad_(True) for a in (d, l, u, s)]
    A = torch.diag_embed(dn[0])
    idx = torch.arange(n)
    par = torch.as_tensor(np.where(parent >= 0, parent, 0))
    has = torch.as_tensor(parent >= 0)
    bi = torch.arange(d.shape[0])[:, None]
    rows, cols = idx[has][None, :], par[has][None, :]
    A = A.index_put((bi, rows, cols), dn[1][:, has], accumulate=True)
    A = A.index_put((bi, cols, rows), dn[2][:, has], accumulate=True)
    x = torch.linalg.solve(A, dn[3])
    (x * w.cpu()).sum().backward()
    for g, r in zip(args, dn):
        np.testing.assert_allclose(g.grad.cpu().numpy(), r.grad.numpy(), rtol=1e-10, atol=1e-10)


@pytest.mark.gpu
def test_tree_solve_gradcheck(cuda_device):
    parent = np.asarray(forests()["ragged_4"])
    kern = ts.make_tree_solve_kernel(parent, cuda_device, mode="levels")
    d, l, u, s = system(parent, 2, np.float64, seed=5)
    args = tuple(torch.as_tensor(a, device=cuda_device).requires_grad_(True) for a in (d, l, u, s))
    assert torch.autograd.gradcheck(lambda *a: ts.fused_tree_solve(kern, *a), args)


def test_default_block_sizes():
    """Registers variant: blocks of at least REG_MIN_BLOCK nodes (a CTA each) unless a
    tree is larger; levels variant: a forest of small trees in at least
    LEVEL_MIN_BLOCKS blocks of at least LEVEL_MIN_BLOCK nodes."""
    rng = np.random.default_rng(5)
    forest = []
    for _ in range(512):
        b = len(forest)
        forest += [-1] + [b + int(rng.integers(0, j)) for j in range(1, 40)]
    forest = np.asarray(forest)
    fs = ts.build_forest_schedule(forest)
    assert fs["block_size"] == ts.REG_MIN_BLOCK
    assert all(int(r[1]) <= ts.REG_MIN_BLOCK for r in fs["block_info"])
    assert ts.build_forest_schedule(forest, max_block=64)["block_size"] == 64
    lv = ts.build_level_schedule(forest)
    assert len(lv["block_info"]) >= ts.LEVEL_MIN_BLOCKS
    assert lv["max_block_nodes"] >= ts.LEVEL_MIN_BLOCK - 40
    assert sum(int(r[1]) for r in lv["block_info"]) == len(forest)
    one = np.asarray(forests()["deep_600"])  # one tree: one block whatever its size
    assert len(ts.build_level_schedule(one)["block_info"]) == 1


@pytest.mark.gpu
def test_env_var_selects_variant(cuda_device, monkeypatch):
    parent = np.asarray(forests()["random_40"])
    monkeypatch.setenv("JAXLEY_PYTORCH_TREE_KERNEL", "levels")
    assert isinstance(ts.make_tree_solve_kernel(parent, cuda_device), ts.LevelTreeSolveKernel)
    monkeypatch.setenv("JAXLEY_PYTORCH_TREE_KERNEL", "registers")
    assert isinstance(ts.make_tree_solve_kernel(parent, cuda_device), ts.TreeSolveKernel)
    monkeypatch.setenv("JAXLEY_PYTORCH_TREE_KERNEL", "auto")
    deep = np.asarray(forests()["deep_600"])
    assert isinstance(ts.make_tree_solve_kernel(deep, cuda_device), ts.LevelTreeSolveKernel)
    assert isinstance(ts.make_tree_solve_kernel(parent, cuda_device), ts.LevelTreeSolveKernel)


def test_op_registry_holds_kernels_weakly():
    """A kernel registered by `fused` leaves the op registry with its last owner."""
    import gc

    parent = np.asarray(forests()["random_40"])
    kern = ts.TreeSolveKernel(ts.build_forest_schedule(parent), "cpu")
    ts._register(kern)
    key = kern.t["block_info"].data_ptr()
    assert ts._KERNELS.get(key) is kern
    del kern
    gc.collect()
    assert key not in ts._KERNELS


@pytest.mark.gpu
@pytest.mark.parametrize("mode", ["registers", "levels"])
def test_op_with_callers_schedule_tensors(cuda_device, mode):
    """The custom op called with schedule tensors of the caller's own (no kernel object
    registered for them) solves the tree its parent_safe / has_parent describe."""
    parent = np.asarray(forests()["forest_mixed"])
    kern = ts.make_tree_solve_kernel(parent, cuda_device, mode=mode)
    d, l, u, s = (torch.as_tensor(a, device=cuda_device) for a in system(parent, 3, np.float64, seed=7))
    ref = kern.solve(d, l, u, s)
    ts._register(kern)
    # Copies of every schedule tensor: addresses the registry has never seen.
    if mode == "registers":
        t = {k: v.clone() for k, v in kern.t.items()}
        x = ts.tree_solve_op(d, l, u, s, t["block_info"], t["rel_parent"], t["rel_height"],
                             t["rel_children"], kern.parent_safe.clone(), kern.has_parent.clone(),
                             kern.block_size, kern.num_slots, kern.num_warps)
    else:
        t = {k: v.clone() for k, v in kern.t.items()}
        x = ts.tree_solve_levels_op(d, l, u, s, t["block_info"], t["level_ptr"], t["perm"],
                                    t["chain_ptop"], t["chain_child"], kern.parent_safe.clone(),
                                    kern.has_parent.clone(), kern.num_slots, 0)
    torch.testing.assert_close(x, ref, rtol=1e-12, atol=1e-12)
