"""Host logic of the work-item groups: blocks whose working set exceeds a CTA's
shared memory go to the global-scratch group; every (block, row range) is covered
exactly once and each group's sizing covers its blocks."""
import numpy as np
import pytest
import torch

from jaxley_pytorch_b200 import _lib, synth
from jaxley_pytorch_b200.lower import lower
from jaxley_pytorch_b200.sim import DeviceModel


def _model(limit, rows=1):
    prob = synth.config_uneven(n_cells=40, n_steps=5, max_comp=400, seed=3)
    low = lower(prob, max_block_nodes=256, keep_currents=False)
    return low, DeviceModel(low, torch.float32, device="cpu", rows_per_item=rows, smem_limit=limit)


@pytest.mark.parametrize("limit", [1 << 30, 48 * 1024, 20 * 1024, 1])
def test_groups_partition_the_items(limit):
    low, m = _model(limit)
    for kind in ("forward", "backward"):
        seen = []
        for g in m.groups[kind]:
            items = g["items"].numpy()
            assert len(items) == g["n_items"]
            seen += [tuple(it[:3]) for it in items]
            blocks = low.blocks[items[:, 0]]
            mx = g["maxima"]
            assert blocks[:, 1].max() <= mx["max_nodes"] and blocks[:, 3].max() <= mx["max_slots"]
            assert blocks[:, 5].max() <= mx["max_chains"] and blocks[:, 7].max() <= mx["max_levels"]
            assert blocks[:, 9].max() <= mx["max_pslots"] and blocks[:, 10].max() <= mx["max_gslots"]
            assert g["stride"] % 256 == 0
            if not g["gm"]:
                assert m._layout_bytes(mx, kind == "backward") <= limit
        assert sorted(seen) == sorted((b, 0, 1) for b in range(len(low.blocks)))
    if limit == 1:  # nothing fits: a single global-scratch group
        assert all(g["gm"] for g in m.groups["forward"]) and len(m.groups["forward"]) == 1
    if limit == 1 << 30:
        assert not any(g["gm"] for k in m.groups for g in m.groups[k])


def test_group_args_fill_the_group_fields():
    low, m = _model(48 * 1024)
    state = torch.zeros((low.batch, low.n_slots))
    base = m.args(state, 3, 0, None)
    assert base.n_items == 0  # filled per group only
    for g in m.groups["backward"]:
        a = m.group_args(base, "backward", g)
        assert a.n_items == g["n_items"] and a.max_nodes == g["maxima"]["max_nodes"]
        assert (a.gscratch is not None) == g["gm"]
        if g["gm"]:
            assert a.gscratch % 256 == 0 and a.gscratch_stride == g["stride"]


def test_block_gradient_slot_counts():
    low, _ = _model(1 << 30)
    # n_gslots of a block = gradient slots of its nodes (gbase is block-relative)
    for b in low.blocks:
        last = b[0] + b[1] - 1
        po, cls = low.poff[last], low.node_class[last]
        npar = sum(int(e[2]) for e in low.entries[low.cls_ptr[cls]:low.cls_ptr[cls + 1]])
        assert b[10] == low.gbase[last] + np.count_nonzero(low.pcol[po:po + npar])
    assert low.max_gslots == low.blocks[:, 10].max()


def test_layout_grows_with_the_block():
    low, m = _model(1 << 30)
    sizes = [m._layout_bytes(m._block_maxima(np.asarray([b])), True) for b in range(len(low.blocks))]
    both = m._layout_bytes(m._block_maxima(np.arange(len(low.blocks))), True)
    assert both >= max(sizes)
    assert _lib.JxbSimArgs.gscratch.offset > _lib.JxbSimArgs.mode.offset


@pytest.mark.parametrize("warps", [1, 4, 16])
def test_node_schedule_covers_every_node_once(warps):
    from jaxley_pytorch_b200.sim import class_costs, node_schedule

    low, _ = _model(1 << 30)
    ptr, sched = node_schedule(low, warps)
    cost = class_costs(low)
    assert len(ptr) == len(low.blocks) + 1 and ptr[-1] == len(sched)
    for b, blk in enumerate(low.blocks):
        part = sched[ptr[b]:ptr[b + 1]].reshape(warps, -1, 32)
        nodes = part[part >= 0]
        assert sorted(nodes.tolist()) == list(range(blk[1]))
        cls = low.node_class[blk[0]:blk[0] + blk[1]]
        loads = []
        for w in range(warps):
            load = 0.0
            for k in range(part.shape[1]):
                chunk = part[w, k][part[w, k] >= 0]
                if len(chunk):
                    assert len(set(cls[chunk].tolist())) == 1  # one class per chunk
                    load += cost[cls[chunk[0]]]
            loads.append(load)
        # greedy balance: no warp exceeds the mean by more than the dearest chunk
        assert max(loads) <= np.mean(loads) + cost.max() + 1e-9
