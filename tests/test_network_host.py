"""Host side of the network path: the device plan of each synapse type (no GPU)."""
import numpy as np
import pytest
import torch

from jaxley_pytorch_b200.lower import lower
from jaxley_pytorch_b200.network import _ptr, _SynType, config_network


def _types():
    p = config_network(n_cells=24, ncomp=3, k=5, batch=2, n_steps=12, seed=1, rate_hz=400.0, amp=0.3)
    low = lower(p, max_block_nodes=4096)
    area = np.asarray(p.params["area"], dtype=np.float64)
    area = area[0] if area.ndim == 2 else area
    return [_SynType(s, low, area, low.batch, torch.float64, "cpu", low.dt) for s in p.synapses], low


def test_kinetic_state_is_row_major():
    # the kernels index the (batch, synapse) state flat as b * E + e
    types, low = _types()
    kin = [ty for ty in types if ty.kinetic]
    assert kin
    for ty in kin:
        assert ty.s0.shape == (low.batch, ty.E) and ty.s0.is_contiguous()
        assert ty.s0.clone().is_contiguous() and torch.empty_like(ty.s0).is_contiguous()


def test_kernel_pointers_refuse_strided_views():
    x = torch.zeros(2, 6, dtype=torch.float64)
    assert _ptr(x, torch.float64, 12, "x") == x.data_ptr()
    with pytest.raises(ValueError):
        _ptr(x.t(), torch.float64, 12, "x")
    with pytest.raises(ValueError):
        _ptr(x[:, :3], torch.float64, 6, "x")
    with pytest.raises(ValueError):
        _ptr(x.float(), torch.float64, 12, "x")
    with pytest.raises(ValueError):
        _ptr(x, torch.float64, 10, "x")
