"""CPU restatement of jaxley-pytorch's per-timestep hot path (numpy, float64).

TEST INFRASTRUCTURE ONLY. This package is the checker that the CUDA path is compared
against: only `tests/`, `__graft_entry__.smoke()` and the `cpu_baseline` / reference
arm of `bench.py` may import it, and only as the checker or the timed CPU baseline.
The product path (`jaxley_pytorch_b200`) never imports it.

Parity pin: `tests/test_oracle_golden.py` checks this restatement against the golden
voltage traces held by the reference's own tests
(`tests/jaxley_identical/test_basic_modules.py`) and against fixtures produced by
running the reference itself (`tests/golden/make_fixtures.py`).
"""
from .step import (  # noqa: F401
    integrate,
    init_steady_states,
    tree_solve,
    x_over_expm1,
    save_exp,
    synapse_step,
    synapse_step_backward,
)
