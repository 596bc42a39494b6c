"""sm_100a (B200) kernels for jaxley-pytorch's per-timestep hot path.

`jaxley_pytorch_b200.integrate` is the entry point with `jx.integrate`'s signature
(defined in the submodule of the same name); a reference module is needed only when
one is passed to it.
"""
from .integrate import integrate  # noqa: F401
