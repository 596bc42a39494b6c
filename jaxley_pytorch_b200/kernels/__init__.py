"""Drop-in kernel modules with the reference's interfaces (`kernels/tree_solve.py`,
`kernels/synapse_step.py` of jaxley-pytorch)."""


def op_namespace(names) -> str:
    """The namespace for this package's custom ops named `names`: the reference's
    `jaxley_pytorch` when none of them is registered there yet, else
    `jaxley_pytorch_b200` (a second definition under a taken name would silently
    replace the reference's op for every caller in the process)."""
    import torch

    if any(hasattr(torch.ops.jaxley_pytorch, n) for n in names):
        return "jaxley_pytorch_b200"
    return "jaxley_pytorch"
