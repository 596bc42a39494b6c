"""Drop-in kernel modules with the reference's interfaces (`kernels/tree_solve.py`,
`kernels/synapse_step.py` of jaxley-pytorch)."""


# Namespace of this package's custom ops. They keep the reference's op names and
# schemas (`tree_solve`, `tree_solve_levels`, `synapse_step`, `synapse_step_backward`)
# under a namespace of their own: torch replaces a custom op that is defined twice
# under one name, silently and for every holder of the first definition, so sharing
# `jaxley_pytorch::` would break whichever of the two packages registered first.
OP_NAMESPACE = "jaxley_pytorch_b200"
