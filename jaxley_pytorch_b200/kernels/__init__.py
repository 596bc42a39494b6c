"""Drop-in kernel modules with the reference's interfaces (`kernels/tree_solve.py`,
`kernels/synapse_step.py` of jaxley-pytorch)."""
