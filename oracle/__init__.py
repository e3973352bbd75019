"""CPU oracle of the reference FDTD engine: test infrastructure only.

Nothing in the product package (efs_b200) imports this package.
"""
