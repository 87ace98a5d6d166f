"""Physical constants (SI), as src/tree_d_3d/constants.py."""

#: Coulomb constant 1 / (4 pi eps_0), in N m^2 / C^2.
K_E: float = 8.9875517923e9
