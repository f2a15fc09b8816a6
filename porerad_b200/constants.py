"""Physical constants of the path (porerad/constants.py:3)."""

SIGMA = 5.670374419e-8
"""Stefan-Boltzmann constant, W m^-2 K^-4."""
