"""Physical constants and material properties of the path (porerad/constants.py:3-11)."""

SIGMA = 5.670374419e-8
"""Stefan-Boltzmann constant, W m^-2 K^-4."""

K_SOLID = 0.20
"""Thermal conductivity of the solid phase, W m^-1 K^-1."""

K_GAS = 0.026
"""Thermal conductivity of the stagnant pore gas, W m^-1 K^-1."""
