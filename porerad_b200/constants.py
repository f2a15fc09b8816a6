"""Constants of the path (porerad/constants.py:3-11): the archived results were computed with these values."""

SIGMA = 5.670374419e-8
"""Stefan-Boltzmann constant (the CODATA 2018 exact value), in W / (m^2 K^4)."""

K_SOLID = 0.20
"""Conductivity of every solid cell, in W / (m K)."""

K_GAS = 0.026
"""Conductivity of every pore cell (still air), in W / (m K)."""
