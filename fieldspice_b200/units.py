"""SI constants used by the elliptic path (values as fieldspice/units.py:20-26)."""

import math

c0 = 299_792_458.0
mu0 = 4e-7 * math.pi * 1.0000000000552
eps0 = 1.0 / (mu0 * c0 * c0)
um = 1e-6
nm = 1e-9

__all__ = ["c0", "mu0", "eps0", "um", "nm"]
