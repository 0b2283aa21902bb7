"""Parasitic extraction front door (``fieldspice/extraction.py``).

:func:`capacitance_matrix` keeps the reference signature
(``extraction.py:41-56``) and routes to the GPU :class:`PoissonSolver`.
"""

from __future__ import annotations

from typing import Sequence

import numpy as np

__all__ = ["capacitance_matrix", "to_spice_matrix"]


def capacitance_matrix(grid, eps_cell: np.ndarray, terminals: Sequence,
                       bc=None, config=None, *, report: dict | None = None,
                       gpu=None) -> np.ndarray:
    """Maxwell capacitance matrix [F], shape ``(nt, nt)``.

    Unit excitation of every terminal in turn (all solved as one block of
    right-hand sides on the GPU), charge integrated on every terminal,
    symmetrised; the pre-symmetrisation asymmetry is in ``report``.
    """
    from .solvers.poisson import PoissonSolver
    solver = PoissonSolver(grid, eps_cell, config, gpu=gpu)
    return solver.capacitance_matrix(list(terminals), bc, report=report)


def to_spice_matrix(c_maxwell: np.ndarray) -> np.ndarray:
    """Maxwell -> SPICE/mutual form (``extraction.py:90-102``)."""
    c = np.asarray(c_maxwell, dtype=float)
    if c.ndim != 2 or c.shape[0] != c.shape[1]:
        raise ValueError("capacitance matrix must be square")
    out = -c.copy()
    np.fill_diagonal(out, c.sum(axis=1))
    return out
