"""Parasitic extraction front door (``fieldspice/extraction.py``).

:func:`capacitance_matrix` keeps the reference signature
(``extraction.py:41-56``) and routes to the GPU :class:`PoissonSolver`.
"""

from __future__ import annotations

import warnings
from typing import Sequence

import numpy as np

__all__ = ["capacitance_matrix", "resistance_matrix", "to_spice_matrix"]


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


def resistance_matrix(grid, sigma_cell: np.ndarray, terminals: Sequence,
                      bc=None, config=None, *, report: dict | None = None,
                      gpu=None) -> np.ndarray:
    """DC resistance matrix [ohm] (``extraction.py:59-87``).

    Every terminal driven to 1 V in turn with the others at 0 V and every wall
    insulating (``bc`` is accepted and ignored, as in the reference); the
    conductance ``Y[i, j]`` is the current into terminal ``i``, integrated in
    FP64 on the GPU like a capacitance extraction with sigma masses.  ``Y`` is
    symmetrised and pseudo-inverted with NumPy's default cutoff, so the
    all-ones direction, null only to round-off, is kept as the reference keeps
    it: only resistance DIFFERENCES (``P R P`` with ``P = I - 11^T/n``) are
    meaningful.  Cells of zero conductivity are allowed; nodes that no
    terminal reaches are pinned to 0 V.
    """
    import torch
    from .device import DeviceOperator, h2d
    from .solvers.base import GPUConfig, SolverConfig, resolve_preconditioner
    from .solvers.poisson import check_terminals, extract_capacitance
    terms = check_terminals(list(terminals), grid)
    if len(terms) < 2:
        raise ValueError("resistance extraction needs at least two terminals")
    sig = np.asarray(sigma_cell, dtype=float)
    if sig.shape != tuple(grid.shape_cells):
        raise ValueError(f"sigma_cell must have shape {grid.shape_cells}, got {sig.shape}")
    if not np.all(np.isfinite(sig)) or np.any(sig < 0.0):
        raise ValueError("sigma_cell must be finite and non-negative [S/m]")
    cfg = config or SolverConfig()
    gcfg = gpu or GPUConfig()
    op = DeviceOperator(grid, sig)
    dev = op.dev
    term_dev = [h2d(np.asarray(t.nodes, np.int64), torch.int64, dev) for t in terms]
    empty = torch.zeros(0, dtype=torch.int64, device=dev)
    Y, _, info = extract_capacitance(op, term_dev, empty, empty, tol=float(cfg.tol),
                                     precision=gcfg.precision, maxiter=gcfg.maxiter,
                                     preconditioner=resolve_preconditioner(cfg, gcfg))
    if info["n_pinned"]:
        warnings.warn(
            f"{info['n_pinned']} unknown(s) are coupled to nothing (empty rows); "
            "they are pinned to zero.  In a conductance matrix this means a "
            "region of zero conductivity that no terminal reaches.",
            RuntimeWarning, stacklevel=2)
    Ys = 0.5 * (Y + Y.T)
    if report is not None:
        scale = float(np.abs(np.diag(Y)).max()) or 1.0
        report.update({"Y": Ys, "asymmetry_rel": float(np.abs(Y - Y.T).max()) / scale,
                       "row_sum_rel": float(np.abs(Ys.sum(axis=1)).max()) / scale,
                       "linear": info})
    return np.linalg.pinv(Ys)


def to_spice_matrix(c_maxwell: np.ndarray) -> np.ndarray:
    """Maxwell -> SPICE/mutual form (``extraction.py:90-102``)."""
    c = np.asarray(c_maxwell, dtype=float)
    if c.ndim != 2 or c.shape[0] != c.shape[1]:
        raise ValueError("capacitance matrix must be square")
    out = -c.copy()
    np.fill_diagonal(out, c.sum(axis=1))
    return out
