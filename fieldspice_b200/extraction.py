"""Parasitic extraction front door (``fieldspice/extraction.py``).

:func:`capacitance_matrix` keeps the reference signature
(``extraction.py:41-56``) and routes to the GPU :class:`PoissonSolver`;
:func:`resistance_matrix` is the same solve with conductivity masses;
:func:`rlgc_2d` runs its three cross-section extractions (real dielectric,
vacuum, conductivity) as one batch of GPU solves.  The transmission-line and
network-parameter helpers below it are the reference's closed forms on small
host matrices (``extraction.py:236-317``).
"""

from __future__ import annotations

import warnings
from typing import Sequence

import numpy as np

__all__ = ["capacitance_matrix", "resistance_matrix", "to_spice_matrix", "rlgc_2d",
           "characteristic_impedance", "check_lc_identity", "s_parameters", "y_to_z",
           "z_to_y", "elmore_delay", "skin_depth"]


def capacitance_matrix(grid, eps_cell: np.ndarray, terminals: Sequence,
                       bc=None, config=None, *, report: dict | None = None,
                       gpu=None) -> np.ndarray:
    """Maxwell capacitance matrix [F], shape ``(nt, nt)``.

    Unit excitation of every terminal in turn (all solved as one block of
    right-hand sides on the GPU), charge integrated on every terminal,
    symmetrised; the pre-symmetrisation asymmetry is in ``report``.
    """
    from .solvers.poisson import PoissonSolver
    # the permittivity upload and check overlap the terminal checks; a bad
    # eps_cell still raises before anything else is reported
    solver = PoissonSolver(grid, eps_cell, config, gpu=gpu, check_later=True)
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
                                     preconditioner=resolve_preconditioner(cfg, gcfg),
                                     coarsening=gcfg.coarsening, mg_params=gcfg.mg_params)
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


# ---------------------------------------------------------------------------
# Transmission lines (extraction.py:105-264)
# ---------------------------------------------------------------------------
def rlgc_2d(grid, eps_cell: np.ndarray, sigma_cell: np.ndarray, terminals: Sequence,
            mu_cell: np.ndarray | None = None, freq: float = 0.0, config=None,
            reference: int | str = -1, *, gpu=None) -> dict[str, np.ndarray]:
    """Per-unit-length R, L, G, C matrices of a 2-D cross-section (``grid.Nz
    == 1``, unit thickness in the collapsed direction), referenced to the
    return conductor ``reference`` (index or name; default the last), as
    ``extraction.py:108-206``.

    ``C`` (real permittivity), ``C_air`` (vacuum everywhere) and ``G``
    (conductivity in place of permittivity, floored at 1e-30 S/m) are three
    capacitance extractions on the same grid, solved as one batch on the GPU;
    ``L = mu_r mu0 eps0 C_air^-1`` by the TEM identity; ``R`` is the
    reference's DC (optionally skin-corrected) series-resistance estimate.
    Returns ``{"R", "L", "G", "C", "C_air", "eps_eff", "Z0", "v_p",
    "reference"}``, matrices ``(nt-1, nt-1)``.
    """
    from .batch import extract_local
    from .solvers.base import GPUConfig, SolverConfig
    from .units import eps0, mu0
    if grid.Nz != 1:
        raise ValueError("rlgc_2d needs a 2D cross-section (grid.Nz == 1)")
    terminals = list(terminals)
    nt = len(terminals)
    if nt < 2:
        raise ValueError(
            "rlgc_2d needs at least two conductors: one signal and one return")
    if isinstance(reference, str):
        names = [t.name for t in terminals]
        if reference not in names:
            raise ValueError(f"reference {reference!r} is not among {names}")
        ref_i = names.index(reference)
    else:
        ref_i = int(reference) % nt
    keep = [i for i in range(nt) if i != ref_i]
    eps_cell = np.asarray(eps_cell, dtype=float)
    sigma_cell = np.asarray(sigma_cell, dtype=float)
    lossy = bool(np.any(sigma_cell > 0))
    problems = [(grid, eps_cell, terminals), (grid, np.full_like(eps_cell, eps0), terminals)]
    if lossy:
        problems.append((grid, np.maximum(sigma_cell, 1e-30), terminals))
    mats = extract_local(problems, config or SolverConfig(), gpu or GPUConfig(),
                         len(problems), None)

    def _reduce(m: np.ndarray) -> np.ndarray:
        return np.asarray(m)[np.ix_(keep, keep)]

    C = _reduce(mats[0])
    C_air = _reduce(mats[1])
    mu_r = 1.0
    if mu_cell is not None:
        mu_r = float(np.mean(np.asarray(mu_cell, dtype=float)) / mu0)
    L = mu_r * mu0 * eps0 * np.linalg.inv(C_air)
    G = _reduce(mats[2]) if lossy else np.zeros_like(C)
    R = _series_resistance(grid, sigma_cell, [terminals[i] for i in keep], freq)
    eps_eff = np.diag(C) / np.diag(C_air)
    v_p = 1.0 / np.sqrt(np.diag(L) * np.diag(C))
    Z0 = np.sqrt(np.diag(L) / np.diag(C))
    return {"R": R, "L": L, "G": G, "C": C, "C_air": C_air, "eps_eff": eps_eff,
            "Z0": Z0, "v_p": v_p, "reference": terminals[ref_i].name}


def _series_resistance(grid, sigma_cell, terminals, freq) -> np.ndarray:
    """DC (or skin-corrected) series resistance per unit length [ohm/m]
    (``extraction.py:209-233``).

    The estimate is the reference's: the conducting cross-section ``A`` is
    the volume of every cell with sigma > 0 over the length along z, sigma
    their mean, ``R = 1 / (sigma A)``; above DC the current is confined to a
    skin of depth delta along a square perimeter ``4 sqrt(A)``, so the area
    used is ``min(A, 4 sqrt(A) delta)`` and R never drops below its DC value.
    Every conductor gets this same value on the diagonal."""
    nt = len(terminals)
    cond = np.asarray(sigma_cell) > 0
    length = float(grid.zn[-1] - grid.zn[0])
    if not cond.any() or length <= 0:
        return np.zeros((nt, nt))
    area = float(np.asarray(grid.cell_volumes())[cond].sum()) / length
    sigma = float(np.mean(np.asarray(sigma_cell)[cond]))
    if area <= 0 or sigma <= 0:
        return np.zeros((nt, nt))
    r = 1.0 / (sigma * area)
    if freq > 0:
        skin_area = min(area, 4.0 * np.sqrt(area) * skin_depth(sigma, freq))
        r = max(r, 1.0 / (sigma * max(skin_area, 1e-300)))
    return r * np.eye(nt)


def characteristic_impedance(rlgc: dict, freq=0.0) -> np.ndarray:
    """``Z0 = sqrt((R + jwL)/(G + jwC))`` [ohm]; lossless at ``freq=0``."""
    R, L, G, C = (np.atleast_2d(rlgc[k]) for k in ("R", "L", "G", "C"))
    w = 2.0 * np.pi * np.asarray(freq, dtype=float)
    if np.all(w == 0):
        return np.sqrt(np.diag(L) / np.diag(C))
    num = np.diag(R) + 1j * w[..., None] * np.diag(L)
    den = np.diag(G) + 1j * w[..., None] * np.diag(C)
    return np.sqrt(num / den)


def check_lc_identity(rlgc: dict, eps_r: float = 1.0, mu_r: float = 1.0) -> float:
    """Max relative deviation of ``L C`` from ``mu eps I`` (TEM identity)."""
    from .units import eps0, mu0
    L = np.atleast_2d(rlgc["L"])
    C = np.atleast_2d(rlgc["C"])
    target = mu_r * mu0 * eps_r * eps0 * np.eye(L.shape[0])
    scale = max(np.abs(target).max(), 1e-300)
    return float(np.abs(L @ C - target).max() / scale)


# ---------------------------------------------------------------------------
# Network parameters (extraction.py:267-317)
# ---------------------------------------------------------------------------
def y_to_z(y: np.ndarray) -> np.ndarray:
    """Admittance (or a stack of them) to impedance."""
    return np.linalg.inv(np.asarray(y))


def z_to_y(z: np.ndarray) -> np.ndarray:
    return np.linalg.inv(np.asarray(z))


def s_parameters(y: np.ndarray, z0=50.0) -> np.ndarray:
    """Scattering matrix of one ``(n, n)`` admittance or a stack
    ``(nf, n, n)`` for a real reference impedance (scalar or per port).

    With ``A = Z0 Y`` the scattering matrix is ``(I - A)(I + A)^-1``; both
    factors are polynomials in ``A`` and commute, so it is also
    ``(I + A)^-1 (I - A)``, computed here as one batched linear solve."""
    y = np.asarray(y)
    n = y.shape[-1]
    z = np.full(n, float(z0)) if np.isscalar(z0) else np.asarray(z0, float)
    A = z[:, None] * y                      # diag(z0) @ Y, broadcast over the stack
    eye = np.eye(n)
    return np.linalg.solve(eye + A, (eye - A).astype(complex))


def elmore_delay(r: np.ndarray, c: np.ndarray) -> float:
    """Elmore delay of an RC ladder, ``sum_i c_i sum_{j<=i} r_j`` [s]."""
    r = np.asarray(r, dtype=float)
    c = np.asarray(c, dtype=float)
    if r.shape != c.shape:
        raise ValueError("r and c must have the same shape")
    return float(np.sum(c * np.cumsum(r)))


def skin_depth(sigma: float, freq: float, mu_r: float = 1.0) -> float:
    """``sqrt(2/(omega mu sigma))`` [m]; infinite at ``freq <= 0``."""
    from .units import mu0
    if freq <= 0:
        return float("inf")
    return float(np.sqrt(2.0 / (2.0 * np.pi * freq * mu_r * mu0 * sigma)))
