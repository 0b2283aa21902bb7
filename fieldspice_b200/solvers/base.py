"""Problem and result types of the solve path.

These mirror ``fieldspice/solvers/base.py`` (``ConvergenceError`` :35-48,
``SolverConfig`` :51-82, ``Terminal`` :85-133, ``Result`` :136-202) so that a
caller of the reference can pass the same objects.  The reference's own
instances are accepted too: every function here reads them by attribute.
"""

from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import Any, Callable, Sequence

import numpy as np

__all__ = ["ConvergenceError", "SolverConfig", "GPUConfig", "Terminal", "Result",
           "resolve_preconditioner"]


class ConvergenceError(RuntimeError):
    """An iterative solve ended above its tolerance.

    ``history`` holds the final relative residuals; ``last_state`` the last
    iterate when one is available (``fieldspice/solvers/base.py:35-48``).
    """

    def __init__(self, msg: str, history: Sequence[float] = (),
                 last_state: np.ndarray | None = None):
        super().__init__(msg)
        self.history = list(history)
        self.last_state = last_state


@dataclass
class SolverConfig:
    """Shared solver knobs (same fields and defaults as the reference).

    ``linear_solver`` is accepted for compatibility; the GPU path always runs
    preconditioned CG on the eliminated system, so ``"direct"`` and ``"amg"``
    select the same GPU solve.  ``tol`` is the relative residual of the
    Jacobi-equilibrated free-node system, exactly SciPy's ``rtol`` in the
    reference (``fieldspice/solvers/poisson.py:542``).
    """
    linear_solver: str = "auto"
    tol: float = 1e-10
    newton_tol: float = 1e-8
    max_newton: int = 60
    damping: float = 1.0
    verbose: int = 0
    store_every: int = 1
    dtype: type = np.float64


@dataclass
class GPUConfig:
    """GPU-only knobs, kept apart from :class:`SolverConfig`.

    precision
        ``"mixed"``: FP32 inner CG with FP64 reliable updates (the residual
        that decides convergence is always FP64).  ``"fp64"``: every vector
        in FP64, the plain method.  ``"auto"`` (default): mixed, continuing
        in FP64 if the FP32 iterations stall on a mode below FP32 resolution
        (extreme conductivity contrast).
    preconditioner
        ``"jacobi"`` (CG on the equilibrated system, the reference's CG
        method), ``"mg"`` (a geometric-multigrid V-cycle as the CG
        preconditioner; same FP64 stopping rule), or ``None``: chosen from
        ``SolverConfig.linear_solver`` (:func:`resolve_preconditioner`).
        ``"learned"``: the multigrid V-cycle with its lower levels replaced
        by a trained U-Net (``learned``, a
        :class:`fieldspice_b200.learned.LearnedPreconditioner`) inside
        flexible CG, falling back to plain multigrid if FCG stalls.
    maxiter
        Iteration cap; ``None`` uses the reference's ``max(500, 10*sqrt(n))``
        (``poisson.py:535-536``).
    learned
        The trained network for ``preconditioner="learned"``.
    coarsening
        How the multigrid levels are built: ``"geometric"`` (every level a
        rediscretisation of the fine operator, trilinear transfers),
        ``"galerkin"`` (2x2x2 node aggregates, coarse operators ``P^T A P``:
        robust when conductors sit in insulators, e.g. copper in oxide at a
        1e6 conductance ratio) or ``"auto"`` (default): galerkin when the
        operator's edge masses span more than three orders of magnitude.
    mg_params
        Multigrid and stencil options of the plans this solver creates, as a
        dict of ``fs_mg_params`` fields (``smooth_deg``, ``smooth_lo``,
        ``coarse_deg``, ``coarse_lo``, ``coarsest_nodes``, ``stencil_kind``,
        ``agg_alpha``); None: the library defaults.  Each plan keeps its own
        copy.
    """
    precision: str = "auto"
    preconditioner: str | None = None
    maxiter: int | None = None
    learned: object | None = None
    coarsening: str = "auto"
    mg_params: dict | None = None


def resolve_preconditioner(cfg, gpu) -> str:
    """GPU preconditioner for a reference ``SolverConfig.linear_solver``.

    ``"cg"`` is the reference's Jacobi-preconditioned CG; ``"auto"``,
    ``"amg"`` and ``"direct"`` map to multigrid-preconditioned CG (the
    reference's ``"auto"`` path on large 3-D systems is AMG-preconditioned
    CG, ``fieldspice/solvers/poisson.py:391-398``).  An explicit
    ``GPUConfig.preconditioner`` wins.
    """
    if gpu is not None and gpu.preconditioner is not None:
        if gpu.preconditioner not in ("jacobi", "mg", "learned"):
            raise ValueError(f"unknown preconditioner {gpu.preconditioner!r}")
        if gpu.preconditioner == "learned" and getattr(gpu, "learned", None) is None:
            raise ValueError("preconditioner='learned' needs GPUConfig.learned "
                             "(a trained LearnedPreconditioner)")
        return gpu.preconditioner
    want = getattr(cfg, "linear_solver", "auto")
    if want not in ("auto", "direct", "cg", "amg"):
        raise ValueError(f"unknown linear_solver {want!r}; expected one of "
                         "'auto', 'direct', 'cg', 'amg'")
    return "jacobi" if want == "cg" else "mg"


@dataclass
class Terminal:
    """An electrode: a set of node indices held at a common potential.

    Same contract as ``fieldspice/solvers/base.py:85-133``: ``nodes`` is made
    unique and sorted, ``voltage`` or ``current`` may be a constant or a
    callable of time.
    """
    name: str
    nodes: np.ndarray
    voltage: float | Callable[[float], float] | None = None
    current: float | Callable[[float], float] | None = None
    circuit_node: str | None = None

    def __post_init__(self):
        self.nodes = np.unique(np.asarray(self.nodes, dtype=np.intp).ravel())
        if self.voltage is not None and self.current is not None:
            raise ValueError(
                f"terminal {self.name!r}: set voltage or current, not both")

    def value_at(self, t: float) -> float | None:
        src = self.voltage if self.voltage is not None else self.current
        if src is None:
            return None
        return float(src(t)) if callable(src) else float(src)

    @property
    def driven(self) -> str:
        if self.voltage is not None:
            return "voltage"
        if self.current is not None:
            return "current"
        return "float"


@dataclass
class Result:
    """Uniform output container (``fieldspice/solvers/base.py:136-202``)."""
    grid: Any
    t: np.ndarray = field(default_factory=lambda: np.zeros(0))
    fields: dict[str, np.ndarray] = field(default_factory=dict)
    terminals: dict[str, dict[str, np.ndarray]] = field(default_factory=dict)
    scalars: dict[str, np.ndarray] = field(default_factory=dict)
    meta: dict[str, Any] = field(default_factory=dict)

    def v(self, terminal: str) -> np.ndarray:
        return self.terminals[terminal]["v"]

    def i(self, terminal: str) -> np.ndarray:
        return self.terminals[terminal]["i"]

    def field(self, name: str, step: int = -1) -> np.ndarray:
        return self.fields[name][step]

    def final(self, name: str) -> np.ndarray:
        return self.fields[name][-1]


def terminal_driven(t) -> str:
    """``Terminal.driven`` for this module's or the reference's terminals."""
    return t.driven


class _Clock:
    """Wall-clock bookkeeping for ``Result.meta`` (base.py:228-237)."""

    def __init__(self):
        self.t0 = time.perf_counter()

    def elapsed(self) -> float:
        return time.perf_counter() - self.t0
