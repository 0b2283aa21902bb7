"""fieldspice_b200: the elliptic solve path of fieldspice on NVIDIA B200.

``G^T M G phi = b`` -- Poisson capacitance extraction and the backward-Euler
electroquasistatic step -- solved matrix-free by hand-written sm_100a CUDA
kernels behind the reference's own Python entry points:

* :func:`fieldspice_b200.extraction.capacitance_matrix`,
  :func:`fieldspice_b200.extraction.resistance_matrix`
* :class:`fieldspice_b200.solvers.poisson.PoissonSolver`
* :class:`fieldspice_b200.solvers.eqs.EQSSolver`
* :class:`fieldspice_b200.solvers.thermal.ThermalSolver`
* :func:`fieldspice_b200.batch.capacitance_matrices` (many geometries)
* :class:`fieldspice_b200.learned.LearnedPreconditioner` (U-Net coarse-level
  correction on tensor cores inside flexible CG)

There is no CPU fallback: the CUDA library must be built and a GPU present.
"""

from . import units
from .boundaries import BoundarySpec, Dirichlet, Neumann, wall_nodes
from .grid import RectilinearGrid
from .solvers.base import ConvergenceError, GPUConfig, Result, SolverConfig, Terminal
from . import extraction, solvers  # noqa: E402
from .solvers import ac, eqs, poisson, thermal  # noqa: E402,F401
from . import batch, circuit, learned  # noqa: E402,F401

__version__ = "0.1.0"

__all__ = ["units", "BoundarySpec", "Dirichlet", "Neumann", "wall_nodes",
           "RectilinearGrid", "ConvergenceError", "GPUConfig", "Result",
           "SolverConfig", "Terminal", "extraction", "solvers", "batch", "learned"]
