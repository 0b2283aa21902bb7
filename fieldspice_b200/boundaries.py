"""Wall boundary conditions consumed by the elliptic path.

Mirrors ``fieldspice/boundaries.py``: :func:`wall_nodes` (``:154-198``) and
``BoundarySpec.dirichlet_nodes`` (``:963-1029``) with its precedence rule --
among Dirichlet-like walls the later wall in ``xlo, xhi, ylo, yhi, zlo, zhi``
wins on a shared node.  Dirichlet, homogeneous Neumann and symmetry walls
are supported on the GPU path; the reference's own ``BoundarySpec`` objects
are accepted as long as every wall is one of those (:func:`check_supported`).
A driven Neumann flux is the right-hand-side load of :func:`neumann_load`
(``BoundarySpec.neumann_load``, ``:1031-1085``), which the reference applies
in ``PoissonSolver.solve`` only (``poisson.py:957-964``).
"""

from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable

import numpy as np

__all__ = ["WALLS", "Dirichlet", "Neumann", "Periodic", "BoundarySpec", "wall_nodes",
           "wall_dual_areas", "dirichlet_nodes", "neumann_load", "check_supported",
           "periodic_mask"]

WALLS = ("xlo", "xhi", "ylo", "yhi", "zlo", "zhi")
_AXIS = {"xlo": 0, "xhi": 0, "ylo": 1, "yhi": 1, "zlo": 2, "zhi": 2}


@dataclass(frozen=True)
class Dirichlet:
    """Prescribed potential on a wall; ``value`` may be a callable of t."""
    value: float | Callable[[float], float] = 0.0

    is_dirichlet_like = True
    is_natural = False

    def prescribed_value(self, t: float = 0.0):
        v = self.value
        return np.asarray(v(t) if callable(v) else v, dtype=float)


@dataclass(frozen=True)
class Neumann:
    """Prescribed outward normal flux density (``boundaries.py:384-460``):
    ``J.n`` [A/m^2] with a conductance operator, ``D.n`` [C/m^2] with a
    capacitance one; a float, a 1-D array over the wall's nodes, or a
    callable of t.  ``0`` is the natural (homogeneous) condition and needs
    nothing; a driven flux enters ``PoissonSolver.solve``'s right-hand side
    through :func:`neumann_load`."""
    flux: float | Callable[[float], float] = 0.0

    is_dirichlet_like = False

    @property
    def is_natural(self) -> bool:
        return not callable(self.flux) and bool(np.all(np.asarray(self.flux, float) == 0.0))

    def flux_at(self, t: float = 0.0) -> np.ndarray:
        f = self.flux(float(t)) if callable(self.flux) else self.flux
        arr = np.asarray(f, dtype=float)
        if arr.ndim > 1:
            raise ValueError(f"Neumann flux must be scalar or 1-D, got shape {arr.shape}")
        if not np.all(np.isfinite(arr)):
            raise ValueError(f"Neumann flux is not finite at t = {t} s")
        return arr

    def prescribed_value(self, t: float = 0.0):
        return None


@dataclass(frozen=True)
class Periodic:
    """Wrap-around identification of the two walls normal to an axis
    (``fieldspice/boundaries.py:462-523``); set it on both walls.  The
    electrostatic path supports ``offset = 0`` and ``phase = 0`` only, as
    the reference's ``PoissonSolver`` does (``poisson.py:942-955``)."""
    offset: float = 0.0
    phase: float = 0.0

    is_dirichlet_like = False
    is_natural = False
    kind = "periodic"

    def prescribed_value(self, t: float = 0.0):
        return None


@dataclass
class BoundarySpec:
    """Six walls, homogeneous Neumann by default."""
    xlo: object = field(default_factory=Neumann)
    xhi: object = field(default_factory=Neumann)
    ylo: object = field(default_factory=Neumann)
    yhi: object = field(default_factory=Neumann)
    zlo: object = field(default_factory=Neumann)
    zhi: object = field(default_factory=Neumann)

    @classmethod
    def all_neumann(cls, grid=None) -> "BoundarySpec":
        return cls()

    def get(self, wall: str):
        return getattr(self, wall)

    def dirichlet_nodes(self, grid, t: float = 0.0):
        return dirichlet_nodes(self, grid, t)


def _wall(spec, w: str):
    return spec.get(w) if hasattr(spec, "get") else getattr(spec, w)


def wall_nodes(grid, wall: str) -> np.ndarray:
    """Ascending flat indices of the nodes on one wall (boundaries.py:154-198)."""
    if wall not in _AXIS:
        raise ValueError(f"unknown wall {wall!r}; expected one of {WALLS}")
    shape = tuple(int(s) for s in grid.shape_nodes)
    strides = (shape[1] * shape[2], shape[2], 1)
    axis = _AXIS[wall]
    plane = 0 if wall.endswith("lo") else shape[axis] - 1
    d0, d1 = [d for d in (0, 1, 2) if d != axis]
    a = np.arange(shape[d0], dtype=np.intp) * strides[d0]
    b = np.arange(shape[d1], dtype=np.intp) * strides[d1]
    return (plane * strides[axis] + a[:, None] + b[None, :]).ravel()


def periodic_mask(spec) -> int:
    """Bit mask of the periodic axes (bit 0 x, 1 y, 2 z).  Periodic must be set
    on both walls of an axis (``boundaries.py:1111-1125``)."""
    mask = 0
    for a, (lo, hi) in enumerate((("xlo", "xhi"), ("ylo", "yhi"), ("zlo", "zhi"))):
        plo = type(_wall(spec, lo)).__name__.lower() == "periodic"
        phi_ = type(_wall(spec, hi)).__name__.lower() == "periodic"
        if plo != phi_:
            raise ValueError(f"axis {'xyz'[a]}: Periodic must be set on both walls "
                             f"({lo} and {hi})")
        if plo:
            mask |= 1 << a
    return mask


def check_supported(spec, allow_periodic: bool = False) -> None:
    """Reject walls the GPU path does not implement, with a clear error.

    Periodic walls (the node-merging reduction of
    ``fieldspice/solvers/poisson.py:665-719``) are accepted where the caller
    implements them (``allow_periodic``: the electrostatic solve and
    capacitance extraction) with zero offset and phase; absorbing walls have
    no quasi-static meaning, and a Neumann wall with non-zero flux needs the
    ``neumann_load`` right-hand side (``boundaries.py:1031-1085``).
    """
    if allow_periodic:
        periodic_mask(spec)  # both walls of a periodic axis
    for w in WALLS:
        bc = _wall(spec, w)
        kind = type(bc).__name__.lower()
        if kind == "periodic" and allow_periodic:
            for nm in ("offset", "phase"):
                if float(getattr(bc, nm, 0.0)) != 0.0:
                    raise ValueError(
                        f"wall {w}: PoissonSolver supports periodic boundaries only "
                        f"with {nm} = 0; impose the drop with a driven terminal instead")
            continue
        if getattr(bc, "is_dirichlet_like", False):
            continue  # Dirichlet, or a PEC symmetry wall at its value
        if kind == "neumann":
            continue  # homogeneous, or a driven flux load (neumann_load)
        if getattr(bc, "is_natural", False) and kind != "periodic":
            continue  # PMC symmetry: the natural zero-flux condition
        raise NotImplementedError(
            f"wall {w}: {type(bc).__name__} walls are not supported on the GPU "
            "path (Dirichlet, Neumann and symmetry walls only)")


def dirichlet_nodes(spec, grid, t: float = 0.0):
    """Fixed wall nodes and values; the later wall wins on a shared node.

    Same precedence as ``BoundarySpec.dirichlet_nodes``
    (``fieldspice/boundaries.py:963-1029``): indices ascending and unique.
    """
    idx_parts, val_parts = [], []
    for w in WALLS:
        bc = _wall(spec, w)
        if not getattr(bc, "is_dirichlet_like", False):
            continue
        v = bc.prescribed_value(t)
        if v is None:
            raise ValueError(f"wall {w}: {type(bc).__name__} claims to be "
                             "Dirichlet-like but prescribes no value")
        idx = wall_nodes(grid, w)
        vals = np.broadcast_to(np.asarray(v, dtype=float), idx.shape).astype(float)
        idx_parts.append(idx)
        val_parts.append(vals)
    if not idx_parts:
        return np.empty(0, dtype=np.intp), np.empty(0, dtype=float)
    if len(idx_parts) == 1:  # one wall: its nodes are ascending and unique already
        return idx_parts[0], val_parts[0]
    idx_all = np.concatenate(idx_parts)
    val_all = np.concatenate(val_parts)
    uniq, first_in_rev = np.unique(idx_all[::-1], return_index=True)
    return uniq.astype(np.intp, copy=False), val_all[::-1][first_in_rev]


def wall_dual_areas(grid, wall: str) -> np.ndarray:
    """Dual-face area of each wall node, in :func:`wall_nodes` order: the
    product of the two in-plane dual widths (half widths at the edges)."""
    if wall not in _AXIS:
        raise ValueError(f"unknown wall {wall!r}; expected one of {WALLS}")
    hd = [np.asarray(grid.hxd, float), np.asarray(grid.hyd, float),
          np.asarray(grid.hzd, float)]
    d0, d1 = [d for d in (0, 1, 2) if d != _AXIS[wall]]
    return (hd[d0][:, None] * hd[d1][None, :]).ravel()


def neumann_load(spec, grid, t: float = 0.0):
    """Right-hand-side load of the driven Neumann walls, or ``None`` when
    every Neumann wall is homogeneous (``boundaries.py:1031-1085``): the
    outward flux density times each wall node's dual-face area, with a minus
    sign (KCL: ``L phi = q - flux * A``); walls add on shared edge and corner
    nodes, and Dirichlet wall nodes get no load."""
    load = None
    for w in WALLS:
        bc = _wall(spec, w)
        if type(bc).__name__.lower() != "neumann" or getattr(bc, "is_natural", True):
            continue
        idx = wall_nodes(grid, w)
        try:
            f = np.broadcast_to(bc.flux_at(t), idx.shape)
        except ValueError as exc:
            raise ValueError(f"wall {w}: Neumann flux of shape {np.shape(bc.flux_at(t))} "
                             f"cannot be broadcast to the {idx.size} nodes on that "
                             "wall") from exc
        if load is None:
            load = np.zeros(int(np.prod(grid.shape_nodes)))
        load[idx] += -f * wall_dual_areas(grid, w)
    if load is not None:
        fixed, _ = dirichlet_nodes(spec, grid, t)
        load[fixed] = 0.0
    return load
