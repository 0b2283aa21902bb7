"""Rectilinear node grid: the metric inputs of the elliptic path.

Mirrors the parts of ``fieldspice/grid.py`` the solve consumes: node
coordinates per axis, primal widths ``h`` and dual widths ``hd`` (half cells
at the walls, ``grid.py:196-207``), the node/cell/edge shapes (``:295-339``)
and the node (dual box) volumes (``:388-396``).  Any object exposing
``xn, yn, zn`` (or ``hx, hy, hz``) and ``shape_nodes`` -- the reference's
``RectilinearGrid`` included -- is accepted wherever a grid is expected.
"""

from __future__ import annotations

from typing import Sequence

import numpy as np

__all__ = ["RectilinearGrid", "axis_metric", "grid_metric"]


def axis_metric(nodes: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
    """Primal widths ``h`` and dual widths ``hd`` of one axis.

    Same arithmetic as ``fieldspice/grid.py:196-207`` so that masses built
    from them are bit-identical to the reference's.
    """
    nodes = np.asarray(nodes, dtype=float).ravel()
    h = np.diff(nodes)
    hd = np.empty(nodes.size)
    hd[1:-1] = 0.5 * (h[:-1] + h[1:])
    hd[0] = 0.5 * h[0]
    hd[-1] = 0.5 * h[-1]
    return h, hd


def grid_metric(grid) -> tuple[tuple[np.ndarray, ...], tuple[np.ndarray, ...]]:
    """``((hx, hy, hz), (hxd, hyd, hzd))`` for this package's or the
    reference's grid (both expose ``hx`` and ``hxd``)."""
    return ((np.asarray(grid.hx, float), np.asarray(grid.hy, float),
             np.asarray(grid.hz, float)),
            (np.asarray(grid.hxd, float), np.asarray(grid.hyd, float),
             np.asarray(grid.hzd, float)))


class RectilinearGrid:
    """Axis-aligned tensor-product grid (``fieldspice/grid.py:210-546``).

    ``x, y, z`` are node coordinates; ``None`` makes a collapsed direction of
    extent ``thickness[d]`` with two node planes, as in the reference.
    """

    def __init__(self, x, y=None, z=None,
                 thickness: tuple[float, float, float] = (1.0, 1.0, 1.0)):
        axes = []
        for a, th in zip((x, y, z), thickness):
            if a is None:
                nodes = np.array([0.0, float(th)])
            else:
                nodes = np.asarray(a, dtype=float).ravel()
                if nodes.size < 2:
                    raise ValueError("an axis needs at least 2 node coordinates")
                if np.any(np.diff(nodes) <= 0):
                    raise ValueError("node coordinates must be strictly increasing")
            axes.append(nodes)
        self.xn, self.yn, self.zn = axes
        (self.hx, self.hy, self.hz) = (np.diff(a) for a in axes)
        (self.hxd, self.hyd, self.hzd) = (axis_metric(a)[1] for a in axes)

    @classmethod
    def uniform(cls, extent: Sequence[tuple[float, float]], n: Sequence[int],
                thickness: tuple[float, float, float] = (1.0, 1.0, 1.0)
                ) -> "RectilinearGrid":
        axes: list[np.ndarray | None] = [None, None, None]
        for d, (ext, ncell) in enumerate(zip(extent, n)):
            axes[d] = np.linspace(ext[0], ext[1], int(ncell) + 1)
        return cls(axes[0], axes[1], axes[2], thickness=thickness)

    @property
    def Nx(self) -> int: return self.hx.size

    @property
    def Ny(self) -> int: return self.hy.size

    @property
    def Nz(self) -> int: return self.hz.size

    @property
    def ncell(self) -> tuple[int, int, int]:
        return (self.Nx, self.Ny, self.Nz)

    @property
    def shape_nodes(self) -> tuple[int, int, int]:
        return (self.Nx + 1, self.Ny + 1, self.Nz + 1)

    @property
    def shape_cells(self) -> tuple[int, int, int]:
        return (self.Nx, self.Ny, self.Nz)

    @property
    def shape_edges(self):
        return ((self.Nx, self.Ny + 1, self.Nz + 1),
                (self.Nx + 1, self.Ny, self.Nz + 1),
                (self.Nx + 1, self.Ny + 1, self.Nz))

    @property
    def n_nodes(self) -> int:
        return int(np.prod(self.shape_nodes))

    @property
    def n_cells(self) -> int:
        return int(np.prod(self.shape_cells))

    @property
    def n_edges_each(self):
        return tuple(int(np.prod(s)) for s in self.shape_edges)

    @property
    def n_edges(self) -> int:
        return int(sum(self.n_edges_each))

    @property
    def xc(self) -> np.ndarray: return 0.5 * (self.xn[:-1] + self.xn[1:])

    @property
    def yc(self) -> np.ndarray: return 0.5 * (self.yn[:-1] + self.yn[1:])

    @property
    def zc(self) -> np.ndarray: return 0.5 * (self.zn[:-1] + self.zn[1:])

    def cell_volumes(self) -> np.ndarray:
        """Primal cell volumes, shape ``shape_cells`` (grid.py:383-386)."""
        return (self.hx[:, None, None] * self.hy[None, :, None]
                * self.hz[None, None, :])

    def node_volumes(self) -> np.ndarray:
        """Dual box volumes, shape ``shape_nodes`` (grid.py:388-396)."""
        return (self.hxd[:, None, None] * self.hyd[None, :, None]
                * self.hzd[None, None, :])

    def courant_dt(self, eps_r_min: float = 1.0, mu_r_min: float = 1.0) -> float:
        """Explicit-FDTD step bound, for ``speedup_vs_courant`` (grid.py:467-486)."""
        from .units import c0
        v = 1.0 / np.sqrt(eps_r_min * mu_r_min)
        inv2 = 0.0
        for h in (self.hx, self.hy, self.hz):
            if h.size > 1:
                inv2 += 1.0 / float(h.min()) ** 2
        if inv2 == 0.0:
            inv2 = 1.0 / float(self.hx.min()) ** 2
        return 1.0 / (c0 * v * np.sqrt(inv2))

    def __repr__(self) -> str:
        nx, ny, nz = self.ncell
        return f"<RectilinearGrid {nx}x{ny}x{nz}, {self.n_nodes:,} nodes>"
