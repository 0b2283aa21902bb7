"""Seeded synthetic workloads of the elliptic path.

Every generator returns plain arrays (node coordinates, per-cell material,
terminal node lists, Dirichlet walls) so that this package, the CPU oracle
and the reference itself can be fed byte-identical inputs.

* :func:`parallel_plate` -- the README capacitor: 2 x 5 x 4 um, 24 x 10 x 8
  cells, SiO2, plates on the x = 0 and x = last node planes.
* :func:`layered_boxes` -- the extraction benchmark family: a uniform grid
  (10 nm pitch), three dielectric layers stacked in z, rectangular
  conductor boxes placed without overlap (1-node gap, never on z = 0), each a
  terminal, the bottom plane grounded.  At 256 x 256 x 128 nodes with eight
  boxes this is the 8-terminal extraction the throughput is quoted on.
* :func:`batch_geometries` -- 64 uneven geometries of the same family.
* :func:`eqs_interconnect` -- copper boxes in oxide over doped silicon for
  the backward-Euler EQS transient.
* :func:`cross_section` -- a 2-D transmission-line cross-section (collapsed
  z, two node planes): coupled microstrips on a two-layer substrate over a
  ground plane, air above, for ``rlgc_2d``.
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .units import eps0

__all__ = ["Workload", "parallel_plate", "layered_boxes", "batch_geometries",
           "eqs_interconnect", "cross_section", "ramp"]

SIO2 = 3.9


@dataclass
class Workload:
    """Inputs of one extraction or transient, as plain arrays."""
    name: str
    x: np.ndarray
    y: np.ndarray
    z: np.ndarray
    eps_cell: np.ndarray                       # absolute [F/m]
    terminals: list[np.ndarray]                # node index arrays
    names: list[str]
    dirichlet_walls: dict[str, float] = field(default_factory=dict)
    sigma_cell: np.ndarray | None = None       # [S/m] for EQS
    boxes: list[tuple[int, ...]] = field(default_factory=list)
    meta: dict = field(default_factory=dict)

    @property
    def shape_nodes(self) -> tuple[int, int, int]:
        return (self.x.size, self.y.size, self.z.size)

    @property
    def n_nodes(self) -> int:
        return int(np.prod(self.shape_nodes))

    def grid(self):
        from .grid import RectilinearGrid
        return RectilinearGrid(self.x, self.y, self.z)

    def terminal_objects(self, voltages=None):
        from .solvers.base import Terminal
        out = []
        for i, (nm, nodes) in enumerate(zip(self.names, self.terminals)):
            v = None if voltages is None else voltages[i]
            out.append(Terminal(nm, nodes, voltage=v))
        return out

    def boundary_spec(self):
        from .boundaries import BoundarySpec, Dirichlet
        kw = {w: Dirichlet(v) for w, v in self.dirichlet_walls.items()}
        return BoundarySpec(**kw)


def parallel_plate() -> Workload:
    """README case: C[0,0] must equal eps*A/d to 1e-12 (README.md:17-31)."""
    x = np.linspace(0, 2e-6, 25)
    y = np.linspace(0, 5e-6, 11)
    z = np.linspace(0, 4e-6, 9)
    eps = np.full((24, 10, 8), SIO2 * eps0)
    nid = np.arange(25 * 11 * 9).reshape(25, 11, 9)
    return Workload("parallel_plate", x, y, z, eps,
                    [nid[0].ravel(), nid[-1].ravel()], ["top", "bottom"],
                    meta={"C_ref": SIO2 * eps0 * 5e-6 * 4e-6 / 2e-6})


def _place_boxes(rng, shape, nbox, ext_xy, ext_z, gap=1, tries=10000):
    """Non-overlapping boxes (node-index extents), 1-node gap, z0 >= 1."""
    nx, ny, nz = shape
    boxes = []
    for _ in range(nbox):
        for _t in range(tries):
            ex = int(rng.integers(ext_xy[0], ext_xy[1] + 1))
            ey = int(rng.integers(ext_xy[0], ext_xy[1] + 1))
            ez = int(rng.integers(ext_z[0], ext_z[1] + 1))
            ex, ey, ez = min(ex, nx - 2), min(ey, ny - 2), min(ez, nz - 2)
            x0 = int(rng.integers(0, nx - ex + 1))
            y0 = int(rng.integers(0, ny - ey + 1))
            z0 = int(rng.integers(1, nz - ez + 1))
            ok = True
            for (a0, b0, c0, a1, b1, c1) in boxes:
                if (x0 < a1 + gap + 1 and a0 < x0 + ex + gap + 1 and
                        y0 < b1 + gap + 1 and b0 < y0 + ey + gap + 1 and
                        z0 < c1 + gap + 1 and c0 < z0 + ez + gap + 1):
                    ok = False
                    break
            if ok:
                boxes.append((x0, y0, z0, x0 + ex - 1, y0 + ey - 1, z0 + ez - 1))
                break
        else:
            raise RuntimeError(f"could not place box {len(boxes)} of {nbox}")
    return boxes


def _layers(rng, ncz, min_cells):
    """Two interface cell planes with every layer >= min_cells thick."""
    lo = min_cells
    z1 = int(rng.integers(lo, max(lo + 1, ncz - 2 * min_cells + 1)))
    z2 = int(rng.integers(z1 + min_cells, max(z1 + min_cells + 1, ncz - min_cells + 1)))
    return z1, z2


def layered_boxes(shape=(256, 256, 128), nbox=8, seed=0, pitch=10e-9,
                  eps_r=(3.9, 2.5, 7.0), ext_xy=(8, 64), ext_z=(4, 12),
                  min_layer_cells=8) -> Workload:
    """The extraction family: layered dielectric, conductor boxes, zlo at 0 V.

    For node shapes smaller than 256 x 256 x 128 the box extents scale with
    the grid so that the same number of boxes fits.
    """
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    sxy = min(nx, ny) / 256.0
    sz = nz / 128.0
    exy = (max(2, int(round(ext_xy[0] * sxy))), max(2, int(round(ext_xy[1] * sxy))))
    ez = (max(2, int(round(ext_z[0] * sz))), max(2, int(round(ext_z[1] * sz))))
    mlc = max(2, int(round(min_layer_cells * sz)))
    x = np.arange(nx) * pitch
    y = np.arange(ny) * pitch
    z = np.arange(nz) * pitch
    z1, z2 = _layers(rng, nz - 1, mlc)
    eps = np.empty((nx - 1, ny - 1, nz - 1))
    eps[:, :, :z1] = eps_r[0] * eps0
    eps[:, :, z1:z2] = eps_r[1] * eps0
    eps[:, :, z2:] = eps_r[2] * eps0
    boxes = _place_boxes(rng, shape, nbox, exy, ez)
    nid = np.arange(nx * ny * nz).reshape(shape)
    terms = [nid[a0:a1 + 1, b0:b1 + 1, c0:c1 + 1].ravel()
             for (a0, b0, c0, a1, b1, c1) in boxes]
    return Workload(f"layered_boxes_{nx}x{ny}x{nz}_k{nbox}_s{seed}", x, y, z, eps,
                    terms, [f"box{i}" for i in range(nbox)], {"zlo": 0.0},
                    boxes=boxes, meta={"z_interfaces": (z1, z2), "seed": seed})


def batch_geometries(count=64, seed=0, lo=(32, 32, 32), hi=(160, 160, 96),
                     eps_choices=(2.5, 3.9, 7.0, 11.7)) -> list[Workload]:
    """Uneven batch: node counts log-uniform between prod(lo) and prod(hi),
    aspect near hi's, 2-16 boxes, per-layer eps_r drawn from eps_choices."""
    rng = np.random.default_rng(seed)
    out = []
    nlo, nhi = float(np.prod(lo)), float(np.prod(hi))
    ax = np.asarray(hi, float) / np.cbrt(nhi)
    for g in range(count):
        ntot = math.exp(rng.uniform(math.log(nlo), math.log(nhi)))
        s = np.cbrt(ntot)
        shape = tuple(int(max(l, round(a * s))) for a, l in zip(ax, (24, 24, 20)))
        nbox = int(rng.integers(2, 17))
        er = tuple(float(rng.choice(eps_choices)) for _ in range(3))
        ext_xy = (max(2, shape[0] // 32), max(3, shape[0] // 6))
        ext_z = (2, max(3, shape[2] // 10))
        w = layered_boxes(shape, nbox=nbox, seed=int(rng.integers(1 << 31)),
                          eps_r=er, ext_xy=(ext_xy[0] * 256 // shape[0],
                                            ext_xy[1] * 256 // shape[0]),
                          ext_z=(ext_z[0] * 128 // shape[2], ext_z[1] * 128 // shape[2]))
        w.name = f"batch{g}_{w.name}"
        out.append(w)
    return out


def ramp(t0: float, v0: float, v1: float, trise: float):
    """Linear edge from v0 to v1 starting at t0 over trise (the waveform of
    ``sources.step(t0, v0, v1, trise)``, sources.py:352-395)."""
    def f(t):
        if trise <= 0.0:
            return v1 if t >= t0 else v0
        a = min(max((t - t0) / trise, 0.0), 1.0)
        return v0 + (v1 - v0) * a
    return f


def eqs_interconnect(shape=(192, 192, 96), nbox=6, nports=2, seed=0,
                     pitch=10e-9, si_cells=24) -> Workload:
    """Copper boxes (5.8e7 S/m, eps_r 1) in oxide (1e-12 S/m, eps_r 3.9)
    above doped silicon (1e2 S/m, eps_r 11.7); the first ``nports`` boxes
    are driven terminals, zlo at 0 V."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    sxy = min(nx, ny) / 256.0
    sz = nz / 128.0
    exy = (max(2, int(round(8 * sxy))), max(3, int(round(64 * sxy))))
    ez = (max(2, int(round(4 * sz))), max(3, int(round(12 * sz))))
    si = min(si_cells, nz - 4)
    x = np.arange(nx) * pitch
    y = np.arange(ny) * pitch
    z = np.arange(nz) * pitch
    eps = np.full((nx - 1, ny - 1, nz - 1), 3.9 * eps0)
    sig = np.full((nx - 1, ny - 1, nz - 1), 1e-12)
    eps[:, :, :si] = 11.7 * eps0
    sig[:, :, :si] = 1e2
    # boxes in the oxide: z0 above the silicon
    boxes = []
    sub = _place_boxes(rng, (nx, ny, nz - si), nbox, exy, ez)
    for (a0, b0, c0, a1, b1, c1) in sub:
        boxes.append((a0, b0, c0 + si, a1, b1, c1 + si))
    for (a0, b0, c0, a1, b1, c1) in boxes:
        # copper cells: those whose 8 corners are all box nodes
        if a1 > a0 and b1 > b0 and c1 > c0:
            eps[a0:a1, b0:b1, c0:c1] = 1.0 * eps0
            sig[a0:a1, b0:b1, c0:c1] = 5.8e7
    nid = np.arange(nx * ny * nz).reshape(shape)
    terms = [nid[a0:a1 + 1, b0:b1 + 1, c0:c1 + 1].ravel()
             for (a0, b0, c0, a1, b1, c1) in boxes[:nports]]
    return Workload(f"eqs_{nx}x{ny}x{nz}_s{seed}", x, y, z, eps, terms,
                    [f"port{i}" for i in range(nports)], {"zlo": 0.0},
                    sigma_cell=sig, boxes=boxes, meta={"seed": seed, "si_cells": si})


def cross_section(nx: int = 301, ny: int = 201, width: float = 60e-6,
                  height: float = 40e-6, nlines: int = 2, seed: int = 0) -> Workload:
    """Coupled microstrips: ``nlines`` traces (6 um wide, 1 um thick, seeded
    gaps) on a 12 um substrate (eps_r 4.4, sigma 1e-3 S/m) under a 2 um
    solder mask (eps_r 3.0), air above, a ground plane on the bottom node
    row; uniform ``nx x ny`` nodes, z collapsed (two planes, 1 m apart).
    Terminals: the traces, then the ground; each holds both z planes."""
    rng = np.random.default_rng(seed)
    x = np.linspace(0.0, width, nx)
    y = np.linspace(0.0, height, ny)
    z = np.array([0.0, 1.0])
    xc = 0.5 * (x[:-1] + x[1:])
    yc = 0.5 * (y[:-1] + y[1:])
    X, Y = np.meshgrid(xc, yc, indexing="ij")
    eps = np.full((nx - 1, ny - 1, 1), eps0)
    sig = np.zeros((nx - 1, ny - 1, 1))
    sub = Y < 0.3 * height
    eps[sub] = 4.4 * eps0
    sig[sub] = 1e-3
    mask = (Y >= 0.3 * height) & (Y < 0.35 * height)
    eps[mask] = 3.0 * eps0
    nid = np.arange(nx * ny * 2).reshape(nx, ny, 2)

    def box(x0, x1, y0, y1):
        i = np.flatnonzero((x >= x0) & (x <= x1))
        j = np.flatnonzero((y >= y0) & (y <= y1))
        return nid[i[0]:i[-1] + 1, j[0]:j[-1] + 1, :].ravel()
    wl, t = 0.1 * width, 0.025 * height
    gaps = rng.uniform(0.5, 1.5, max(0, nlines - 1)) * wl
    span = nlines * wl + gaps.sum()
    x0 = 0.5 * (width - span)
    terms, names = [], []
    y0 = 0.3 * height
    for k in range(nlines):
        terms.append(box(x0, x0 + wl, y0, y0 + t))
        names.append(f"line{k}")
        x0 += wl + (gaps[k] if k < nlines - 1 else 0.0)
    terms.append(box(0.0, width, 0.0, 0.0))
    names.append("gnd")
    w = Workload(f"cross_section_{nx}x{ny}", x, y, z, eps, terms, names,
                 sigma_cell=sig)
    return w
