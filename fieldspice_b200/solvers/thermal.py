"""Fourier heat conduction on the GPU: ``C_th dT/dt + G^T M_kappa G T = Q``.

Drop-in for ``fieldspice/solvers/thermal.py``'s ``ThermalSolver``
(``:86-319``): same constructor, ``steady`` (fixed-temperature walls and
convective walls ``-kappa dT/dn = h (T - T_inf)``), ``transient`` (theta
scheme, backward Euler by default), ``thermal_resistance`` and ``solve``.

The operator is the electrostatic one with thermal-conductance masses plus a
node-diagonal term: convection ``h A_dual`` on wall nodes (steady) and the
heat capacity ``C_th / dt`` (transient).  The diagonal rides in the CG plan
(``fs_pcg_plan_create_diag``): it enters the classification and the FP64
residual and is restricted to the multigrid levels; the FP32 inner
iteration is unchanged because the equilibrated operator keeps a unit
diagonal.  Per transient step the explicit part ``(C/dt - (1-theta)(K +
D_conv)) T`` is one FP64 stencil apply plus a diagonal term on the device;
each step's CG starts from the previous temperature (same fixed point, same
stopping rule as the reference's cached factorisation).
"""

from __future__ import annotations

import time
import warnings
from typing import Callable, Mapping

import numpy as np

from .. import _lib as L
from ..boundaries import BoundarySpec, check_supported, dirichlet_nodes, wall_nodes
from ..device import DeviceOperator, EliminatedSystem, d2h, h2d
from ..grid import grid_metric
from .base import GPUConfig, Result, SolverConfig, resolve_preconditioner
from .poisson import raise_on_status

__all__ = ["ThermalSolver", "WALLS", "cell_to_node", "wall_dual_areas"]

WALLS = ("xlo", "xhi", "ylo", "yhi", "zlo", "zhi")


def cell_to_node(grid, prop) -> np.ndarray:
    """Dual-volume-weighted average of a per-cell property onto nodes, cells
    edge-padded (``operators.py:270-296``); shape ``grid.shape_nodes``."""
    prop = np.asarray(prop, dtype=float)
    (hx, hy, hz), _ = grid_metric(grid)
    p = np.pad(prop, 1, mode="edge")
    nx, ny, nz = (int(v) for v in grid.shape_nodes)
    acc = np.zeros((nx, ny, nz))
    wacc = np.zeros((nx, ny, nz))
    halves = [(np.concatenate([[0.0], 0.5 * h]), np.concatenate([0.5 * h, [0.0]]))
              for h in (hx, hy, hz)]
    for di in (0, 1):
        for dj in (0, 1):
            for dk in (0, 1):
                w = (halves[0][di][:, None, None] * halves[1][dj][None, :, None]
                     * halves[2][dk][None, None, :])
                acc += p[di:di + nx, dj:dj + ny, dk:dk + nz] * w
                wacc += w
    return acc / np.where(wacc > 0, wacc, 1.0)


def wall_dual_areas(grid, wall: str) -> np.ndarray:
    """Exposed dual face area of every node on a wall, in ``wall_nodes``
    order (``boundaries.py:200-218``)."""
    if wall not in WALLS:
        raise ValueError(f"unknown wall {wall!r}; expected one of {WALLS}")
    _, duals = grid_metric(grid)
    axis = {"x": 0, "y": 1, "z": 2}[wall[0]]
    d0, d1 = [d for d in (0, 1, 2) if d != axis]
    return (duals[d0][:, None] * duals[d1][None, :]).ravel()


class ThermalSolver:
    """Heat conduction (``thermal.py:86-140``): ``kappa_cell`` [W/(m K)],
    ``rho_cp_cell`` [J/(m^3 K)] (transient only); ``gpu`` selects precision
    and preconditioner."""

    name = "thermal"
    assumptions = ("A2", "A10")

    def __init__(self, grid, kappa_cell, rho_cp_cell=None, config: SolverConfig | None = None,
                 operators=None, *, gpu: GPUConfig | None = None):
        self.grid = grid
        self.cfg = config or SolverConfig()
        self.gpu = gpu or GPUConfig()
        kappa_cell = np.asarray(kappa_cell, dtype=float)
        if kappa_cell.shape != tuple(grid.shape_cells):
            raise ValueError(f"kappa_cell must have shape {tuple(grid.shape_cells)}, "
                             f"got {kappa_cell.shape}")
        if np.any(kappa_cell <= 0.0):
            raise ValueError(
                "kappa_cell must be strictly positive [W/(m K)]; a zero makes "
                "the heat equation singular in that region. Use a small "
                "positive floor for vacuum.")
        self.kappa_cell = kappa_cell
        self.op = DeviceOperator(grid, kappa_cell)
        _, (hxd, hyd, hzd) = grid_metric(grid)
        self.node_vol = (hxd[:, None, None] * hyd[None, :, None] * hzd[None, None, :]).ravel()
        if rho_cp_cell is not None:
            rho_cp_cell = np.asarray(rho_cp_cell, dtype=float)
            if rho_cp_cell.shape != tuple(grid.shape_cells):
                raise ValueError(f"rho_cp_cell must have shape {tuple(grid.shape_cells)}")
            if np.any(rho_cp_cell <= 0.0):
                raise ValueError("rho_cp_cell must be strictly positive")
            self.C_th = cell_to_node(grid, rho_cp_cell).ravel() * self.node_vol
        else:
            self.C_th = None
        self._K = None

    @property
    def K(self):
        """Thermal conductance matrix ``G^T M_kappa G`` [W/K] (host CSR, lazy)."""
        if self._K is None:
            from .poisson import assemble_csr
            self._K = assemble_csr(self.grid, self.op.edge_vector())
        return self._K

    # -- boundary terms ------------------------------------------------------------
    def _wall_terms(self, convection: Mapping[str, tuple[float, float]] | None):
        """Diagonal and right-hand-side contributions of convective walls
        (``thermal.py:142-160``)."""
        n = self.op.N
        diag = np.zeros(n)
        rhs = np.zeros(n)
        if not convection:
            return diag, rhs
        for wall, spec in convection.items():
            if wall not in WALLS:
                raise ValueError(f"unknown wall {wall!r}; expected one of {WALLS}")
            h, t_inf = float(spec[0]), float(spec[1])
            if h < 0.0:
                raise ValueError("heat transfer coefficient must be >= 0")
            nodes = wall_nodes(self.grid, wall)
            area = wall_dual_areas(self.grid, wall)
            np.add.at(diag, nodes, h * area)
            np.add.at(rhs, nodes, h * area * t_inf)
        return diag, rhs

    def _dirichlet(self, bc, t: float):
        if bc is None:
            return np.zeros(0, dtype=np.intp), np.zeros(0)
        check_supported(bc)
        idx, val = dirichlet_nodes(bc, self.grid, t)
        return np.asarray(idx, dtype=np.intp), np.asarray(val, dtype=float)

    def _system(self, op, fixed, diag):
        import torch
        dev = self.op.dev
        label = torch.zeros(self.op.N, dtype=torch.uint8, device=dev)
        fixed_d = h2d(fixed.astype(np.int64), torch.int64, dev)
        if fixed.size:
            label[fixed_d] = L.LABEL_FIXED
        system = EliminatedSystem(op, label, 1, precision=self.gpu.precision, with_source=True,
                                  preconditioner=resolve_preconditioner(self.cfg, self.gpu),
                                  diag=h2d(diag, torch.float64, dev),
                                  coarsening=self.gpu.coarsening,
                                  mg_params=self.gpu.mg_params)
        return system, fixed_d

    def _q(self, q_node) -> np.ndarray:
        n = self.op.N
        q = (np.full(n, float(q_node)) if np.isscalar(q_node)
             else np.asarray(q_node, dtype=float).ravel())
        if q.size == 1:
            q = np.full(n, float(q[0]))
        if q.size != n:
            raise ValueError(f"q_node must have {n} entries, got {q.size}")
        return q

    # -- steady --------------------------------------------------------------------
    def steady(self, q_node=0.0, bc=None,
               convection: Mapping[str, tuple[float, float]] | None = None) -> Result:
        """Steady-state temperature [K] (``thermal.py:200-245``)."""
        import torch
        t_wall = time.perf_counter()
        q = self._q(q_node)
        diag, rhs = self._wall_terms(convection)
        fixed, vals = self._dirichlet(bc, 0.0)
        if fixed.size == 0 and not np.any(diag):
            warnings.warn(
                "thermal problem has neither a fixed-temperature boundary nor "
                "convection: it is fully adiabatic, so with any net heat input "
                "there is no steady state and the solution is defined only up "
                "to an additive constant. Add a Dirichlet wall (a perfect heat "
                "sink) or a convection coefficient (a finite one).",
                RuntimeWarning, stacklevel=2)
        system, fixed_d = self._system(self.op, fixed, diag)
        dev = self.op.dev
        system.f.copy_(h2d(q + rhs, torch.float64, dev))
        if fixed.size:
            system.phi[fixed_d] = h2d(vals, torch.float64, dev)
        tol = float(self.cfg.tol)
        _, stats = system.solve(tol, self.gpu.maxiter)
        raise_on_status(stats, tol, "gpu-cg")
        T = d2h(system.phi[:self.op.N]).copy()
        system.close()
        res = Result(grid=self.grid, t=np.zeros(1), fields={"T": T[None, :]})
        res.scalars["power_in"] = np.array([float(q.sum())])
        res.scalars["T_max"] = np.array([float(T.max())])
        res.scalars["T_rise"] = np.array([float(T.max() - T.min())])
        res.meta.update(solver=self.name, assumptions=list(self.assumptions), mode="steady",
                        wall_time=time.perf_counter() - t_wall,
                        linear={"iterations": stats[0]["iterations"],
                                "relres_fp64": stats[0]["relres"],
                                "fp64_fallback": bool(system.fell_back)})
        return res

    # -- transient -----------------------------------------------------------------
    def transient(self, q_node, t_end: float, dt: float, T0=300.0, bc=None,
                  convection: Mapping[str, tuple[float, float]] | None = None,
                  theta: float = 1.0, store: bool = False, store_every: int = 1) -> Result:
        """Transient temperature [K], theta scheme (``thermal.py:247-300``)."""
        import torch
        if self.C_th is None:
            raise ValueError(
                "transient thermal solve needs rho_cp_cell; pass it to the "
                "constructor (rho * c_p per cell, J/(m^3 K))")
        if dt <= 0:
            raise ValueError("dt must be positive")
        if not 0.0 <= theta <= 1.0:
            raise ValueError("theta must lie in [0, 1]")
        t_wall = time.perf_counter()
        n_nodes = self.op.N
        T = (np.full(n_nodes, float(T0)) if np.isscalar(T0)
             else np.asarray(T0, dtype=float).copy())
        if T.shape != (n_nodes,):
            raise ValueError(f"T0 must have shape ({n_nodes},)")
        conv_diag, wall_rhs = self._wall_terms(convection)
        n = int(np.ceil(t_end / dt))
        times = dt * np.arange(n + 1)
        q_fn: Callable = q_node if callable(q_node) else (lambda t: q_node)
        dev = self.op.dev
        # implicit operator: theta K (masses) + C/dt + theta D_conv (diagonal);
        # explicit part: (C/dt - (1-theta) D_conv) T - (1-theta) K T
        op_imp = self.op.combine(theta, self.op, 0.0)
        op_exp = self.op.combine(-(1.0 - theta), self.op, 0.0)
        d_imp = self.C_th / dt + theta * conv_diag
        d_exp = h2d(self.C_th / dt - (1.0 - theta) * conv_diag, torch.float64, dev)
        wall_rhs_d = h2d(wall_rhs, torch.float64, dev)
        fixed, _ = self._dirichlet(bc, float(times[0]))
        system, fixed_d = self._system(op_imp, fixed, d_imp)
        system.phi.copy_(h2d(T, torch.float64, dev))
        prev = system.phi.clone()
        nx, ny, nz = self.op.shape
        lib = L.lib()
        tol = float(self.cfg.tol)
        t_max, t_mean = [float(T.max())], [float(T.mean())]
        stored = [T.copy()] if store else []
        iters = []
        for k in range(1, n + 1):
            t = float(times[k])
            f_fix, vals = self._dirichlet(bc, t)
            if not np.array_equal(f_fix, fixed):
                raise NotImplementedError(
                    "the set of fixed-temperature nodes changes during the run; the "
                    "GPU path keeps one eliminated system per run")
            prev.copy_(system.phi)
            q = self._q(q_fn(t))
            add = d_exp * prev + h2d(q, torch.float64, dev) + wall_rhs_d
            st = lib.fs_apply_laplacian(L.ptr(op_exp.mx), L.ptr(op_exp.my), L.ptr(op_exp.mz),
                                        L.ptr(prev), L.ptr(add), L.ptr(system.f),
                                        nx, ny, nz, 1, L.stream_ptr())
            L.check("fs_apply_laplacian", st)
            if fixed.size:
                system.phi[fixed_d] = h2d(vals, torch.float64, dev)
            _, stats = system.solve(tol, self.gpu.maxiter, warm=True)
            raise_on_status(stats, tol, "gpu-cg")
            iters.append(stats[0]["iterations"])
            Tk = system.phi[:n_nodes]
            t_max.append(float(Tk.max()))
            t_mean.append(float(Tk.mean()))
            if store and k % max(1, store_every) == 0:
                stored.append(d2h(Tk).copy())
        fell_back = bool(system.fell_back)
        system.close()
        res = Result(grid=self.grid, t=times)
        if store:
            res.fields["T"] = np.array(stored)
        res.scalars["T_max"] = np.array(t_max)
        res.scalars["T_mean"] = np.array(t_mean)
        res.meta.update(solver=self.name, assumptions=list(self.assumptions),
                        mode="transient", theta=theta, dt=dt, n_factorisations=1,
                        wall_time=time.perf_counter() - t_wall, iterations=iters,
                        warm_start=True, fp64_fallback=fell_back)
        return res

    def solve(self, q_node=0.0, t_end: float | None = None, dt: float | None = None,
              **kw) -> Result:
        """``steady`` without ``t_end``/``dt``, ``transient`` with them."""
        if t_end is None or dt is None:
            return self.steady(q_node, **kw)
        return self.transient(q_node, t_end, dt, **kw)

    def thermal_resistance(self, source_nodes, bc=None, convection=None,
                           power: float = 1.0) -> float:
        """Thermal resistance [K/W] from a node set to the boundary
        (``thermal.py:302-319``): ``power`` spread over the nodes by dual
        volume, mean temperature rise per watt."""
        q = np.zeros(self.op.N)
        nodes = np.asarray(source_nodes, dtype=np.intp).ravel()
        w = self.node_vol[nodes]
        w = w / w.sum() if w.sum() > 0 else np.full(nodes.size, 1.0 / nodes.size)
        q[nodes] = power * w
        T = self.steady(q, bc=bc, convection=convection).fields["T"][0]
        T_ref = 0.0
        if bc is not None:
            fixed, vals = self._dirichlet(bc, 0.0)
            if fixed.size:
                T_ref = float(np.mean(vals))
        return float((float(np.dot(w, T[nodes])) - T_ref) / power)
