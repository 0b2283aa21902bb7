"""Electrostatics on the GPU: ``G^T M_eps G phi = q`` and capacitance extraction.

Drop-in for ``fieldspice/solvers/poisson.py``'s ``PoissonSolver``
(``:793-1281``): same constructor, same ``capacitance_matrix`` /
``spice_capacitance_matrix`` / ``solve`` / ``energy`` / ``node_charge``
signatures, same input checks and the same report keys.  The assembled CSR
and SciPy solve are replaced by the device operator and the matrix-free CG
plan of ``libfieldspice_b200``; results are FP64 and the convergence test is
the reference's (relative residual of the equilibrated free-node system).
"""

from __future__ import annotations

import ctypes
import time
import warnings
from typing import Any, Sequence

import numpy as np

from .. import _lib as L
from ..boundaries import (BoundarySpec, check_supported, dirichlet_nodes, neumann_load,
                          periodic_mask)
from ..device import (DeviceOperator, EliminatedSystem, block_rhs, d2h, h2d, mark,
                      pad_rhs, rhs_blocks, upload_groups)
from .base import ConvergenceError, GPUConfig, Result, SolverConfig, resolve_preconditioner

__all__ = ["PoissonSolver", "check_terminals", "as_cell_array", "raise_on_status",
           "upload_cell_property", "shield_nodes"]


def as_cell_array(a, grid, name: str) -> np.ndarray:
    """Shape and finiteness checks of ``poisson.py:733-742``."""
    arr = np.asarray(a, dtype=float)
    if arr.shape == ():
        arr = np.full(grid.shape_cells, float(arr))
    if arr.shape != tuple(grid.shape_cells):
        raise ValueError(f"{name} must have shape {tuple(grid.shape_cells)}, "
                         f"got {arr.shape}")
    if not np.all(np.isfinite(arr)):
        raise ValueError(f"{name} contains non-finite values")
    return arr


def upload_cell_property(a, grid, name: str, *, wait: bool = True):
    """The checks of ``as_cell_array`` with the pass over the values on the
    device: shape on the host, then one upload and one device reduction for
    non-finite entries, min and max.  Returns ``(host array, device tensor,
    min, max)``.

    ``wait=False`` returns ``(host array, device tensor, pending)`` at once:
    the upload (asynchronous from page-locked memory) and the reduction are
    enqueued, and ``cell_property_range(pending, name)`` later waits for them
    and raises as the eager form does, so the host can work meanwhile."""
    import torch
    from ..device import TRANSFERS, device
    arr = np.asarray(a, dtype=float)
    if arr.shape == ():
        arr = np.full(grid.shape_cells, float(arr))
    if arr.shape != tuple(grid.shape_cells):
        raise ValueError(f"{name} must have shape {tuple(grid.shape_cells)}, "
                         f"got {arr.shape}")
    src = torch.as_tensor(arr)
    dev = torch.empty(arr.shape, dtype=torch.float64, device=device())
    dev.copy_(src, non_blocking=True)
    TRANSFERS["h2d"] += arr.nbytes
    pending = L.prop_stats_begin(dev)
    if not wait:
        return arr, dev, pending
    lo, hi = cell_property_range(pending, name)
    return arr, dev, lo, hi


def cell_property_range(pending, name: str) -> tuple[float, float]:
    """(min, max) of an uploaded cell property; raises on non-finite values."""
    lo, hi, bad = pending.result()
    if bad > 0:
        raise ValueError(f"{name} contains non-finite values")
    return lo, hi


def shield_nodes(wall_dev, term_dev, n_nodes: int):
    """Wall nodes that belong to no terminal (sorted, on the device)."""
    import torch
    if wall_dev.numel() == 0:
        return wall_dev
    mark = torch.zeros(n_nodes, dtype=torch.bool, device=wall_dev.device)
    for t in term_dev:
        mark[t] = True
    return wall_dev[~mark[wall_dev]]


def as_node_vector(a, grid, name: str) -> np.ndarray:
    """``poisson.py:745-756``: scalar, node-shaped or flat node vector."""
    n = int(np.prod(grid.shape_nodes))
    arr = np.asarray(a, dtype=float)
    if arr.shape == ():
        return np.full(n, float(arr))
    if arr.shape == tuple(grid.shape_nodes):
        return arr.ravel()
    if arr.shape == (n,):
        return arr
    raise ValueError(f"{name} must have shape {tuple(grid.shape_nodes)} or ({n},), "
                     f"got {arr.shape}")


def check_terminals(terminals, grid) -> tuple:
    """Disjoint, non-empty, in-range electrodes (``poisson.py:759-787``)."""
    if terminals is None:
        return ()
    if hasattr(terminals, "nodes") and hasattr(terminals, "name"):
        raise ValueError("pass a sequence of Terminal, not a bare Terminal")
    out = tuple(terminals)
    n_nodes = int(np.prod(grid.shape_nodes))
    names: set[str] = set()
    owner = {}
    for t in out:
        if not (hasattr(t, "nodes") and hasattr(t, "name")):
            raise ValueError(f"expected Terminal instances, got {type(t).__name__}")
        if t.name in names:
            raise ValueError(f"duplicate terminal name {t.name!r}")
        names.add(t.name)
        nodes = np.asarray(t.nodes)
        if nodes.size == 0:
            raise ValueError(f"terminal {t.name!r} has no nodes")
        if nodes.min() < 0 or nodes.max() >= n_nodes:
            raise ValueError(f"terminal {t.name!r} references node index outside "
                             f"[0, {n_nodes})")
        owner[t.name] = nodes
    if len(out) > 1:
        allnodes = np.concatenate([np.asarray(t.nodes, np.int64) for t in out])
        tag = np.concatenate([np.full(np.asarray(t.nodes).size, i)
                              for i, t in enumerate(out)])
        order = np.argsort(allnodes, kind="stable")
        s = allnodes[order]
        dup = np.flatnonzero(s[1:] == s[:-1])
        if dup.size:
            a, b = tag[order[dup[0]]], tag[order[dup[0] + 1]]
            raise ValueError(
                f"terminals {out[a].name!r} and {out[b].name!r} share node "
                f"{int(s[dup[0]])}; electrodes must be disjoint")
    return out


def prepare_bc(bc, grid, allow_periodic: bool = False):
    """Default all-Neumann; reject walls the GPU path does not implement."""
    bc = BoundarySpec.all_neumann() if bc is None else bc
    if not hasattr(bc, "get") and not hasattr(bc, "xlo"):
        raise ValueError(f"bc must be a BoundarySpec, got {type(bc).__name__}")
    if hasattr(bc, "validate"):
        bc.validate(grid)
    check_supported(bc, allow_periodic=allow_periodic)
    return bc


def wrap_map(shape, mask: int) -> np.ndarray:
    """Full node -> node of the wrap-around grid whose periodic axes (``mask``)
    lose their last plane to the first (``poisson.py:942-955`` pairs)."""
    nx, ny, nz = (int(v) for v in shape)
    rx, ry, rz = nx - (mask & 1), ny - ((mask >> 1) & 1), nz - ((mask >> 2) & 1)
    i = np.arange(nx)
    j = np.arange(ny)
    k = np.arange(nz)
    if mask & 1:
        i[-1] = 0
    if mask & 2:
        j[-1] = 0
    if mask & 4:
        k[-1] = 0
    return ((i[:, None, None] * ry + j[None, :, None]) * rz + k[None, None, :]).ravel()


def raise_on_status(stats: list[dict], tol: float, method: str) -> None:
    """Map per-RHS results to the reference's errors (poisson.py:576-587)."""
    hard = max(1e-6, 100.0 * tol)
    for s in stats:
        if s["status"] == L.FS_NAN:
            raise ConvergenceError(f"{method} broke down: residual became NaN/Inf "
                                   f"after {s['iterations']} iterations",
                                   history=[s["relres"]])
        res = s["relres"]
        if res > hard:
            raise ConvergenceError(
                f"{method} failed: relative residual {res:.3e} after "
                f"{s['iterations']} iterations (requested {tol:.1e})",
                history=[res])
        if res > max(tol * 10.0, 1e-12):
            warnings.warn(f"{method} stopped at relative residual {res:.3e}, "
                          f"looser than the requested {tol:.1e}",
                          RuntimeWarning, stacklevel=3)


class PoissonSolver:
    r"""Electrostatic potential from ``G^T M_eps G phi = q`` on the GPU.

    Same parameters as the reference (``poisson.py:864-867``) plus ``gpu``, a
    :class:`GPUConfig` for precision and preconditioner.  ``eps_cell`` is the
    ABSOLUTE permittivity per cell [F/m]; a relative one raises.
    """

    name = "poisson"
    assumptions: tuple[str, ...] = ("A1a", "A2", "A3", "A10", "A12")

    def __init__(self, grid, eps_cell, config: SolverConfig | None = None,
                 operators=None, *, eps_mode: str = "parallel",
                 gpu: GPUConfig | None = None, check_later: bool = False) -> None:
        self.grid = grid
        self.cfg = config or SolverConfig()
        self.gpu = gpu or GPUConfig()
        # check_later (the one-call extraction): the upload and the device
        # check of eps run while the host checks the terminals; the value
        # errors below are raised by the first method that needs eps
        eps_cell, eps_dev, self._eps_pending = upload_cell_property(
            eps_cell, grid, "eps_cell", wait=False)
        self.eps_cell = eps_cell
        self.eps_mode = eps_mode
        if not check_later:
            self._check_eps()
        mark("eps_upload_and_check")
        self.op = DeviceOperator(grid, eps_dev, mode=eps_mode)
        mark("masses")
        if self._eps_range is not None:
            self._set_contrast()

    _eps_range = None

    def _check_eps(self) -> None:
        """Wait for the eps check (once) and raise on a bad permittivity."""
        if self._eps_range is not None:
            return
        eps_min, eps_max = cell_property_range(self._eps_pending, "eps_cell")
        if eps_min <= 0.0:
            raise ValueError("eps_cell must be strictly positive [F/m]")
        if eps_min >= 1e-6:
            raise ValueError(
                f"eps_cell looks like a RELATIVE permittivity (min "
                f"{eps_min:.4g}); fieldspice is strict SI and wants the "
                "absolute value in F/m. Multiply by eps0.")
        self._eps_range = (eps_min, eps_max)
        self._eps_pending = None
        if getattr(self, "op", None) is not None:
            self._set_contrast()

    def _set_contrast(self) -> None:
        lo, hi = self._eps_range
        self.op.material_contrast = hi / lo if lo > 0.0 else None
        self._L = None
        self.last_capacitance_report: dict[str, Any] = {}
        self.last_device_time = 0.0

    # -- compatibility accessors --------------------------------------------
    @property
    def L(self):
        """Nodal capacitance matrix ``G^T M_eps G`` as SciPy CSR (host, lazy).

        Assembled from the device masses for callers that want the matrix;
        the solve itself never forms it.
        """
        self._check_eps()
        if self._L is None:
            self._L = assemble_csr(self.grid, self.op.edge_vector())
        return self._L

    @property
    def eps_edge(self) -> np.ndarray:
        """Permittivity averaged onto edges [F/m] in [x|y|z] edge order
        (``poisson.py:894-897``), recovered from the device masses as
        ``m_e * L_e / A_e``."""
        self._check_eps()
        return self.op.edge_vector() / edge_area_over_length(self.grid)

    @property
    def node_volumes(self) -> np.ndarray:
        return np.asarray(self.grid.node_volumes(), float).ravel()

    def _phi_dev(self, phi):
        import torch
        self._check_eps()
        p = as_node_vector(phi, self.grid, "phi")
        return torch.as_tensor(p, dtype=torch.float64, device=self.op.dev)

    def energy(self, phi) -> float:
        """``0.5 phi^T L phi`` [J] (poisson.py:905-913), FP64 on the GPU."""
        return 0.5 * float(self.op.quadform(self._phi_dev(phi))[0])

    def node_charge(self, phi) -> np.ndarray:
        """``L phi`` [C] per node (poisson.py:915-922)."""
        return self.op.apply(self._phi_dev(phi)).cpu().numpy()

    # -- capacitance extraction ------------------------------------------------
    def capacitance_matrix(self, terminals: Sequence, bc=None, *,
                           report: dict[str, Any] | None = None,
                           symmetrise: bool = True) -> np.ndarray:
        """Maxwell capacitance matrix [F] by unit excitation.

        Same algorithm and report as ``poisson.py:1100-1249``: terminal ``j``
        at 1 V, every other terminal and every Dirichlet wall at 0 V, and
        ``C[i, j] = sum_{n in T_i} (L phi_j)_n``.  All excitations share one
        eliminated system and are solved as blocks of right-hand sides (up to
        8 per device solve in mixed precision, 4 in FP64: 32-byte nodes).
        """
        import torch
        t_start = time.perf_counter()
        grid = self.grid
        try:
            # host-side checks while the eps upload and check may still run;
            # a bad eps is reported first, as the constructor would
            terms = check_terminals(terminals, grid)
            if not terms:
                raise ValueError("capacitance extraction needs at least one terminal")
            bc = prepare_bc(bc, grid, allow_periodic=True)
            mask = periodic_mask(bc)
            dev = self.op.dev
            wall_idx, _ = dirichlet_nodes(bc, grid, 0.0)
            mark("terminal_checks")
            term_nodes = [np.asarray(t.nodes, np.int64) for t in terms]
            term_dev = [h2d(n, torch.int64, dev) for n in term_nodes]
            wall_dev = h2d(wall_idx.astype(np.int64), torch.int64, dev)
            shield_dev = shield_nodes(wall_dev, term_dev, self.op.N)
        except Exception:
            self._check_eps()
            raise
        self._check_eps()
        mark("node_upload")
        op, charges = self.op, None
        if mask:
            # periodic walls: solve on the wrap-around grid (the reference's
            # P^T L P node merge), integrate the charges on the full grid
            wmap = wrap_map(self.op.shape, mask)
            op = self.op.reduced(mask)
            groups = term_dev + ([shield_dev] if shield_dev.numel() else [])
            charges = (self.op, h2d(wmap, torch.int64, dev), groups)
            term_dev = [h2d(np.unique(wmap[n]), torch.int64, dev) for n in term_nodes]
            wall_dev = h2d(np.unique(wmap[wall_idx]).astype(np.int64), torch.int64, dev)
            shield_dev = shield_nodes(wall_dev, term_dev, op.N)
        C, q_shield, info = extract_capacitance(
            op, term_dev, wall_dev, shield_dev, tol=float(self.cfg.tol),
            precision=self.gpu.precision, maxiter=self.gpu.maxiter,
            preconditioner=resolve_preconditioner(self.cfg, self.gpu),
            learned=None if mask else self.gpu.learned, charges=charges,
            coarsening=self.gpu.coarsening,
            mg_params=self.gpu.mg_params)
        info["solve_time"] = time.perf_counter() - t_start
        rep = capacitance_report(C, q_shield, info, symmetrise)
        mark("report")
        rep["terminals"] = tuple(t.name for t in terms)
        if symmetrise:
            C = 0.5 * (C + C.T)
        scale = float(np.abs(np.diag(C)).max()) or 1.0
        if rep["max_offdiag"] > 1e-9 * scale:
            warnings.warn(
                f"Maxwell capacitance matrix has a positive off-diagonal entry "
                f"({rep['max_offdiag']:.4g} F): the solve is not converged, or "
                "two electrodes are not electrically distinct.",
                RuntimeWarning, stacklevel=2)
        self.last_capacitance_report = rep
        if report is not None:
            report.update(rep)
        return C

    def spice_capacitance_matrix(self, terminals: Sequence, bc=None, *,
                                 report: dict[str, Any] | None = None) -> np.ndarray:
        """Mutual (SPICE) matrix from the Maxwell one (poisson.py:1251-1281)."""
        Cm = self.capacitance_matrix(terminals, bc, report=report)
        Cs = -Cm.copy()
        np.fill_diagonal(Cs, Cm.sum(axis=1))
        return Cs

    # -- single potential solve -------------------------------------------------
    def solve(self, terminals: Sequence | None = None, bc=None, rho_node=None,
              *, t: float = 0.0) -> Result:
        """Potential for voltage-driven, floating and charge-driven terminals,
        Dirichlet walls and free charge (``poisson.py:967-1063``).

        The reference merges every floating or charge-driven electrode into one
        unknown (``P^T L P``, ``poisson.py:665-719``).  Here the same solution
        comes from superposition, with the electrodes held as Dirichlet
        conductors: one block solve gives the potential with every such
        electrode at 0 V and the unit potential of each, and the small system
        ``C V = Q - q_0`` (``C`` their mutual capacitances, ``Q`` the
        prescribed charges, 0 for a floating one) fixes their potentials.
        Periodic walls (also a node merge) are not implemented.
        """
        import torch
        self._check_eps()
        t0 = time.perf_counter()
        grid = self.grid
        terms = check_terminals(terminals, grid)
        bc = prepare_bc(bc, grid, allow_periodic=True)
        mask = periodic_mask(bc)
        dev = self.op.dev
        N = self.op.N
        vnode = self.node_volumes
        b_free = np.zeros(N)
        if rho_node is not None:
            b_free += as_node_vector(rho_node, grid, "rho_node") * vnode
        # driven Neumann walls: their flux load joins the free charge
        # (poisson.py:957-964)
        load = neumann_load(bc, grid, t)
        with_load = load is not None
        if with_load:
            b_free += load

        fixed, vals = _dirichlet_sets(bc, terms, grid, t)
        floats = [tt for tt in terms if tt.driven != "voltage"]
        if mask:
            if floats:
                raise NotImplementedError(
                    "floating or charge-driven electrodes together with periodic walls "
                    "are not supported on the GPU path")
            return self._solve_periodic(terms, mask, fixed, vals, b_free,
                                        rho_node is not None or with_load, t0)
        if floats:
            return self._solve_floating(terms, floats, fixed, vals, b_free,
                                        rho_node is not None or with_load, t, t0)
        label = torch.zeros(N, dtype=torch.uint8, device=dev)
        pinned = None
        if fixed.size == 0:
            # All-Neumann: pin the node with the largest diagonal to 0 V, as
            # LinearSystem does (poisson.py:297-322).
            diag = self._diagonal()
            pinned = int(np.argmax(np.abs(diag)))
            fixed = np.array([pinned], dtype=np.intp)
            vals = np.zeros(1)
            warnings.warn(
                "singular all-Neumann system: no Dirichlet node was found, so "
                f"node {pinned} is pinned to 0 to fix the gauge.  Only "
                "potential DIFFERENCES in the result are meaningful; the "
                "absolute level is arbitrary.", RuntimeWarning, stacklevel=2)
        fixed_d = torch.as_tensor(fixed, device=dev)
        label[fixed_d] = L.LABEL_FIXED
        with_src = rho_node is not None or with_load
        system = EliminatedSystem(self.op, label, 1, precision=self.gpu.precision,
                                  with_source=with_src,
                                  preconditioner=resolve_preconditioner(self.cfg, self.gpu),
                                  coarsening=self.gpu.coarsening,
                                  mg_params=self.gpu.mg_params)
        system.phi.zero_()
        system.phi[fixed_d] = torch.as_tensor(vals, dtype=torch.float64, device=dev)
        if with_src:
            system.f.copy_(torch.as_tensor(b_free, dtype=torch.float64, device=dev))
        tol = float(self.cfg.tol)
        _, stats = system.solve(tol, self.gpu.maxiter)
        raise_on_status(stats, tol, "gpu-cg")
        info = {"method": f"gpu-cg-{system.preconditioner}-{self.gpu.precision}", "n": N,
                "n_factorised": system.n_free, "iterations": stats[0]["iterations"],
                "residual": stats[0]["relres"], "pinned": pinned,
                "setup_time": system.setup_time,
                "solve_time": time.perf_counter() - t0}
        res = self._potential_result(system.phi, terms, b_free, info, fixed.size, t0)
        system.close()
        return res

    def _solve_periodic(self, terms, mask: int, fixed, vals, b_free, with_src: bool,
                        t0: float) -> Result:
        """Periodic walls: the solve on the wrap-around grid (the reference's
        node merge P^T L P x = P^T b, ``poisson.py:1041-1058``), expanded back
        to the full grid, where the charges and energy are evaluated."""
        import torch
        dev = self.op.dev
        wmap = wrap_map(self.op.shape, mask)
        op = self.op.reduced(mask)
        Nr = op.N
        b_r = np.bincount(wmap, weights=b_free, minlength=Nr)
        # merged Dirichlet nodes: the value of the last one in index order wins,
        # as numpy's assignment in apply_dirichlet does
        fr = wmap[fixed]
        uniq, last = np.unique(fr[::-1], return_index=True)
        fixed_r, vals_r = uniq, np.asarray(vals)[::-1][last]
        pinned = None
        if fixed_r.size == 0:
            d = self._diagonal(op)
            pinned = int(np.argmax(np.abs(d)))
            fixed_r, vals_r = np.array([pinned]), np.zeros(1)
            warnings.warn(
                "singular all-Neumann system: no Dirichlet node was found, so "
                f"node {pinned} is pinned to 0 to fix the gauge.  Only "
                "potential DIFFERENCES in the result are meaningful; the "
                "absolute level is arbitrary.", RuntimeWarning, stacklevel=3)
        label = torch.zeros(Nr, dtype=torch.uint8, device=dev)
        fixed_d = h2d(fixed_r.astype(np.int64), torch.int64, dev)
        label[fixed_d] = L.LABEL_FIXED
        system = EliminatedSystem(op, label, 1, precision=self.gpu.precision,
                                  with_source=with_src, preconditioner="jacobi")
        system.phi.zero_()
        system.phi[fixed_d] = h2d(vals_r, torch.float64, dev)
        if with_src:
            system.f.copy_(h2d(b_r, torch.float64, dev))
        tol = float(self.cfg.tol)
        _, stats = system.solve(tol, self.gpu.maxiter)
        raise_on_status(stats, tol, "gpu-cg")
        phi_full = system.phi.index_select(0, h2d(wmap, torch.int64, dev))
        info = {"method": f"gpu-cg-jacobi-{self.gpu.precision}", "n": Nr,
                "n_factorised": system.n_free, "iterations": stats[0]["iterations"],
                "residual": stats[0]["relres"], "pinned": pinned, "periodic": mask,
                "setup_time": system.setup_time, "solve_time": time.perf_counter() - t0}
        res = self._potential_result(phi_full, terms, b_free, info, fixed_r.size, t0)
        res.meta["n_unknowns"] = Nr
        system.close()
        return res

    def _solve_floating(self, terms, floats, fixed, vals, b_free, with_src: bool,
                        t: float, t0: float) -> Result:
        """Floating / charge-driven electrodes by superposition (see solve)."""
        import torch
        N = self.op.N
        dev = self.op.dev
        nf = len(floats)
        if fixed.size == 0:
            raise NotImplementedError(
                "floating electrodes without any Dirichlet node (a driven terminal or "
                "a grounded wall): the potential has no reference on the GPU path")
        fnodes = [np.asarray(tt.nodes, np.intp) for tt in floats]
        if np.isin(np.concatenate(fnodes), fixed).any():
            raise NotImplementedError(
                "a floating or charge-driven electrode touches a Dirichlet node")
        # columns: 0 = the driven potentials (every floating electrode at 0 V)
        # with the free charge, 1 + f = electrode f at 1 V and everything else
        # at 0 V; solved in blocks of 32-byte nodes on one system
        ncol = nf + 1
        chunks = rhs_blocks(ncol, block_rhs(self.gpu.precision))
        k = pad_rhs(len(chunks[0]))
        label = torch.zeros(N, dtype=torch.uint8, device=dev)
        fixed_d = torch.as_tensor(fixed, device=dev)
        label[fixed_d] = L.LABEL_FIXED
        fnodes_d = [h2d(nd.astype(np.int64), torch.int64, dev) for nd in fnodes]
        for nd in fnodes_d:
            label[nd] = L.LABEL_FIXED
        system = EliminatedSystem(self.op, label, len(chunks[0]), precision=self.gpu.precision,
                                  with_source=with_src,
                                  preconditioner=resolve_preconditioner(self.cfg, self.gpu),
                                  coarsening=self.gpu.coarsening,
                                  mg_params=self.gpu.mg_params)
        tol = float(self.cfg.tol)
        Q = np.zeros((nf, ncol))
        sols, stats_all = [], []
        for cols in chunks:
            system.nrhs = len(cols)
            phi_h = np.zeros((N, k))
            for c, j in enumerate(cols):
                if j == 0:
                    phi_h[fixed, c] = vals
                else:
                    phi_h[fnodes[j - 1], c] = 1.0
            system.phi.copy_(h2d(phi_h.ravel(), torch.float64, dev))
            if with_src:
                f_h = np.zeros((N, k))
                if cols[0] == 0:
                    f_h[:, 0] = b_free
                system.f.copy_(h2d(f_h.ravel(), torch.float64, dev))
            _, stats = system.solve(tol, self.gpu.maxiter)
            raise_on_status(stats, tol, "gpu-cg")
            stats_all.extend(stats)
            Q[:, cols] = self.op.group_sums(system.phi, fnodes_d, nrhs=k)[:, :len(cols)]
            sols.append((cols, system.phi.clone() if len(chunks) > 1 else system.phi))
        q0 = Q[:, 0] - np.array([b_free[nd].sum() for nd in fnodes])
        Cff = Q[:, 1:]
        target = np.array([float(tt.value_at(t)) if tt.driven == "current" else 0.0
                           for tt in floats])
        V = np.linalg.solve(Cff, target - q0)
        weight = np.concatenate([[1.0], V])
        phi_d = torch.empty(N, dtype=torch.float64, device=dev)
        for i, (cols, sol) in enumerate(sols):
            coef = (ctypes.c_double * len(cols))(*weight[cols])
            L.check("fs_rhs_superpose", L.lib().fs_rhs_superpose(
                L.ptr(sol), k, 0, len(cols), coef, None if i == 0 else L.ptr(phi_d),
                L.ptr(phi_d), N, L.stream_ptr()))
        info = {"method": f"gpu-cg-{system.preconditioner}-{self.gpu.precision}", "n": N,
                "n_factorised": system.n_free,
                "iterations": max(s["iterations"] for s in stats_all),
                "residual": max(s["relres"] for s in stats_all), "pinned": None,
                "floating_potentials": V.tolist(), "blocks": len(chunks),
                "setup_time": system.setup_time,
                "solve_time": time.perf_counter() - t0}
        res = self._potential_result(phi_d, terms, b_free, info, fixed.size, t0)
        system.close()
        return res

    def _potential_result(self, phi_d, terms, b_free, info, n_fixed: int, t0: float) -> Result:
        """``Result`` of a potential solve (poisson.py:1082-1097)."""
        grid = self.grid
        N = self.op.N
        phi = phi_d.cpu().numpy().copy()
        qnode = self.op.apply(phi_d).cpu().numpy() - b_free
        res = Result(grid=grid)
        res.fields["phi"] = phi.reshape((1,) + tuple(grid.shape_nodes))
        res.fields["e"] = (-grad_edges(grid, phi)).reshape(1, -1)
        for tt in terms:
            res.terminals[tt.name] = {
                "v": np.array([float(phi[tt.nodes[0]])]),
                "q": np.array([float(qnode[tt.nodes].sum())]),
            }
        res.scalars["energy"] = np.array([0.5 * float(self.op.quadform(phi_d)[0])])
        res.scalars["total_charge"] = np.array([float(qnode.sum())])
        res.meta["linear"] = info
        res.meta["n_unknowns"] = N
        res.meta["n_dirichlet"] = int(n_fixed)
        res.meta.setdefault("solver", self.name)
        res.meta.setdefault("assumptions", list(self.assumptions))
        res.meta.setdefault("wall_time", time.perf_counter() - t0)
        res.meta.setdefault("grid_cells", tuple(grid.shape_cells))
        return res

    def _diagonal(self, op=None) -> np.ndarray:
        """Sum of the incident masses per node (with the wrap edges of a
        periodic operator)."""
        op = self.op if op is None else op
        nx, ny, nz = op.shape
        m = op.m.cpu().numpy().reshape(3, nx, ny, nz)
        d = m[0] + m[1] + m[2]
        d[1:] += m[0, :-1]
        d[:, 1:] += m[1, :, :-1]
        d[:, :, 1:] += m[2, :, :, :-1]
        if op.periodic & 1:
            d[0] += m[0, -1]
        if op.periodic & 2:
            d[:, 0] += m[1, :, -1]
        if op.periodic & 4:
            d[:, :, 0] += m[2, :, :, -1]
        return d.ravel()


def extract_capacitance(op: DeviceOperator, term_dev, wall_dev, shield_dev, *,
                        tol: float, precision: str = "auto",
                        maxiter: int | None = None, preconditioner: str = "jacobi",
                        learned=None, charges=None, coarsening: str = "auto",
                        mg_params: dict | None = None):
    """Device core of the extraction: inputs already in HBM.

    ``term_dev``: sorted unique int64 node tensors, one per terminal;
    ``wall_dev``: Dirichlet wall nodes (grounded); ``shield_dev``: wall nodes
    that belong to no terminal.  Returns ``(C, q_shield, info)`` with ``C``
    not yet symmetrised (``poisson.py:1196-1224``).

    ``charges``: for a wrap-around (periodic) ``op``, ``(full_op, node_map,
    groups)``: each solution is expanded to the full grid through
    ``node_map`` (full node -> reduced node) and the charges integrated there
    on the full-grid node sets ``groups`` (terminals, then the shield), as the
    reference does (``poisson.py:1218-1223``).
    """
    import torch
    dev = op.dev
    N = op.N
    nt = len(term_dev)
    label = torch.zeros(N, dtype=torch.uint8, device=dev)
    if wall_dev.numel():
        label[wall_dev] = L.LABEL_FIXED
    for n in term_dev:
        label[n] = L.LABEL_FIXED
    group = torch.empty(N, dtype=torch.int16, device=dev)
    has_shield = shield_dev.numel() > 0
    groups = list(term_dev) + ([shield_dev] if has_shield else [])
    gdev = upload_groups(groups, dev)
    C = np.zeros((nt, nt))
    q_shield = np.zeros(nt)
    stats_all: list[dict] = []
    system = None
    gdev_full = None
    launches = 0
    setup_time = 0.0
    nx, ny, nz = op.shape
    # blocks of at most 32-byte nodes (8 FP32 / 4 FP64 RHS), near-equal in
    # size so that one plan of one padded width solves them all
    blocks = rhs_blocks(nt, block_rhs(precision))
    k = pad_rhs(len(blocks[0]))
    for cols in blocks:
        kb = len(cols)
        if system is None:
            mark("labels")
            system = EliminatedSystem(op, label, len(blocks[0]), precision=precision,
                                      preconditioner=preconditioner, learned=learned,
                                      coarsening=coarsening, mg_params=mg_params)
            setup_time += system.setup_time
            mark("plan")
        system.nrhs = kb
        group.fill_(-1)
        for c, j in enumerate(cols):
            group[term_dev[j]] = c
        st = L.lib().fs_fill_unit_excitation(L.ptr(group), L.ptr(label),
                                             L.ptr(system.phi), nx, ny, nz, k,
                                             L.stream_ptr())
        L.check("fs_fill_unit_excitation", st)
        _, stats = system.solve(tol, maxiter)
        mark("solve")
        launches += system.launches + 1
        raise_on_status(stats, tol, "gpu-cg")
        stats_all.extend(stats)
        if charges is None:
            Q = op.group_sums(system.phi, groups, nrhs=k, nodes_dev=gdev)
        else:
            full_op, node_map, full_groups = charges
            if gdev_full is None:
                gdev_full = upload_groups(full_groups, dev)
            phi_full = system.phi.view(op.N, k).index_select(0, node_map).reshape(-1)
            Q = full_op.group_sums(phi_full, full_groups, nrhs=k, nodes_dev=gdev_full)
        launches += 1
        mark("charge_and_readback")
        for c, j in enumerate(cols):
            C[:, j] = Q[:nt, c]
            if has_shield:
                q_shield[j] = Q[nt, c]
    info = {
        "method": f"gpu-cg-{preconditioner}-{precision}",
        "n": N,
        "n_factorised": system.n_free,
        "n_decoupled": system.n_fixed + system.n_solo,
        "n_solo": system.n_solo,
        "equilibrated": True,
        "symmetric": True,
        "singular": False,
        "pinned": None,
        "n_pinned": system.n_pinned,
        "setup_time": setup_time,
        "iterations": [s["iterations"] for s in stats_all],
        "residual": max(s["relres"] for s in stats_all),
        "relres_fp64": [s["relres"] for s in stats_all],
        "reliable_updates": [s["reliable_updates"] for s in stats_all],
        "fp64_fallback": bool(system.fell_back),
        "coarsening": system.coarsening,
        "learned_fallback": bool(system.learned_fallback),
        "gpu_launches": launches,
        "kernel_ms": system.kernel_times(),
        "notes": (),
    }
    system.close()
    mark("plan_release")
    return C, q_shield, info


def capacitance_report(C: np.ndarray, q_shield: np.ndarray, info: dict,
                       symmetrise: bool = True) -> dict[str, Any]:
    """Quality metrics of ``poisson.py:1225-1239`` for an unsymmetrised C."""
    nt = C.shape[0]
    rep: dict[str, Any] = {}
    scale = float(np.abs(np.diag(C)).max()) or 1.0
    asym = float(np.abs(C - C.T).max())
    rep["asymmetry_abs"] = asym
    rep["asymmetry_rel"] = asym / scale
    Cs = 0.5 * (C + C.T) if symmetrise else C
    rows = Cs.sum(axis=1)
    rep["row_sum"] = rows
    rep["row_sum_rel"] = float(np.abs(rows).max() / scale)
    off = Cs - np.diag(np.diag(Cs))
    rep["max_offdiag"] = float(off.max()) if nt > 1 else 0.0
    rep["shield_charge"] = q_shield
    rep["linear"] = info
    return rep


def _dirichlet_sets(bc, terms, grid, t: float):
    """Fixed nodes and values, a terminal beating a wall (poisson.py:1065-1080)."""
    idx_parts, val_parts = [], []
    w_idx, w_val = dirichlet_nodes(bc, grid, t)
    if w_idx.size:
        idx_parts.append(w_idx)
        val_parts.append(w_val)
    for tt in terms:
        if tt.driven == "voltage":
            idx_parts.append(np.asarray(tt.nodes, np.intp))
            val_parts.append(np.full(np.asarray(tt.nodes).size, float(tt.value_at(t))))
    if not idx_parts:
        return np.empty(0, dtype=np.intp), np.empty(0, dtype=float)
    idx = np.concatenate(idx_parts)
    val = np.concatenate(val_parts)
    uniq, first_in_rev = np.unique(idx[::-1], return_index=True)
    return uniq.astype(np.intp), val[::-1][first_in_rev]


def edge_area_over_length(grid) -> np.ndarray:
    """``A_dual / L`` per edge in [x|y|z] order (grid.py:398-420)."""
    hx, hy, hz = (np.asarray(a, float) for a in (grid.hx, grid.hy, grid.hz))
    hxd, hyd, hzd = (np.asarray(a, float) for a in (grid.hxd, grid.hyd, grid.hzd))
    ax = (hyd[None, :, None] * hzd[None, None, :]) / hx[:, None, None]
    ay = (hxd[:, None, None] * hzd[None, None, :]) / hy[None, :, None]
    az = (hxd[:, None, None] * hyd[None, :, None]) / hz[None, None, :]
    return np.concatenate([ax.ravel(), ay.ravel(), az.ravel()])


def grad_edges(grid, phi: np.ndarray) -> np.ndarray:
    """``G phi`` in the reference's [x|y|z] edge order (operators.py:71-91)."""
    p = np.asarray(phi, float).reshape(tuple(grid.shape_nodes))
    return np.concatenate([np.diff(p, axis=0).ravel(), np.diff(p, axis=1).ravel(),
                           np.diff(p, axis=2).ravel()])


def assemble_csr(grid, mass_edge: np.ndarray):
    """``G^T diag(m) G`` as SciPy CSR from an edge-ordered mass vector."""
    import scipy.sparse as sp
    shape = tuple(int(s) for s in grid.shape_nodes)
    nid = np.arange(int(np.prod(shape))).reshape(shape)
    heads = [nid[1:].ravel(), nid[:, 1:].ravel(), nid[:, :, 1:].ravel()]
    tails = [nid[:-1].ravel(), nid[:, :-1].ravel(), nid[:, :, :-1].ravel()]
    h = np.concatenate(heads)
    tl = np.concatenate(tails)
    E = h.size
    G = sp.csr_matrix((np.concatenate([np.ones(E), -np.ones(E)]),
                       (np.concatenate([np.arange(E), np.arange(E)]),
                        np.concatenate([h, tl]))), shape=(E, nid.size))
    return sp.csr_matrix(G.T @ sp.diags(mass_edge) @ G)
