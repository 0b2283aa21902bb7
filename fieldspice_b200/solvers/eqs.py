"""Electroquasistatic transient on the GPU: ``G^T (M_sigma + M_eps d/dt) G phi = i``.

Drop-in for ``fieldspice/solvers/eqs.py``'s ``EQSSolver`` (``:42-386``):
same constructor, ``solve`` (theta scheme, backward Euler by default),
``consistent_initial_condition``, ``steady_state``, ``terminal_current``,
``stored_energy``, ``dissipation`` and ``capacitance_matrix``.

Per time step (``eqs.py:291-307``) the device computes the explicit part
``f = Kexp phi_prev (+ injected current)`` with ``Kexp = L_eps/dt -
(1-theta) L_sigma``, writes the step's Dirichlet values, and solves
``K phi = f`` with ``K = L_eps/dt + theta L_sigma`` by the same CG plan as the
electrostatic path.  The plan (the reference's cached ``LinearSystem``) is
built once per run because the fixed-node set does not change.  Unlike the
reference, each step's CG starts from the previous step's potential (a warm
start converging to the same fixed point under the same stopping rule,
relative to ``||b||``).  Terminal currents are evaluated on the device from
the unconstrained operators, ``I_T = sum_{n in T} (K phi_new - Kexp
phi_old)_n`` (identical to ``eqs.py:328-340``).
"""

from __future__ import annotations

import time
import warnings
from typing import Any, Sequence

import numpy as np

from .. import _lib as L
from ..boundaries import BoundarySpec, check_supported, dirichlet_nodes
from ..device import DeviceOperator, EliminatedSystem, d2h, h2d, upload_groups
from .base import GPUConfig, Result, SolverConfig, resolve_preconditioner
from .poisson import check_terminals, raise_on_status

__all__ = ["EQSSolver"]


def _contrast(prop: np.ndarray):
    """Largest over smallest positive cell value (None when none is)."""
    pos = prop[prop > 0]
    return float(pos.max() / pos.min()) if pos.size else None


def _walls_time_dependent(bc) -> bool:
    """Whether a Dirichlet wall of ``bc`` takes a callable value."""
    from ..boundaries import WALLS
    for w in WALLS:
        wall = bc.get(w) if hasattr(bc, "get") else getattr(bc, w, None)
        if getattr(wall, "is_dirichlet_like", False) and callable(getattr(wall, "value", None)):
            return True
    return False


class EQSSolver:
    """Time-domain electroquasistatic solver (``eqs.py:42-103``).

    ``eps_cell`` absolute permittivity [F/m], ``sigma_cell`` conductivity
    [S/m], both ``grid.shape_cells``; ``gpu`` selects precision.
    """

    name = "eqs"
    assumptions = ("A1a", "A2", "A3", "A10", "A12")

    def __init__(self, grid, eps_cell, sigma_cell, config: SolverConfig | None = None,
                 operators=None, *, eps_mode: str = "parallel",
                 sigma_mode: str = "parallel", gpu: GPUConfig | None = None):
        self.grid = grid
        self.cfg = config or SolverConfig()
        self.gpu = gpu or GPUConfig()
        eps_cell = np.asarray(eps_cell, dtype=float)
        sigma_cell = np.asarray(sigma_cell, dtype=float)
        for arr, nm in ((eps_cell, "eps_cell"), (sigma_cell, "sigma_cell")):
            if arr.shape != tuple(grid.shape_cells):
                raise ValueError(f"{nm} must have shape {tuple(grid.shape_cells)}, "
                                 f"got {arr.shape}")
            if not np.all(np.isfinite(arr)):
                raise ValueError(f"{nm} contains non-finite values")
        if np.any(eps_cell <= 0.0):
            raise ValueError("eps_cell must be positive and ABSOLUTE [F/m]; multiply a "
                             "relative permittivity by eps0")
        if float(np.min(eps_cell)) > 1e-6:
            raise ValueError(f"eps_cell looks like a RELATIVE permittivity (min "
                             f"{float(np.min(eps_cell)):.4g}); it must be absolute [F/m].")
        if np.any(sigma_cell < 0.0):
            raise ValueError("sigma_cell must be non-negative [S/m]")
        self.eps_cell, self.sigma_cell = eps_cell, sigma_cell
        self.ops = operators  # handed to monitors as state["ops"], as the reference does
        self.op_eps = DeviceOperator(grid, eps_cell, mode=eps_mode)
        self.op_sig = DeviceOperator(grid, sigma_cell, mode=sigma_mode)
        self._vnode = np.asarray(grid.node_volumes(), float).ravel()

    # -- bookkeeping ----------------------------------------------------------
    def _dirichlet(self, terminals, bc, t: float):
        """Fixed nodes and values at t; later entries win (eqs.py:108-129):
        terminals first, then the walls."""
        idx, val = [], []
        for term in terminals:
            if term.driven == "voltage":
                idx.append(np.asarray(term.nodes, np.intp))
                val.append(np.full(np.asarray(term.nodes).size, float(term.value_at(t))))
        if bc is not None:
            bidx, bval = dirichlet_nodes(bc, self.grid, t)
            if bidx.size:
                idx.append(bidx)
                val.append(bval)
        if not idx:
            return np.zeros(0, np.intp), np.zeros(0)
        fixed = np.concatenate(idx)
        values = np.concatenate(val)
        uniq, last = np.unique(fixed[::-1], return_index=True)
        return uniq, values[::-1][last]

    def _dirichlet_values(self, terminals, bc, fixed, dev):
        """Per-step Dirichlet values of the fixed set ``fixed`` (fixed for the
        run; the later source wins on a shared node, eqs.py:108-129) as a
        function of t returning a device tensor.  When every source is
        uniform (a terminal's voltage, a wall of one value) only the source
        values cross to the device each step and a gather spreads them."""
        import torch
        srcs = [("term", tt) for tt in terminals if tt.driven == "voltage"]
        idx = [np.asarray(tt.nodes, np.intp) for _, tt in srcs]
        bidx, bval0 = (dirichlet_nodes(bc, self.grid, 0.0) if bc is not None
                       else (np.zeros(0, np.intp), np.zeros(0)))
        if bidx.size:
            idx.append(bidx)
        if not idx:
            return lambda t: torch.zeros(0, dtype=torch.float64, device=dev)
        cat = np.concatenate(idx)
        owner = np.concatenate([np.full(a.size, j) for j, a in enumerate(idx)])
        uniq, last = np.unique(cat[::-1], return_index=True)
        pick = cat.size - 1 - last
        assert np.array_equal(uniq, fixed)
        walls_uniform = bidx.size == 0 or bool(np.all(np.asarray(bval0) == bval0[0]))
        if walls_uniform and not (bc is not None and _walls_time_dependent(bc)):
            owner_d = h2d(owner[pick].astype(np.int64), torch.int64, dev)
            wall_v = float(bval0[0]) if bidx.size else 0.0

            def values(t):
                v = [float(tt.value_at(t)) for _, tt in srcs]
                if bidx.size:
                    v.append(wall_v)
                return h2d(np.asarray(v), torch.float64, dev)[owner_d]
            return values

        def values_general(t):
            parts = [np.full(a.size, float(tt.value_at(t))) for a, (_, tt) in zip(idx, srcs)]
            if bidx.size:
                parts.append(np.asarray(dirichlet_nodes(bc, self.grid, t)[1], float))
            return h2d(np.concatenate(parts)[pick], torch.float64, dev)
        return values_general

    def _node_weights(self, nodes) -> np.ndarray:
        """Dual-volume weights of a terminal's nodes (eqs.py:131-154)."""
        w = self._vnode[np.asarray(nodes, np.intp)]
        total = float(w.sum())
        return w / total if total > 0 else np.full(w.size, 1.0 / w.size)

    def _inject_dev(self, terminals, t: float, dev):
        """Injected node currents of current-driven terminals (eqs.py:156-163)."""
        import torch
        rhs = None
        for term in terminals:
            if term.driven == "current":
                if rhs is None:
                    rhs = torch.zeros(self.op_eps.N, dtype=torch.float64, device=dev)
                i_tot = float(term.value_at(t))
                w = h2d(i_tot * self._node_weights(term.nodes), torch.float64, dev)
                rhs[h2d(np.asarray(term.nodes, np.int64), torch.int64, dev)] += w
        return rhs

    def _prepare(self, terminals, bc):
        terms = check_terminals(terminals, self.grid)
        if bc is not None:
            check_supported(bc)
        return terms, bc

    def _solve_static(self, op: DeviceOperator, terms, bc, t, rhs_dev=None):
        """One Dirichlet solve with operator ``op``; returns the device phi."""
        import torch
        dev = op.dev
        fixed, vals = self._dirichlet(terms, bc, t)
        label = torch.zeros(op.N, dtype=torch.uint8, device=dev)
        if fixed.size:
            label[h2d(fixed.astype(np.int64), torch.int64, dev)] = L.LABEL_FIXED
        system = EliminatedSystem(op, label, 1, precision=self.gpu.precision,
                                  with_source=rhs_dev is not None,
                                  preconditioner=resolve_preconditioner(self.cfg, self.gpu),
                                  coarsening=self.gpu.coarsening,
                                  mg_params=self.gpu.mg_params)
        if fixed.size:
            system.phi[h2d(fixed.astype(np.int64), torch.int64, dev)] = \
                h2d(vals, torch.float64, dev)
        if rhs_dev is not None:
            system.f.copy_(rhs_dev)
        _, stats = system.solve(float(self.cfg.tol), self.gpu.maxiter)
        raise_on_status(stats, float(self.cfg.tol), "gpu-cg")
        phi = system.phi.clone()
        info = {"iterations": stats[0]["iterations"], "residual": stats[0]["relres"],
                "n_free": system.n_free, "n_pinned": system.n_pinned}
        system.close()
        return phi, info

    # -- initial condition ------------------------------------------------------
    def consistent_initial_condition(self, terminals: Sequence, bc=None,
                                     t: float = 0.0) -> np.ndarray:
        """Electrostatic potential at t: the capacitive divider (eqs.py:176-195)."""
        terms, bc = self._prepare(terminals, bc)
        fixed, _ = self._dirichlet(terms, bc, t)
        if fixed.size == 0:
            return np.zeros(self.op_eps.N)
        phi, _ = self._solve_static(self.op_eps, terms, bc, t)
        return d2h(phi)

    # -- steady state -------------------------------------------------------------
    def steady_state(self, terminals: Sequence, bc=None, t: float = 0.0) -> Result:
        """DC solve with ``L_sigma`` only (eqs.py:200-224)."""
        t0 = time.perf_counter()
        terms, bc = self._prepare(terminals, bc)
        dev = self.op_sig.dev
        rhs = self._inject_dev(terms, t, dev)
        phi_d, info = self._solve_static(self.op_sig, terms, bc, t, rhs)
        phi = d2h(phi_d)
        res = Result(grid=self.grid, t=np.zeros(1), fields={"phi": phi[None, :]})
        groups = [np.asarray(tt.nodes, np.int64) for tt in terms]
        if groups:
            cur = self.op_sig.group_sums(phi_d, groups)[:, 0]
            for j, tt in enumerate(terms):
                w = self._node_weights(tt.nodes)
                res.terminals[tt.name] = {"v": np.array([float(w @ phi[tt.nodes])]),
                                          "i": np.array([float(cur[j])])}
        res.scalars["dissipation"] = np.array([float(self.op_sig.quadform(phi_d)[0])])
        res.meta.update(solver=self.name, assumptions=list(self.assumptions),
                        wall_time=time.perf_counter() - t0, mode="steady_state",
                        linear=info, grid_cells=tuple(self.grid.shape_cells))
        return res

    # -- transient ----------------------------------------------------------------
    def solve(self, terminals: Sequence, t_end: float, dt: float, bc=None,
              theta: float = 1.0, monitors=None, phi0=None, store: bool = False,
              store_every: int = 1, t_start: float = 0.0) -> Result:
        """Step from ``t_start`` to ``t_end`` (eqs.py:229-323)."""
        import torch
        if dt <= 0.0:
            raise ValueError("dt must be positive")
        if t_end <= t_start:
            raise ValueError("t_end must exceed t_start")
        if not 0.0 <= theta <= 1.0:
            raise ValueError("theta must lie in [0, 1]")
        t_wall = time.perf_counter()
        terms, bc = self._prepare(terminals, bc)
        dev = self.op_eps.dev
        N = self.op_eps.N
        if phi0 is None:
            phi0 = self.consistent_initial_condition(terms, bc, t_start)
        phi0 = np.asarray(phi0, dtype=float)
        if phi0.shape != (N,):
            raise ValueError(f"phi0 must have shape ({N},)")
        n = int(np.ceil((t_end - t_start) / dt))
        times = t_start + dt * np.arange(n + 1)

        K = self.op_eps.combine(1.0 / dt, self.op_sig, theta)
        K.material_contrast = _contrast(self.eps_cell / dt + theta * self.sigma_cell)
        Kexp = self.op_eps.combine(1.0 / dt, self.op_sig, -(1.0 - theta))
        fixed, _ = self._dirichlet(terms, bc, times[0])
        label = torch.zeros(N, dtype=torch.uint8, device=dev)
        fixed_d = h2d(fixed.astype(np.int64), torch.int64, dev)
        if fixed.size:
            label[fixed_d] = L.LABEL_FIXED
        system = EliminatedSystem(K, label, 1, precision=self.gpu.precision,
                                  with_source=True,
                                  preconditioner=resolve_preconditioner(self.cfg, self.gpu),
                                  coarsening=self.gpu.coarsening,
                                  mg_params=self.gpu.mg_params)
        system.phi.copy_(h2d(phi0, torch.float64, dev))
        prev = system.phi.clone()

        groups = [np.asarray(tt.nodes, np.int64) for tt in terms]
        gdev = upload_groups(groups, dev) if groups else None
        nt = len(terms)
        f64 = dict(dtype=torch.float64, device=dev)
        # per-step records stay on the device and come back once at the end
        cur_d = torch.zeros((n + 1, max(nt, 1)), **f64)
        volt_d = torch.zeros((n + 1, max(nt, 1)), **f64)
        en_d = torch.zeros(n + 1, **f64)
        diss_d = torch.zeros(n + 1, **f64)
        if nt:
            # terminal voltage = dual-volume weighted mean: one segment sum
            seg = h2d(np.concatenate([np.full(gr.size, j) for j, gr in enumerate(groups)]),
                      torch.int64, dev)
            wcat = h2d(np.concatenate([self._node_weights(gr) for gr in groups]),
                       torch.float64, dev)
            ncat = gdev[0]
        stored, stored_t = [], []
        iters = []

        def record(k, phi_d):
            if nt:
                volt_d[k].index_add_(0, seg, phi_d[ncat] * wcat)
            self.op_eps.quadform(phi_d, out=en_d[k:k + 1])
            self.op_sig.quadform(phi_d, out=diss_d[k:k + 1])
            if store and (k == 0 or k % max(1, store_every) == 0):
                stored.append(d2h(phi_d).copy())
                stored_t.append(times[k])

        record(0, system.phi)
        mset = monitors
        if mset is not None:
            self._record_monitors(mset, system.phi, float(times[0]), dt)
        tol = float(self.cfg.tol)
        nx, ny, nz = self.op_eps.shape
        lib = L.lib()
        step_values = self._dirichlet_values(terms, bc, fixed, dev)
        for k in range(1, n + 1):
            t = float(times[k])
            prev.copy_(system.phi)
            inj = self._inject_dev(terms, t, dev)
            st = lib.fs_apply_laplacian(L.ptr(Kexp.mx), L.ptr(Kexp.my), L.ptr(Kexp.mz),
                                        L.ptr(prev), L.ptr(inj), L.ptr(system.f),
                                        nx, ny, nz, 1, L.stream_ptr())
            L.check("fs_apply_laplacian", st)
            if fixed.size:
                system.phi[fixed_d] = step_values(t)
            _, stats = system.solve(tol, self.gpu.maxiter, warm=True)
            raise_on_status(stats, tol, "gpu-cg")
            iters.append(stats[0]["iterations"])
            if nt:
                K.group_sums(system.phi, groups, minus=Kexp, w=prev, nodes_dev=gdev,
                             out=cur_d[k])
            record(k, system.phi)
            if mset is not None:
                self._record_monitors(mset, system.phi, t, dt)
        if n >= 1:
            cur_d[0] = cur_d[1]
        cur = d2h(cur_d)[:, :nt]
        volt = d2h(volt_d)[:, :nt]
        energy = 0.5 * d2h(en_d)
        diss = d2h(diss_d)
        system.close()

        res = Result(grid=self.grid, t=times)
        if store:
            res.fields["phi"] = np.array(stored)
            res.scalars["t_stored"] = np.array(stored_t)
        for j, tt in enumerate(terms):
            res.terminals[tt.name] = {"v": volt[:, j].copy(), "i": cur[:, j].copy()}
        res.scalars["energy_electric"] = energy
        res.scalars["dissipation"] = diss
        if mset is not None:
            res.meta["monitors"] = mset.finalize()
        res.meta.update(solver=self.name, assumptions=list(self.assumptions),
                        wall_time=time.perf_counter() - t_wall,
                        grid_cells=tuple(self.grid.shape_cells), mode="transient",
                        theta=theta, dt=dt, n_factorisations=1,
                        speedup_vs_courant=dt / self.grid.courant_dt(),
                        iterations=iters, warm_start=True,
                        fp64_fallback=bool(system.fell_back),
                        coarsening=system.coarsening)
        return res

    def _record_monitors(self, mset, phi_d, t: float, dt: float) -> None:
        """One monitor sample (``eqs.py:377-386``): the state dict the
        reference hands its monitors, with this step's potential copied to
        the host.  A failing monitor never ends the solve; the error is
        reported when ``SolverConfig.verbose`` is at least 1."""
        if not hasattr(self, "_edge_props"):
            from .poisson import edge_area_over_length
            al = edge_area_over_length(self.grid)
            self._edge_props = (self.op_eps.edge_vector() / al, self.op_sig.edge_vector() / al)
        state = {"phi": d2h(phi_d), "grid": self.grid, "ops": self.ops,
                 "eps_edge": self._edge_props[0], "sigma_edge": self._edge_props[1],
                 "step": 0, "dt": dt}
        try:
            mset.record(state, t)
        except Exception as exc:  # a monitor must never kill a solve
            if getattr(self.cfg, "verbose", 0) >= 1:
                print(f"[eqs] monitor error at t={t:.4g}: {exc}", flush=True)

    # -- derived quantities ---------------------------------------------------------
    def terminal_current(self, phi_new, phi_old, dt: float, nodes,
                         theta: float = 1.0) -> float:
        """Current into the mesh from an electrode [A] (eqs.py:328-340)."""
        import torch
        dev = self.op_eps.dev
        pn = h2d(np.asarray(phi_new, float), torch.float64, dev)
        po = h2d(np.asarray(phi_old, float), torch.float64, dev)
        a = self.op_eps.apply(pn - po) / dt
        b = self.op_sig.apply(theta * pn + (1 - theta) * po)
        idx = h2d(np.asarray(nodes, np.int64), torch.int64, dev)
        return float((a + b)[idx].sum())

    def stored_energy(self, phi) -> float:
        """``0.5 phi^T L_eps phi`` [J] (eqs.py:342-344)."""
        import torch
        p = h2d(np.asarray(phi, float), torch.float64, self.op_eps.dev)
        return 0.5 * float(self.op_eps.quadform(p)[0])

    def dissipation(self, phi) -> float:
        """``phi^T L_sigma phi`` [W] (eqs.py:346-348)."""
        import torch
        p = h2d(np.asarray(phi, float), torch.float64, self.op_sig.dev)
        return float(self.op_sig.quadform(p)[0])

    def speedup_vs_courant(self, dt_used: float, eps_r_min: float = 1.0) -> float:
        return dt_used / self.grid.courant_dt(eps_r_min=eps_r_min)

    def capacitance_matrix(self, terminals: Sequence, bc=None):
        """Maxwell capacitance matrix of the same structure (eqs.py:350-357)."""
        from .poisson import PoissonSolver
        p = PoissonSolver(self.grid, self.eps_cell, self.cfg, gpu=self.gpu)
        return p.capacitance_matrix(terminals, bc)
