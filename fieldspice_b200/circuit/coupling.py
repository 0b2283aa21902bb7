"""A meshed electroquasistatic region stamped into a netlist, reduced on the GPU.

Drop-in for ``fieldspice/circuit/coupling.py``'s ``FieldRegion`` (``:55-275``):
same constructor, the netlist-device protocol of ``circuit/devices.py``
(``stamp_dc``, ``stamp_tran``, ``accept_timestep``, ``reset_state``,
``reset_history``, ``set_time``, ``op``), ``terminal_admittance`` and
``asymmetry``, so that the reference's ``Netlist.add_device`` (which reads
devices by duck typing, ``circuit/mna.py:457-492``) accepts it unchanged.

Per distinct step size (cached, ``coupling.py:140-181``) the operator is
``K = L_eps/dt + L_sigma`` (``L_sigma`` alone at dc) with every electrode node
fixed.  The ``nE`` unit excitations are solved together as one block of
right-hand sides by the GPU CG plan; each solution is
``phi_b = P^T e_b - S^T W e_b`` with ``W = K_ii^-1 K_it``, and the electrode
charge integration on the device gives
``Y[a, b] = sum_{n in T_a} (K phi_b)_n = (K_tt - K_ti W)[a, b]``.

Per time step (``coupling.py:183-193``) one more solve gives the history
source: ``K phi' = f`` on the interior with the electrodes at 0 and
``f = (L_eps/dt) phi``, so ``f_eff[a] = sum_{n in T_a} (f - K phi')_n``.  The
back-substitution after an accepted step (``coupling.py:248-262``,
``u = K_ii^-1 (f_i - K_it v)``) is, by linearity, ``phi' + sum_b v_b phi_b``:
the cached unit solutions make it one superposition kernel instead of a
second solve.  The AC stamp (``K = L_sigma + j w L_eps``) is the same unit
excitation with the complex-symmetric solve of ``solvers/ac.py``.
"""

from __future__ import annotations

import ctypes
from typing import Any, Mapping, Sequence

import numpy as np

from .. import _lib as L
from ..device import (DeviceOperator, EliminatedSystem, block_rhs, d2h, h2d, pad_rhs,
                      rhs_blocks, upload_groups)
from ..solvers.base import GPUConfig, SolverConfig, resolve_preconditioner
from ..solvers.poisson import raise_on_status, upload_cell_property

__all__ = ["FieldRegion", "FieldCircuitSystem"]


def _stamp_g(G, i: int, j: int, value: float) -> None:
    """Accumulate into ``G[i, j]``; ground (negative) rows and columns are
    dropped; ``G`` may expose ``add(i, j, v)`` (``circuit/devices.py:186-200``)."""
    if i < 0 or j < 0:
        return
    add = getattr(G, "add", None)
    if add is not None:
        add(i, j, value)
    else:
        G[i, j] += value


def _stamp_i(I, i: int, value: float) -> None:
    """Accumulate into ``I[i]``; the ground row is dropped (``devices.py:203-207``)."""
    if i < 0:
        return
    I[i] += value


class _Reduction:
    """The cached reduction for one step size: ``K``, ``Y`` and the device
    unit-excitation solutions, plus the lazily built history system."""

    def __init__(self, dt):
        self.dt = dt
        self.K: DeviceOperator | None = None
        self.K_hist: DeviceOperator | None = None   # L_eps / dt
        self.Y: np.ndarray | None = None
        self.blocks: list[tuple[int, int, int, Any]] = []   # (b0, cols, k, phi)
        self.solved = False          # interior exists and K is nonzero
        self.history: EliminatedSystem | None = None
        self.f_eff: np.ndarray | None = None
        self.f_version = -1

    def close(self):
        if self.history is not None:
            self.history.close()
            self.history = None
        self.blocks = []


class FieldRegion:
    """A meshed quasi-static field region stamped into a netlist.

    ``grid``, ``eps_cell`` (absolute [F/m]) and ``sigma_cell`` [S/m] describe
    the region; each of ``terminals`` becomes one circuit node, named by
    ``circuit_nodes`` (default: each terminal's ``circuit_node`` or its name).
    ``config.tol`` is the relative residual every GPU solve reaches; ``gpu``
    selects precision and preconditioner as for the Poisson solver.
    """

    linear = True
    dynamic = True
    assumptions = ("A1a", "A2", "A3", "A10", "A12")

    def __init__(self, name: str, grid, eps_cell, sigma_cell,
                 terminals: Sequence, circuit_nodes: Sequence[str] | None = None,
                 config: SolverConfig | None = None, *, gpu: GPUConfig | None = None):
        import torch
        self.name = str(name)
        self.grid = grid
        self.cfg = config or SolverConfig()
        self.gpu = gpu or GPUConfig()
        self.terminals = list(terminals)
        if len(self.terminals) < 1:
            raise ValueError("a field region needs at least one terminal")
        if circuit_nodes is None:
            circuit_nodes = [getattr(t, "circuit_node", None) or t.name
                             for t in self.terminals]
        circuit_nodes = [str(c) for c in circuit_nodes]
        if len(circuit_nodes) != len(self.terminals):
            raise ValueError("circuit_nodes must match terminals in length")
        self.nodes = tuple(circuit_nodes)
        shape = tuple(grid.shape_cells)
        for arr, nm in ((eps_cell, "eps_cell"), (sigma_cell, "sigma_cell")):
            if np.shape(arr) != shape:
                raise ValueError(f"{nm} must have shape {shape}")
        n = int(np.prod(grid.shape_nodes))
        elec = [np.asarray(t.nodes, np.int64).ravel() for t in self.terminals]
        flat = np.concatenate(elec)
        if np.unique(flat).size != flat.size:
            raise ValueError("terminals overlap: a node belongs to two electrodes")
        if flat.size and (flat.min() < 0 or flat.max() >= n):
            raise ValueError("terminal node index out of range")
        for t, e in zip(self.terminals, elec):
            if e.size == 0:
                raise ValueError(f"terminal {t.name!r} has no nodes")
        _, eps_dev, eps_min, _ = upload_cell_property(eps_cell, grid, "eps_cell")
        if eps_min <= 0.0:
            raise ValueError("eps_cell must be positive and ABSOLUTE [F/m]")
        _, sig_dev, _, _ = upload_cell_property(sigma_cell, grid, "sigma_cell")
        self.op_eps = DeviceOperator(grid, eps_dev)
        self.op_sig = DeviceOperator(grid, sig_dev)
        dev = self.op_eps.dev
        self.N = n
        self.n_interior = n - int(flat.size)
        self._elec = [h2d(e, torch.int64, dev) for e in elec]
        self._gdev = upload_groups(self._elec, dev)
        self._label = torch.zeros(n, dtype=torch.uint8, device=dev)
        self._group = torch.full((n,), -1, dtype=torch.int16, device=dev)
        for c, e in enumerate(self._elec):
            self._label[e] = L.LABEL_FIXED
        self._cache: dict[float, _Reduction] = {}
        self._phi = torch.zeros(n, dtype=torch.float64, device=dev)
        self._version = 0
        self.asymmetry: float = 0.0
        self.last_history_stats: dict | None = None   # the last history solve's
        self.t: float = 0.0
        self.limited: bool = False

    # -- state ---------------------------------------------------------------
    @property
    def phi(self) -> np.ndarray:
        """The stored field (integration history) [V], a host copy."""
        return d2h(self._phi)

    @phi.setter
    def phi(self, value) -> None:
        import torch
        a = np.asarray(value, dtype=float).ravel()
        if a.size != self.N:
            raise ValueError(f"phi must have {self.N} entries")
        self._phi = h2d(a, torch.float64, self.op_eps.dev)
        self._version += 1

    # -- reduction -------------------------------------------------------------
    def _excite(self, phi, cols: Sequence[int], k: int) -> None:
        """Unit excitations of electrodes ``cols`` into an N*k block."""
        self._group.fill_(-1)
        for c, j in enumerate(cols):
            self._group[self._elec[j]] = c
        nx, ny, nz = self.op_eps.shape
        L.check("fs_fill_unit_excitation", L.lib().fs_fill_unit_excitation(
            L.ptr(self._group), L.ptr(self._label), L.ptr(phi), nx, ny, nz, k,
            L.stream_ptr()))

    def _reduce(self, dt: float | None) -> _Reduction:
        """Schur-complement reduction for a step size (cached; coupling.py:140-181)."""
        import torch
        key = float(dt) if dt is not None else 0.0
        if key in self._cache:
            return self._cache[key]
        entry = _Reduction(dt)
        K = self.op_sig if dt is None else self.op_eps.combine(1.0 / dt, self.op_sig, 1.0)
        entry.K = K
        if dt is not None:
            entry.K_hist = self.op_eps.combine(1.0 / dt, self.op_sig, 0.0)
        nE = len(self._elec)
        stats = L.prop_stats(K.m)
        if stats[0] == 0.0 and stats[1] == 0.0:
            # no coupling at all (e.g. sigma == 0 at dc): an open circuit
            entry.Y = np.zeros((nE, nE))
            self.asymmetry = 0.0
            self._cache[key] = entry
            return entry
        Y = np.zeros((nE, nE))
        tol = float(self.cfg.tol)
        # electrodes in blocks of 32-byte nodes (8 FP32 / 4 FP64 RHS)
        for cols in rhs_blocks(nE, block_rhs(self.gpu.precision)):
            b0 = cols[0]
            k = pad_rhs(len(cols))
            if self.n_interior == 0:
                phi = torch.zeros(self.N * k, dtype=torch.float64, device=self.op_eps.dev)
                self._excite(phi, cols, k)
            else:
                system = EliminatedSystem(K, self._label, len(cols),
                                          precision=self.gpu.precision,
                                          preconditioner=resolve_preconditioner(
                                              self.cfg, self.gpu),
                                          coarsening=self.gpu.coarsening,
                                          mg_params=self.gpu.mg_params)
                self._excite(system.phi, cols, k)
                _, st = system.solve(tol, self.gpu.maxiter)
                raise_on_status(st, tol, "gpu-cg")
                phi = system.phi.clone()
                system.close()
                entry.blocks.append((b0, len(cols), k, phi))
            Q = K.group_sums(phi, self._elec, nrhs=k, nodes_dev=self._gdev)
            Y[:, cols] = Q[:, :len(cols)]
        entry.solved = self.n_interior > 0
        self.asymmetry = float(np.abs(Y - Y.T).max() / max(np.abs(Y).max(), 1e-300))
        entry.Y = 0.5 * (Y + Y.T)
        self._cache[key] = entry
        return entry

    def _history(self, entry: _Reduction, dt: float | None) -> np.ndarray:
        """``f_eff`` [A]: the history current source of the stored field
        (coupling.py:183-193); one interior solve per new field."""
        import torch
        nE = len(self._elec)
        if dt is None:
            return np.zeros(nE)
        if entry.f_version == self._version:
            return entry.f_eff
        if not entry.solved:
            # P f with f = (L_eps/dt) phi: the electrode sums of K_hist phi
            f = entry.K_hist.group_sums(self._phi, self._elec, nodes_dev=self._gdev)[:, 0]
        else:
            if entry.history is None:
                entry.history = EliminatedSystem(
                    entry.K, self._label, 1, precision=self.gpu.precision,
                    with_source=True,
                    preconditioner=resolve_preconditioner(self.cfg, self.gpu),
                    coarsening=self.gpu.coarsening,
                    mg_params=self.gpu.mg_params)
            hs = entry.history
            nx, ny, nz = self.op_eps.shape
            m = entry.K_hist
            L.check("fs_apply_laplacian", L.lib().fs_apply_laplacian(
                L.ptr(m.mx), L.ptr(m.my), L.ptr(m.mz), L.ptr(self._phi), None,
                L.ptr(hs.f), nx, ny, nz, 1, L.stream_ptr()))
            tol = float(self.cfg.tol)
            _, st = hs.solve(tol, self.gpu.maxiter, warm=True)
            self.last_history_stats = st[0]
            raise_on_status(st, tol, "gpu-cg")
            # sum_{n in T} (K phi' - (L_eps/dt) phi)_n = K_ti u - P f
            f = -entry.K.group_sums(hs.phi, self._elec, minus=m, w=self._phi,
                                    nodes_dev=self._gdev)[:, 0]
        entry.f_eff = np.asarray(f, dtype=float)
        entry.f_version = self._version
        return entry.f_eff

    # -- netlist-device protocol --------------------------------------------------
    def extra_unknowns(self) -> tuple[str, ...]:
        return ()

    def set_time(self, t: float) -> None:
        self.t = float(t)

    def _indices(self, nmap: Mapping[str, int]) -> list[int]:
        return [nmap.get(n, -1) for n in self.nodes]

    def stamp_dc(self, G, I, x, nmap: Mapping[str, int], t=None) -> None:
        Y = self._reduce(None).Y
        idx = self._indices(nmap)
        for a in range(len(idx)):
            for b in range(len(idx)):
                _stamp_g(G, idx[a], idx[b], Y[a, b])

    def stamp_tran(self, G, I, x, x_prev, dt: float, nmap: Mapping[str, int],
                   t=None) -> None:
        entry = self._reduce(dt)
        Y = entry.Y
        f = self._history(entry, dt)
        idx = self._indices(nmap)
        for a in range(len(idx)):
            for b in range(len(idx)):
                _stamp_g(G, idx[a], idx[b], Y[a, b])
            _stamp_i(I, idx[a], f[a])

    def stamp_ac(self, Y_mat, J, x_op, omega: float, nmap: Mapping[str, int]) -> None:
        """Frequency domain, ``K = L_sigma + j w L_eps`` with no history
        (coupling.py:214-236): the complex Schur complement by unit excitation
        of the electrodes, one complex-symmetric GPU solve per electrode block."""
        from ..solvers.ac import complex_admittance
        opB = self.op_eps.combine(float(omega), self.op_eps, 0.0)
        Yeff, _ = complex_admittance(self.op_sig, opB, self._elec, float(self.cfg.tol),
                                     self.gpu)
        idx = self._indices(nmap)
        for a in range(len(idx)):
            for b in range(len(idx)):
                _stamp_g(Y_mat, idx[a], idx[b], Yeff[a, b])

    def accept_timestep(self, x, x_prev, dt: float, nmap: Mapping[str, int]) -> None:
        """Back-substitute the field once the step is accepted (coupling.py:248-262)."""
        import torch
        entry = self._reduce(dt)
        v = [0.0 if nmap.get(n, -1) < 0 else float(x[nmap[n]]) for n in self.nodes]
        if entry.solved and dt is not None:
            self._history(entry, dt)           # phi' for the stored field
            base = entry.history.phi
            out = torch.empty_like(self._phi)
            lib = L.lib()
            for b0, cols, k, phi in entry.blocks:
                coef = (ctypes.c_double * cols)(*v[b0:b0 + cols])
                L.check("fs_rhs_superpose", lib.fs_rhs_superpose(
                    L.ptr(phi), k, 0, cols, coef, L.ptr(base), L.ptr(out), self.N,
                    L.stream_ptr()))
                base = out
        else:
            out = torch.zeros_like(self._phi)
            for e, vb in zip(self._elec, v):
                out[e] = vb
        self._phi = out
        self._version += 1

    def reset_state(self) -> None:
        """Per-Newton-iteration reset: deliberately a no-op, the stored field
        is integration history (coupling.py:264-280)."""
        return None

    def reset_history(self) -> None:
        """Discard the stored field, starting a fresh transient."""
        self._phi = self._phi.new_zeros(self.N)
        self._version += 1

    def terminal_admittance(self, dt: float | None = None) -> np.ndarray:
        """The reduced ``nE x nE`` terminal admittance [S] for a step size."""
        return self._reduce(dt).Y

    def op(self, x, nmap: Mapping[str, int]) -> dict[str, float]:
        return {f"{self.name}.v[{n}]": (0.0 if nmap.get(n, -1) < 0 else float(x[nmap[n]]))
                for n in self.nodes}

    def close(self) -> None:
        """Release the cached device systems."""
        for e in self._cache.values():
            e.close()
        self._cache.clear()

    def __repr__(self) -> str:
        return f"FieldRegion({self.name!r}, nodes={self.nodes})"


class FieldCircuitSystem:
    """A field region plus a netlist, solved together.

    ``netlist`` is any netlist with ``add_device`` (the reference's
    ``fieldspice.circuit.mna.Netlist``); ``solver`` the MNA solver class
    (default: the reference's ``MNASolver``, imported when first needed; the
    circuit simulator itself is not part of this package).
    """

    def __init__(self, region: FieldRegion, netlist, solver=None):
        self.region = region
        self.netlist = netlist
        self._solver = solver
        netlist.add_device(region)

    def _mna(self):
        if self._solver is None:
            try:
                from fieldspice.circuit.mna import MNASolver
            except ImportError as exc:
                raise ImportError("FieldCircuitSystem needs an MNA solver: pass "
                                  "solver=, or install the fieldspice package") from exc
            self._solver = MNASolver
        return self._solver(self.netlist)

    def transient(self, t_end: float, dt: float, **kw):
        return self._mna().transient(t_end=t_end, dt=dt, **kw)

    def dc(self):
        return self._mna().dc()
