"""Harmonic (phasor) quasi-static solve on the GPU.

Drop-in for ``fieldspice/solvers/ac.py``'s ``ACSolver`` (``:34-164``): same
constructor (absolute permittivity that may be complex, ``eps' - j eps''``, or
a callable of frequency; conductivity), ``solve``, ``admittance_matrix``,
``impedance_matrix`` and ``s_parameters``.

Per frequency the system is ``K phi = 0`` with ``K = L_sigma + j w L_eps``
(``ac.py:92-95``) and ``phi`` fixed on every terminal's nodes; every wall is
insulating (the reference ignores ``bc``).  The reference factorises ``K``
with a sparse LU; here ``fs_ac_solve`` runs conjugate-orthogonal CG (the
Krylov method for complex-symmetric matrices) preconditioned by the real
multigrid V-cycle of ``|A| + |B|`` (``K = A + jB``), all unit excitations of
one frequency as one block (up to 8 complex right-hand sides per solve).
Terminal currents are the FP64 charge integrals ``sum_{n in T} (K phi)_n``.
"""

from __future__ import annotations

import ctypes
import math
import time
from typing import Callable, Sequence

import numpy as np

from .. import _lib as L
from ..device import DeviceOperator, d2h, h2d, upload_groups
from .base import GPUConfig, Result, SolverConfig
from .poisson import check_terminals, raise_on_status

__all__ = ["ACSolver", "complex_admittance"]

MAX_CPLX = 8


def _k_columns(nc: int) -> int:
    k = 2
    while k < 2 * nc:
        k *= 2
    return k


def _ac_block(opA: DeviceOperator, opB: DeviceOperator, label, phi, nc: int, tol: float,
              maxiter: int | None, precond: int):
    """One ``fs_ac_solve`` call; ``phi`` (N x K FP64 device, Dirichlet values in
    place) receives the solution.  Returns the per-RHS stats dicts."""
    import torch
    lib = L.lib()
    nx, ny, nz = opA.shape
    nb = ctypes.c_size_t()
    L.check("fs_ac_workspace_bytes",
            lib.fs_ac_workspace_bytes(nx, ny, nz, nc, precond, ctypes.byref(nb)))
    ws = torch.empty(nb.value, dtype=torch.uint8, device=opA.dev)
    if ws.data_ptr() % 256:
        raise RuntimeError("device allocation is not 256-byte aligned")
    stats = (L.FsRhsStats * nc)()
    mi = max(500, int(10 * math.sqrt(opA.N))) if maxiter is None else int(maxiter)
    st = lib.fs_ac_solve(nx, ny, nz, nc, precond, L.ptr(opA.m), L.ptr(opB.m), L.ptr(label),
                         L.ptr(phi), float(tol), mi, L.ptr(ws), nb.value, stats,
                         L.stream_ptr())
    L.check("fs_ac_solve", st)
    return [{"iterations": s.iterations, "status": s.status, "relres": s.relres,
             "bnorm": s.bnorm, "reliable_updates": s.reliable_updates} for s in stats[:nc]]


def _complex_charges(opA: DeviceOperator, opB: DeviceOperator, phi, k: int, nodes_dev):
    """``sum_{n in T_g} (K phi_c)_n`` for every group g and complex column c
    (``K = A + jB``; phi N x k with real parts in columns < k/2)."""
    h = k // 2
    QA = opA.group_sums(phi, None, nrhs=k, nodes_dev=nodes_dev)
    QB = opB.group_sums(phi, None, nrhs=k, nodes_dev=nodes_dev)
    return (QA[:, :h] - QB[:, h:]) + 1j * (QA[:, h:] + QB[:, :h])


def complex_admittance(opA: DeviceOperator, opB: DeviceOperator, term_dev, tol: float,
                       gpu: GPUConfig | None = None) -> tuple[np.ndarray, list]:
    """``Y[i, j] = sum_{n in T_i} (K phi_j)_n`` with terminal ``j`` at 1 V and
    every other terminal at 0 V (``ac.py:116-148``), ``K = A + jB`` given by
    its edge masses; ``term_dev``: int64 node tensors per terminal.  Returns
    ``(Y, stats)``; with no free node ``Y = K_tt`` (no solve)."""
    import torch
    gpu = gpu or GPUConfig()
    N = opA.N
    nt = len(term_dev)
    dev = opA.dev
    label = torch.zeros(N, dtype=torch.uint8, device=dev)
    for t in term_dev:
        label[t] = L.LABEL_FIXED
    n_fixed = int(sum(int(t.numel()) for t in term_dev))
    gdev = upload_groups(list(term_dev), dev)
    group = torch.full((N,), -1, dtype=torch.int16, device=dev)
    precond = L.PRECOND_JACOBI if gpu.preconditioner == "jacobi" else L.PRECOND_MG
    Y = np.zeros((nt, nt), dtype=complex)
    stats_all: list = []
    nx, ny, nz = opA.shape
    for b0 in range(0, nt, MAX_CPLX):
        cols = list(range(b0, min(nt, b0 + MAX_CPLX)))
        nc = len(cols)
        k = _k_columns(nc)
        phi = torch.zeros(N * k, dtype=torch.float64, device=dev)
        group.fill_(-1)
        for c, j in enumerate(cols):
            group[term_dev[j]] = c
        L.check("fs_fill_unit_excitation", L.lib().fs_fill_unit_excitation(
            L.ptr(group), L.ptr(label), L.ptr(phi), nx, ny, nz, k, L.stream_ptr()))
        if n_fixed < N:
            st = _ac_block(opA, opB, label, phi, nc, tol, gpu.maxiter, precond)
            raise_on_status(st, tol, "gpu-cocg")
            stats_all.extend(st)
        Q = _complex_charges(opA, opB, phi, k, gdev)
        Y[:, cols] = Q[:, :nc]
    return Y, stats_all


class ACSolver:
    """Harmonic (phasor) quasi-static solver (``ac.py:34-77``).

    ``eps_cell``: absolute permittivity [F/m] per cell, possibly complex
    (``eps' - j eps''`` for dielectric loss) or a callable ``f(freq)``
    returning such an array; ``sigma_cell``: conductivity [S/m] per cell.
    ``gpu`` selects the preconditioner (multigrid by default).
    """

    name = "ac"
    assumptions = ("A1a", "A2", "A10", "A12")

    def __init__(self, grid, eps_cell: np.ndarray | Callable[[float], np.ndarray],
                 sigma_cell: np.ndarray, config: SolverConfig | None = None,
                 operators=None, *, gpu: GPUConfig | None = None):
        self.grid = grid
        self.cfg = config or SolverConfig()
        self.gpu = gpu or GPUConfig()
        shape = tuple(grid.shape_cells)
        self._eps_fn = eps_cell if callable(eps_cell) else None
        if not callable(eps_cell):
            eps = np.asarray(eps_cell)
            if eps.shape != shape:
                raise ValueError(f"eps_cell must have shape {shape}")
            self._eps = eps
        sigma_cell = np.asarray(sigma_cell, dtype=float)
        if sigma_cell.shape != shape:
            raise ValueError(f"sigma_cell must have shape {shape}")
        if np.any(sigma_cell < 0):
            raise ValueError("sigma_cell must be non-negative")
        self.op_sig = DeviceOperator(grid, sigma_cell)
        self._eps_cache: dict = {}
        self._t0 = 0.0

    # -- operators ---------------------------------------------------------------
    def _eps_ops(self, freq: float):
        """Device masses of Re and Im of the permittivity (ac.py:79-90)."""
        eps = self._eps_fn(freq) if self._eps_fn is not None else self._eps
        key = id(eps) if self._eps_fn is None else hash(float(freq))
        if key in self._eps_cache:
            return self._eps_cache[key]
        eps = np.asarray(eps)
        if eps.shape != tuple(self.grid.shape_cells):
            raise ValueError(f"eps_cell must have shape {tuple(self.grid.shape_cells)}")
        op_re = DeviceOperator(self.grid, np.real(eps).astype(float))
        op_im = None
        if np.iscomplexobj(eps) and np.any(np.imag(eps) != 0.0):
            op_im = DeviceOperator(self.grid, np.imag(eps).astype(float))
        self._eps_cache[key] = (op_re, op_im)
        return op_re, op_im

    def _system(self, freq: float):
        """``(A, B)`` with ``K = L_sigma + j w L_eps = A + jB`` (ac.py:92-95)."""
        w = 2.0 * np.pi * float(freq)
        op_re, op_im = self._eps_ops(freq)
        opA = self.op_sig if op_im is None else self.op_sig.combine(1.0, op_im, -w)
        opB = op_re.combine(w, op_re, 0.0)
        return opA, opB

    # -- solves -------------------------------------------------------------------
    def solve(self, terminals: Sequence, freqs, bc=None) -> Result:
        """Terminal voltages and currents at each frequency (ac.py:97-121):
        every terminal held at its (complex) value, currents by charge
        integration of ``K phi``."""
        import torch
        self._t0 = time.perf_counter()
        freqs = np.atleast_1d(np.asarray(freqs, dtype=float))
        terms = check_terminals(list(terminals), self.grid)
        N = self.op_sig.N
        dev = self.op_sig.dev
        term_dev = [h2d(np.asarray(t.nodes, np.int64), torch.int64, dev) for t in terms]
        gdev = upload_groups(term_dev, dev) if term_dev else None
        label = torch.zeros(N, dtype=torch.uint8, device=dev)
        for t in term_dev:
            label[t] = L.LABEL_FIXED
        n_fixed = int(sum(int(t.numel()) for t in term_dev))
        precond = L.PRECOND_JACOBI if self.gpu.preconditioner == "jacobi" else L.PRECOND_MG
        out_v = {t.name: np.zeros(freqs.size, dtype=complex) for t in terms}
        out_i = {t.name: np.zeros(freqs.size, dtype=complex) for t in terms}
        iters = []
        tol = float(self.cfg.tol)
        for kf, f in enumerate(freqs):
            opA, opB = self._system(f)
            phi_h = np.zeros((N, 2))
            for t in terms:
                v = complex(t.value_at(0.0) or 0.0)
                phi_h[t.nodes, 0] = v.real
                phi_h[t.nodes, 1] = v.imag
            phi = h2d(phi_h.ravel(), torch.float64, dev)
            if terms and n_fixed < N:
                st = _ac_block(opA, opB, label, phi, 1, tol, self.gpu.maxiter, precond)
                raise_on_status(st, tol, "gpu-cocg")
                iters.append(st[0]["iterations"])
            ph = d2h(phi).reshape(N, 2)
            if terms:
                Q = _complex_charges(opA, opB, phi, 2, gdev)
            for j, t in enumerate(terms):
                out_v[t.name][kf] = np.mean(ph[t.nodes, 0] + 1j * ph[t.nodes, 1])
                out_i[t.name][kf] = Q[j, 0]
        res = Result(grid=self.grid, t=np.zeros(0))
        res.scalars["freq"] = freqs
        for t in terms:
            res.terminals[t.name] = {"v": out_v[t.name], "i": out_i[t.name]}
        res.meta.update(solver=self.name, assumptions=list(self.assumptions),
                        wall_time=time.perf_counter() - self._t0,
                        grid_cells=tuple(self.grid.shape_cells), mode="ac",
                        n_freqs=int(freqs.size), iterations=iters)
        return res

    def admittance_matrix(self, terminals: Sequence, freqs, bc=None) -> np.ndarray:
        """``(nf, nt, nt)`` admittance [S] by unit excitation (ac.py:123-148)."""
        import torch
        freqs = np.atleast_1d(np.asarray(freqs, dtype=float))
        terms = check_terminals(list(terminals), self.grid)
        dev = self.op_sig.dev
        term_dev = [h2d(np.asarray(t.nodes, np.int64), torch.int64, dev) for t in terms]
        nt = len(terms)
        Y = np.zeros((freqs.size, nt, nt), dtype=complex)
        self.last_stats = []
        for kf, f in enumerate(freqs):
            opA, opB = self._system(f)
            Y[kf], st = complex_admittance(opA, opB, term_dev, float(self.cfg.tol), self.gpu)
            self.last_stats.append(st)
        return Y

    def impedance_matrix(self, terminals, freqs, bc=None) -> np.ndarray:
        """Pseudo-inverse of the admittance matrix [ohm] (ac.py:150-157)."""
        Y = self.admittance_matrix(terminals, freqs, bc)
        return np.stack([np.linalg.pinv(y) for y in Y])

    def s_parameters(self, terminals, freqs, z0: float = 50.0, bc=None) -> np.ndarray:
        from ..extraction import s_parameters as _s
        return _s(self.admittance_matrix(terminals, freqs, bc), z0)
