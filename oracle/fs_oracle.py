"""CPU oracle of fieldspice's elliptic solve path -- TEST INFRASTRUCTURE ONLY.

This module restates, in NumPy/SciPy, the reference algorithm of the path the
GPU library replaces.  Only ``tests/``, ``__graft_entry__.smoke()`` and the
CPU-baseline leg of ``bench.py`` may import it, to check results against,
never as the thing measured or shipped.  The product path
(``fieldspice_b200``) does not import it and has no CPU fallback.

Parity pin: ``tests/golden/make_golden.py`` imported the reference package
and recorded its outputs (masses, Laplacians, capacitance matrices, EQS
currents) as ``tests/golden/*.npz``; ``tests/test_oracle_golden.py`` checks
this restatement against every one of them.

Every function cites the reference file:line it follows (paths inside the
fieldspice project).  SciPy (the reference's own dependency, installed here
at 1.18) provides the CSR products and ``cg``/``splu``, as in the reference.
"""

from __future__ import annotations

import math
import warnings
from dataclasses import dataclass

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

EPS0 = 1.0 / ((4e-7 * math.pi * 1.0000000000552) * 299_792_458.0 ** 2)  # units.py:20-26


# ---------------------------------------------------------------------------
# Grid metric -- fieldspice/grid.py:196-207 (_make_axis), :322-327, :398-420
# ---------------------------------------------------------------------------
@dataclass
class Grid:
    """Node coordinates per axis; metric arrays as in grid.py."""
    xn: np.ndarray
    yn: np.ndarray
    zn: np.ndarray

    @classmethod
    def uniform(cls, extent, n):
        # grid.py:533-546
        axes = [np.linspace(e[0], e[1], int(k) + 1) for e, k in zip(extent, n)]
        return cls(*axes)

    @classmethod
    def from_any(cls, g):
        return cls(np.asarray(g.xn, float), np.asarray(g.yn, float),
                   np.asarray(g.zn, float))

    def _axis(self, a):
        h = np.diff(a)
        hd = np.empty(a.size)
        hd[1:-1] = 0.5 * (h[:-1] + h[1:])
        hd[0] = 0.5 * h[0]
        hd[-1] = 0.5 * h[-1]
        return h, hd

    @property
    def hx(self): return self._axis(self.xn)[0]
    @property
    def hy(self): return self._axis(self.yn)[0]
    @property
    def hz(self): return self._axis(self.zn)[0]
    @property
    def hxd(self): return self._axis(self.xn)[1]
    @property
    def hyd(self): return self._axis(self.yn)[1]
    @property
    def hzd(self): return self._axis(self.zn)[1]

    @property
    def shape_nodes(self):
        return (self.xn.size, self.yn.size, self.zn.size)

    @property
    def shape_cells(self):
        return (self.xn.size - 1, self.yn.size - 1, self.zn.size - 1)

    @property
    def shape_edges(self):
        nx, ny, nz = self.shape_cells
        return ((nx, ny + 1, nz + 1), (nx + 1, ny, nz + 1), (nx + 1, ny + 1, nz))

    @property
    def n_nodes(self):
        return int(np.prod(self.shape_nodes))

    @property
    def n_edges(self):
        return int(sum(np.prod(s) for s in self.shape_edges))

    def node_volumes(self):
        # grid.py:388-396
        return (self.hxd[:, None, None] * self.hyd[None, :, None]
                * self.hzd[None, None, :])

    def edge_lengths(self):
        # grid.py:398-405
        sx, sy, sz = self.shape_edges
        return (np.ascontiguousarray(np.broadcast_to(self.hx[:, None, None], sx)),
                np.ascontiguousarray(np.broadcast_to(self.hy[None, :, None], sy)),
                np.ascontiguousarray(np.broadcast_to(self.hz[None, None, :], sz)))

    def edge_dual_areas(self):
        # grid.py:407-420
        sx, sy, sz = self.shape_edges
        ax = np.broadcast_to(self.hyd[None, :, None] * self.hzd[None, None, :], sx)
        ay = np.broadcast_to(self.hxd[:, None, None] * self.hzd[None, None, :], sy)
        az = np.broadcast_to(self.hxd[:, None, None] * self.hyd[None, :, None], sz)
        return (np.ascontiguousarray(ax), np.ascontiguousarray(ay),
                np.ascontiguousarray(az))


# ---------------------------------------------------------------------------
# Incidence operators -- fieldspice/operators.py:59-138
# ---------------------------------------------------------------------------
def _ids(shape, offset=0):
    return (offset + np.arange(int(np.prod(shape)))).reshape(shape)


def _assemble(terms, shape):
    # operators.py:63-68
    rows = np.concatenate([np.asarray(r).ravel() for r, _, _ in terms])
    cols = np.concatenate([np.asarray(c).ravel() for _, c, _ in terms])
    vals = np.concatenate([np.full(np.asarray(c).size, v, dtype=np.float64)
                           for _, c, v in terms])
    return sp.coo_matrix((vals, (rows, cols)), shape=shape).tocsr()


def grad_node_edge(g: Grid):
    """``(G phi)_e = phi_head - phi_tail`` (operators.py:71-91)."""
    nid = _ids(g.shape_nodes)
    sx, sy, sz = g.shape_edges
    nex, ney = int(np.prod(sx)), int(np.prod(sy))
    ex, ey, ez = _ids(sx, 0), _ids(sy, nex), _ids(sz, nex + ney)
    terms = [(ex, nid[1:, :, :], 1.0), (ex, nid[:-1, :, :], -1.0),
             (ey, nid[:, 1:, :], 1.0), (ey, nid[:, :-1, :], -1.0),
             (ez, nid[:, :, 1:], 1.0), (ez, nid[:, :, :-1], -1.0)]
    return _assemble(terms, (g.n_edges, g.n_nodes))


def _face_shapes(g: Grid):
    nx, ny, nz = g.shape_cells
    return ((nx + 1, ny, nz), (nx, ny + 1, nz), (nx, ny, nz + 1))


def curl_edge_face(g: Grid):
    """Right-handed face circulation (operators.py:94-119)."""
    sx, sy, sz = g.shape_edges
    fx, fy, fz = _face_shapes(g)
    nex, ney = int(np.prod(sx)), int(np.prod(sy))
    nfx, nfy = int(np.prod(fx)), int(np.prod(fy))
    ex, ey, ez = _ids(sx, 0), _ids(sy, nex), _ids(sz, nex + ney)
    Fx, Fy, Fz = _ids(fx, 0), _ids(fy, nfx), _ids(fz, nfx + nfy)
    terms = [(Fx, ez[:, 1:, :], 1.0), (Fx, ez[:, :-1, :], -1.0),
             (Fx, ey[:, :, :-1], 1.0), (Fx, ey[:, :, 1:], -1.0),
             (Fy, ex[:, :, 1:], 1.0), (Fy, ex[:, :, :-1], -1.0),
             (Fy, ez[:-1, :, :], 1.0), (Fy, ez[1:, :, :], -1.0),
             (Fz, ey[1:, :, :], 1.0), (Fz, ey[:-1, :, :], -1.0),
             (Fz, ex[:, :-1, :], 1.0), (Fz, ex[:, 1:, :], -1.0)]
    nf = sum(int(np.prod(s)) for s in (fx, fy, fz))
    return _assemble(terms, (nf, g.n_edges))


def div_face_cell(g: Grid):
    """Net outward flux per cell (operators.py:122-138)."""
    fx, fy, fz = _face_shapes(g)
    nfx, nfy = int(np.prod(fx)), int(np.prod(fy))
    Fx, Fy, Fz = _ids(fx, 0), _ids(fy, nfx), _ids(fz, nfx + nfy)
    cid = _ids(g.shape_cells)
    terms = [(cid, Fx[1:, :, :], 1.0), (cid, Fx[:-1, :, :], -1.0),
             (cid, Fy[:, 1:, :], 1.0), (cid, Fy[:, :-1, :], -1.0),
             (cid, Fz[:, :, 1:], 1.0), (cid, Fz[:, :, :-1], -1.0)]
    nf = sum(int(np.prod(s)) for s in (fx, fy, fz))
    return _assemble(terms, (int(np.prod(g.shape_cells)), nf))


# ---------------------------------------------------------------------------
# Material averaging and masses -- fieldspice/operators.py:144-237, :302-315
# ---------------------------------------------------------------------------
def _combine(q, w, mode):
    # operators.py:225-237: sums over the quadrant axis, left to right
    wsum = w.sum(axis=0)
    safe = np.where(wsum > 0, wsum, 1.0)
    if mode in ("parallel", "arithmetic"):
        return (q * w).sum(axis=0) / safe
    if mode in ("harmonic", "series"):
        qq = np.where(q > 0, q, np.finfo(float).tiny)
        return safe / (w / qq).sum(axis=0)
    raise ValueError(f"unknown averaging mode {mode!r}")


def cell_to_edge(g: Grid, prop, mode="parallel"):
    """Dual-area weighted mean of the four cells around each edge.

    operators.py:144-222: cells are edge-padded at the walls; quadrants are
    taken in the order (0,0), (0,1), (1,0), (1,1).
    """
    prop = np.asarray(prop, dtype=float)
    if prop.shape != g.shape_cells:
        raise ValueError(f"prop must have shape {g.shape_cells}, got {prop.shape}")
    p = np.pad(prop, 1, mode="edge")

    def halves(h):
        return (np.concatenate([[0.0], 0.5 * h]), np.concatenate([0.5 * h, [0.0]]))

    ylo, yhi = halves(g.hy)
    zlo, zhi = halves(g.hz)
    xlo, xhi = halves(g.hx)
    combos = [(0, 0), (0, 1), (1, 0), (1, 1)]
    out = []
    sx = g.shape_edges[0]
    q, w = np.empty((4,) + sx), np.empty((4,) + sx)
    c = p[1:-1, :, :]
    for m, (dj, dk) in enumerate(combos):
        q[m] = c[:, dj:dj + sx[1], dk:dk + sx[2]]
        wy = (ylo if dj == 0 else yhi)[None, :, None]
        wz = (zlo if dk == 0 else zhi)[None, None, :]
        w[m] = np.broadcast_to(wy * wz, sx)
    out.append(_combine(q, w, mode))
    sy = g.shape_edges[1]
    q, w = np.empty((4,) + sy), np.empty((4,) + sy)
    c = p[:, 1:-1, :]
    for m, (di, dk) in enumerate(combos):
        q[m] = c[di:di + sy[0], :, dk:dk + sy[2]]
        wx = (xlo if di == 0 else xhi)[:, None, None]
        wz = (zlo if dk == 0 else zhi)[None, None, :]
        w[m] = np.broadcast_to(wx * wz, sy)
    out.append(_combine(q, w, mode))
    sz = g.shape_edges[2]
    q, w = np.empty((4,) + sz), np.empty((4,) + sz)
    c = p[:, :, 1:-1]
    for m, (di, dj) in enumerate(combos):
        q[m] = c[di:di + sz[0], dj:dj + sz[1], :]
        wx = (xlo if di == 0 else xhi)[:, None, None]
        wy = (ylo if dj == 0 else yhi)[None, :, None]
        w[m] = np.broadcast_to(wx * wy, sz)
    out.append(_combine(q, w, mode))
    return np.concatenate([o.ravel() for o in out])


def edge_mass_vector(g: Grid, prop_edge):
    """``prop * A_dual / L`` per edge (operators.py:302-315)."""
    prop_edge = np.asarray(prop_edge, dtype=float).ravel()
    Lv = np.concatenate([a.ravel() for a in g.edge_lengths()])
    A = np.concatenate([a.ravel() for a in g.edge_dual_areas()])
    return prop_edge * A / Lv


def nodal_laplacian(g: Grid, mass_edge):
    """``G^T diag(m) G`` (operators.py:340-351)."""
    G = grad_node_edge(g)
    return sp.csr_matrix(G.T @ sp.diags(mass_edge, format="dia") @ G)


def padded_masses(g: Grid, mass_edge):
    """Edge vector -> three node-shaped arrays (0 on the last plane)."""
    nx, ny, nz = g.shape_nodes
    sx, sy, sz = g.shape_edges
    n1, n2 = int(np.prod(sx)), int(np.prod(sy))
    out = np.zeros((3, nx, ny, nz))
    out[0, :-1] = mass_edge[:n1].reshape(sx)
    out[1, :, :-1] = mass_edge[n1:n1 + n2].reshape(sy)
    out[2, :, :, :-1] = mass_edge[n1 + n2:].reshape(sz)
    return out.reshape(3, -1)


def apply_dirichlet(A, b, fixed, values):
    """Symmetric elimination (operators.py:362-407)."""
    A = sp.csr_matrix(A, copy=True)
    b = np.array(b, dtype=float, copy=True)
    n = A.shape[0]
    fixed = np.asarray(fixed)
    idx = np.flatnonzero(fixed) if fixed.dtype == bool else fixed.astype(np.intp)
    vals = np.broadcast_to(np.asarray(values, dtype=float), idx.shape)
    x0 = np.zeros(n)
    x0[idx] = vals
    b -= A @ x0
    mask = np.ones(n, dtype=bool)
    mask[idx] = False
    Dm = sp.diags(mask.astype(float))
    A = Dm @ A @ Dm
    A = A + sp.diags((~mask).astype(float))
    b[idx] = vals
    return sp.csr_matrix(A), b


# ---------------------------------------------------------------------------
# Walls -- fieldspice/boundaries.py:154-198, :963-1029
# ---------------------------------------------------------------------------
_AXIS = {"xlo": 0, "xhi": 0, "ylo": 1, "yhi": 1, "zlo": 2, "zhi": 2}
WALLS = ("xlo", "xhi", "ylo", "yhi", "zlo", "zhi")


def wall_nodes(g: Grid, wall: str):
    shape = g.shape_nodes
    strides = (shape[1] * shape[2], shape[2], 1)
    axis = _AXIS[wall]
    plane = 0 if wall.endswith("lo") else shape[axis] - 1
    d0, d1 = [d for d in (0, 1, 2) if d != axis]
    a = np.arange(shape[d0], dtype=np.intp) * strides[d0]
    b = np.arange(shape[d1], dtype=np.intp) * strides[d1]
    return (plane * strides[axis] + a[:, None] + b[None, :]).ravel()


def dirichlet_nodes(g: Grid, walls: dict[str, float]):
    """``walls``: {wall: value} of Dirichlet walls; later wall wins."""
    idx_parts, val_parts = [], []
    for w in WALLS:
        if w not in walls:
            continue
        idx = wall_nodes(g, w)
        idx_parts.append(idx)
        val_parts.append(np.full(idx.size, float(walls[w])))
    if not idx_parts:
        return np.empty(0, np.intp), np.empty(0)
    ia, va = np.concatenate(idx_parts), np.concatenate(val_parts)
    u, first = np.unique(ia[::-1], return_index=True)
    return u.astype(np.intp), va[::-1][first]


def unique_last(idx, val):
    # poisson.py:722-727
    if idx.size == 0:
        return idx.astype(np.intp), val.astype(float)
    u, first = np.unique(idx[::-1], return_index=True)
    return u.astype(np.intp), val[::-1][first]


# ---------------------------------------------------------------------------
# LinearSystem restated for the SPD eliminated system -- poisson.py:260-589
# ---------------------------------------------------------------------------
class LinearSystemCPU:
    """Prepared eliminated system: solo split, equilibration, CG or LU.

    Follows poisson.py:336-381 (decoupled rows split off, symmetric Jacobi
    equilibration) and :487-589 (solve, un-scale, true residual).  ``method``
    is "cg" (SciPy CG with the Jacobi preconditioner the reference falls back
    to when its incomplete LU is unavailable, :477-484) or "direct" (SuperLU,
    :457).  The default CG+ILU branch is not restated: it stalls on these
    systems.
    """

    def __init__(self, A, method="cg", tol=1e-10, maxiter=None):
        A = sp.csr_matrix(A)
        self.n = A.shape[0]
        self.tol = tol
        # empty rows (a zero-conductivity region no terminal reaches) are
        # pinned to zero with an identity row, poisson.py:286-325,600-611
        row_abs = np.asarray(abs(A).sum(axis=1)).ravel()
        self.empty = np.flatnonzero(row_abs == 0.0)
        if self.empty.size:
            keep = np.ones(self.n)
            keep[self.empty] = 0.0
            A = sp.csr_matrix(sp.diags(keep) @ A @ sp.diags(keep) + sp.diags(1.0 - keep))
            row_abs = np.asarray(abs(A).sum(axis=1)).ravel()
        d = A.diagonal()
        solo = (row_abs <= np.abs(d)) & (d != 0)
        self.solo = np.flatnonzero(solo)
        self.free = np.flatnonzero(~solo)
        self.solo_diag = d[self.solo]
        self.split = bool(self.solo.size) and self.free.size > 0
        if self.split:
            A = sp.csr_matrix(A[self.free][:, self.free])
        dreal = A.diagonal()
        self.dhalf = np.sqrt(dreal)
        self.dinv = 1.0 / self.dhalf
        S = sp.diags(self.dinv)
        self.A = sp.csr_matrix(S @ A @ S)
        self.n_free = self.A.shape[0]
        self.method = method
        self.maxiter = maxiter
        if method == "direct":
            self.lu = spla.splu(self.A.tocsc(), permc_spec="MMD_AT_PLUS_A")
        else:
            dd = self.A.diagonal()
            dd = np.where(np.abs(dd) > 0, dd, 1.0)
            self.M = spla.LinearOperator(self.A.shape, lambda v: v / dd,
                                         dtype=self.A.dtype)
        self.info = {}

    def solve(self, b, x0=None):
        b = np.asarray(b, dtype=float).copy()
        b[self.empty] = 0.0
        bf = b[self.free] if self.split else b
        bs = bf * self.dinv
        iters = 0
        if self.method == "direct":
            xs = self.lu.solve(bs)
        else:
            maxiter = self.maxiter or max(500, int(10 * np.sqrt(self.n_free)))
            counter = {"n": 0}

            def cb(_):
                counter["n"] += 1
            kw = {"rtol": self.tol, "atol": 0.0, "maxiter": maxiter, "M": self.M,
                  "callback": cb}
            if x0 is not None:
                g0 = np.asarray(x0, float)
                if self.split:
                    g0 = g0[self.free]
                kw["x0"] = g0 * self.dhalf
            xs, flag = spla.cg(self.A, bs, **kw)
            iters = counter["n"]
            if flag != 0:
                warnings.warn(f"cg flag {flag} after {iters} iterations",
                              RuntimeWarning, stacklevel=2)
        xf = xs * self.dinv
        if self.split:
            x = np.zeros(self.n)
            x[self.free] = xf
            x[self.solo] = b[self.solo] / self.solo_diag
        else:
            x = xf
        rs = bs - self.A @ xs
        nb = float(np.linalg.norm(bs))
        self.info = {"iterations": iters,
                     "relres": float(np.linalg.norm(rs) / nb) if nb > 0 else 0.0}
        return x


# ---------------------------------------------------------------------------
# Capacitance extraction -- poisson.py:1100-1249
# ---------------------------------------------------------------------------
def capacitance_matrix(g: Grid, eps_cell, terminals, dirichlet_walls=None,
                       method="cg", tol=1e-10, symmetrise=True, mode="parallel",
                       charge="csr"):
    """Maxwell C by unit excitation; returns (C, report).

    ``charge="csr"`` integrates ``L @ phi`` with the assembled matrix, as the
    reference (poisson.py:1219-1224); ``charge="edges"`` evaluates the same
    ``G^T (m * G phi)`` edge by edge, which avoids the cancellation of the
    CSR diagonal against its off-diagonals on electrodes that carry very
    large masses (a copper conductor inside an electrode: ``d ~ 1e8`` and the
    round-off of ``d - sum m`` reaches the charge at ~1e-8).

    ``terminals``: list of node-index arrays.  ``dirichlet_walls``: {wall:
    value} (values are ignored, every Dirichlet wall is a grounded shield).
    """
    m = edge_mass_vector(g, cell_to_edge(g, eps_cell, mode))
    Lmat = nodal_laplacian(g, m)
    wall_idx, _ = dirichlet_nodes(g, dirichlet_walls or {})
    terms = [np.unique(np.asarray(t, np.intp)) for t in terminals]
    term_nodes = np.concatenate(terms)
    fixed = np.concatenate([wall_idx, term_nodes]).astype(np.intp)
    fixed, _ = unique_last(fixed, np.zeros(fixed.size))
    shield = np.setdiff1d(wall_idx, term_nodes)
    A_bc, _ = apply_dirichlet(Lmat, np.zeros(g.n_nodes), fixed, np.zeros(fixed.size))
    ls = LinearSystemCPU(A_bc, method=method, tol=tol)
    nt = len(terms)
    C = np.zeros((nt, nt))
    q_shield = np.zeros(nt)
    iters, relres, phis = [], [], []
    for j, tj in enumerate(terms):
        x0 = np.zeros(g.n_nodes)
        x0[tj] = 1.0
        b = -(Lmat @ x0)
        b[fixed] = x0[fixed]
        phi = ls.solve(b)
        phis.append(phi)
        iters.append(ls.info["iterations"])
        relres.append(ls.info["relres"])
        if charge == "edges":
            Gm = grad_node_edge(g)
            q = Gm.T @ (m * (Gm @ phi))
        else:
            q = Lmat @ phi
        for i, ti in enumerate(terms):
            C[i, j] = float(q[ti].sum())
        if shield.size:
            q_shield[j] = float(q[shield].sum())
    scale = float(np.abs(np.diag(C)).max()) or 1.0
    rep = {"asymmetry_abs": float(np.abs(C - C.T).max())}
    rep["asymmetry_rel"] = rep["asymmetry_abs"] / scale
    if symmetrise:
        C = 0.5 * (C + C.T)
    rows = C.sum(axis=1)
    rep["row_sum"] = rows
    rep["row_sum_rel"] = float(np.abs(rows).max() / scale)
    off = C - np.diag(np.diag(C))
    rep["max_offdiag"] = float(off.max()) if nt > 1 else 0.0
    rep["shield_charge"] = q_shield
    rep["iterations"] = iters
    rep["relres"] = relres
    rep["phis"] = phis
    return C, rep


# ---------------------------------------------------------------------------
# EQS backward Euler / theta -- fieldspice/solvers/eqs.py:97-101, :176-195,
# :229-323, :328-340
# ---------------------------------------------------------------------------
def resistance_matrix(g: Grid, sigma_cell, terminals, method="cg", tol=1e-10,
                      mode="parallel"):
    """DC resistance matrix [ohm] (``fieldspice/extraction.py:59-87``).

    Unit excitation of every terminal with all terminal nodes fixed and every
    wall insulating; ``Y[i, j] = sum_{n in T_i} (L_sigma phi_j)_n``,
    symmetrised, then the pseudo-inverse (``Y`` is singular: the all-ones
    vector drives no current).  Returns ``(R, Y_unsymmetrised)``.
    """
    terms = [np.unique(np.asarray(t, np.intp)) for t in terminals]
    if len(terms) < 2:
        raise ValueError("resistance extraction needs at least two terminals")
    m = edge_mass_vector(g, cell_to_edge(g, np.asarray(sigma_cell, float), mode))
    Lmat = nodal_laplacian(g, m)
    fixed = np.concatenate(terms)
    nt = len(terms)
    Y = np.zeros((nt, nt))
    A_bc, _ = apply_dirichlet(Lmat, np.zeros(g.n_nodes), fixed, np.zeros(fixed.size))
    ls = LinearSystemCPU(A_bc, method=method, tol=tol)
    for j, tj in enumerate(terms):
        x0 = np.zeros(g.n_nodes)
        x0[tj] = 1.0
        b = -(Lmat @ x0)
        b[fixed] = x0[fixed]
        phi = ls.solve(b)
        q = Lmat @ phi
        for i, ti in enumerate(terms):
            Y[i, j] = float(q[ti].sum())
    Ys = 0.5 * (Y + Y.T)
    return np.linalg.pinv(Ys), Y


# ---------------------------------------------------------------------------
# Heat conduction -- solvers/thermal.py:104-300
# ---------------------------------------------------------------------------
def node_volumes(g: Grid):
    """Dual (box) volumes, flat C order (grid.py:388-396)."""
    return (g.hxd[:, None, None] * g.hyd[None, :, None] * g.hzd[None, None, :]).ravel()


def cell_to_node(g: Grid, prop):
    """Dual-volume-weighted average of a cell property onto nodes, cells
    edge-padded (operators.py:270-296)."""
    prop = np.asarray(prop, dtype=float)
    p = np.pad(prop, 1, mode="edge")
    nx, ny, nz = g.shape_nodes
    acc = np.zeros((nx, ny, nz))
    wacc = np.zeros((nx, ny, nz))
    halves = [(np.concatenate([[0.0], 0.5 * h]), np.concatenate([0.5 * h, [0.0]]))
              for h in (g.hx, g.hy, g.hz)]
    for di in (0, 1):
        for dj in (0, 1):
            for dk in (0, 1):
                q = p[di:di + nx, dj:dj + ny, dk:dk + nz]
                w = (halves[0][di][:, None, None] * halves[1][dj][None, :, None]
                     * halves[2][dk][None, None, :])
                acc += q * w
                wacc += w
    return acc / np.where(wacc > 0, wacc, 1.0)


def wall_dual_areas(g: Grid, wall: str):
    """Dual face area of every node on a wall, ordered as wall_nodes
    (boundaries.py:200-218)."""
    axis = {"x": 0, "y": 1, "z": 2}[wall[0]]
    duals = (g.hxd, g.hyd, g.hzd)
    d0, d1 = [d for d in (0, 1, 2) if d != axis]
    return (duals[d0][:, None] * duals[d1][None, :]).ravel()


def _thermal_walls(g: Grid, convection):
    diag = np.zeros(g.n_nodes)
    rhs = np.zeros(g.n_nodes)
    for wall, (h, t_inf) in (convection or {}).items():
        nodes = wall_nodes(g, wall)
        area = wall_dual_areas(g, wall)
        diag[nodes] += float(h) * area
        rhs[nodes] += float(h) * area * float(t_inf)
    return diag, rhs


def thermal_steady(g: Grid, kappa_cell, q_node, dirichlet=None, convection=None,
                   method="cg", tol=1e-10):
    """Steady temperature: (K + diag(h A)) T = q + h A T_inf, fixed-temperature
    walls eliminated (thermal.py:200-245)."""
    K = nodal_laplacian(g, edge_mass_vector(g, cell_to_edge(g, kappa_cell)))
    diag, rhs = _thermal_walls(g, convection)
    A = sp.csr_matrix(K + sp.diags(diag))
    b = np.broadcast_to(np.asarray(q_node, float), (g.n_nodes,)).copy() + rhs
    idx, val = dirichlet_nodes(g, dirichlet or {})
    if idx.size:
        A, b = apply_dirichlet(A, b, idx, val)
    return LinearSystemCPU(A, method=method, tol=tol).solve(b)


def thermal_transient(g: Grid, kappa_cell, rho_cp_cell, q_node, t_end, dt, T0,
                      dirichlet=None, convection=None, theta=1.0, method="cg", tol=1e-10):
    """theta-scheme transient (thermal.py:247-300): (C/dt + theta K) T+ =
    (C/dt - (1 - theta) K) T + q + h A T_inf.  Returns the list of T."""
    K = nodal_laplacian(g, edge_mass_vector(g, cell_to_edge(g, kappa_cell)))
    diag, wall_rhs = _thermal_walls(g, convection)
    Kc = sp.csr_matrix(K + sp.diags(diag))
    C = cell_to_node(g, rho_cp_cell).ravel() * node_volumes(g)
    A_imp = sp.csr_matrix(sp.diags(C / dt) + theta * Kc)
    A_exp = sp.csr_matrix(sp.diags(C / dt) - (1.0 - theta) * Kc)
    n = int(np.ceil(t_end / dt))
    T = np.full(g.n_nodes, float(T0)) if np.isscalar(T0) else np.asarray(T0, float).copy()
    q = np.broadcast_to(np.asarray(q_node, float), (g.n_nodes,))
    idx, val = dirichlet_nodes(g, dirichlet or {})
    A, _ = apply_dirichlet(A_imp, np.zeros(g.n_nodes), idx, val) if idx.size else (A_imp, None)
    ls = LinearSystemCPU(A, method=method, tol=tol)
    out = [T.copy()]
    for _ in range(n):
        b = A_exp @ T + q + wall_rhs
        if idx.size:
            _, b = apply_dirichlet(A_imp, b, idx, val)
        T = ls.solve(b)
        out.append(T.copy())
    return out


def eqs_transient(g: Grid, eps_cell, sigma_cell, fixed_groups, values_at,
                  dt, nsteps, theta=1.0, method="cg", tol=1e-10,
                  dirichlet_walls=None, t_start=0.0):
    """Backward-Euler EQS with terminal currents.

    ``fixed_groups``: list of node arrays (voltage-driven terminals);
    ``values_at(t)``: their voltages at time t.  Dirichlet walls (values
    fixed) come first, terminals after (eqs.py:108-129: a terminal listed
    later wins).  Returns (phis, currents[nsteps+1, nterm]).
    """
    me = edge_mass_vector(g, cell_to_edge(g, eps_cell))
    ms = edge_mass_vector(g, cell_to_edge(g, sigma_cell))
    Le = nodal_laplacian(g, me)
    Ls = nodal_laplacian(g, ms)
    walls = dirichlet_walls or {}

    def dirichlet(t):
        idx, val = [], []
        vt = values_at(t)
        for grp, v in zip(fixed_groups, vt):
            idx.append(np.asarray(grp, np.intp))
            val.append(np.full(len(grp), float(v)))
        widx, wval = dirichlet_nodes(g, walls)
        if widx.size:
            idx.append(widx)
            val.append(wval)
        fixed = np.concatenate(idx)
        vals = np.concatenate(val)
        u, last = np.unique(fixed[::-1], return_index=True)
        return u, vals[::-1][last]

    # consistent initial condition (eqs.py:176-195)
    fixed, vals = dirichlet(t_start)
    A0, b0 = apply_dirichlet(Le, np.zeros(g.n_nodes), fixed, vals)
    phi = LinearSystemCPU(A0, method=method, tol=tol).solve(b0)
    K = (Le / dt + theta * Ls).tocsr()
    Kexp = (Le / dt - (1.0 - theta) * Ls).tocsr()
    ls = None
    phis = [phi.copy()]
    for k in range(1, nsteps + 1):
        t = t_start + dt * k
        fixed, vals = dirichlet(t)
        rhs = Kexp @ phi
        A, b = apply_dirichlet(K, rhs, fixed, vals)
        if ls is None:
            ls = LinearSystemCPU(A, method=method, tol=tol)
        phi = ls.solve(b)
        phis.append(phi.copy())
    cur = np.zeros((nsteps + 1, len(fixed_groups)))
    for k in range(1, nsteps + 1):
        resid = (Le @ (phis[k] - phis[k - 1]) / dt
                 + Ls @ (theta * phis[k] + (1 - theta) * phis[k - 1]))
        for j, grp in enumerate(fixed_groups):
            cur[k, j] = float(resid[np.asarray(grp, np.intp)].sum())
    if nsteps >= 1:
        cur[0] = cur[1]
    return phis, cur


def laplacian_apply(g: Grid, mass_edge, x):
    """``L @ x`` with the assembled CSR (reference arithmetic)."""
    return nodal_laplacian(g, mass_edge) @ x


# ---------------------------------------------------------------------------
# Field region stamped into a netlist -- circuit/coupling.py:55-275
# ---------------------------------------------------------------------------
class FieldRegionCPU:
    """Exact reduction of a meshed EQS region to its electrodes.

    ``reduce(dt)`` follows coupling.py:140-181: ``K = L_eps/dt + L_sigma``
    (``L_sigma`` at dc), split by the electrode map ``P`` and interior
    selector ``S`` (:117-125); ``Y = K_tt - K_ti K_ii^-1 K_it``, measured
    asymmetry, then symmetrised; an all-zero ``K`` gives ``Y = 0`` (:156-167).
    ``history(dt)`` is ``f_eff = P f - K_ti K_ii^-1 S f`` with ``f = (L_eps/dt)
    phi`` (:183-193); ``accept(v, dt)`` back-substitutes the interior
    ``u = K_ii^-1 (f_i - K_it v)`` with the electrodes at ``v`` (:248-262).
    ``terminals``: node-index arrays, one per electrode.
    """

    def __init__(self, g: Grid, eps_cell, sigma_cell, terminals, method="direct",
                 tol=1e-12, mode="parallel"):
        self.g = g
        eps_cell = np.asarray(eps_cell, float)
        sigma_cell = np.asarray(sigma_cell, float)
        self.L_eps = nodal_laplacian(g, edge_mass_vector(g, cell_to_edge(g, eps_cell, mode)))
        self.L_sig = nodal_laplacian(g, edge_mass_vector(g, cell_to_edge(g, sigma_cell, mode)))
        elec = [np.asarray(t, np.intp).ravel() for t in terminals]
        flat = np.concatenate(elec)
        if np.unique(flat).size != flat.size:
            raise ValueError("terminals overlap: a node belongs to two electrodes")
        n = g.n_nodes
        self.interior = np.setdiff1d(np.arange(n), flat)
        rows = np.concatenate([np.full(e.size, k) for k, e in enumerate(elec)])
        self.P = sp.csr_matrix((np.ones(flat.size), (rows, flat)), shape=(len(elec), n))
        self.S = sp.csr_matrix((np.ones(self.interior.size),
                                (np.arange(self.interior.size), self.interior)),
                               shape=(self.interior.size, n))
        self.elec = elec
        self.method, self.tol = method, tol
        self.cache: dict = {}
        self.phi = np.zeros(n)
        self.asymmetry = 0.0

    def reduce(self, dt):
        key = 0.0 if dt is None else float(dt)
        if key in self.cache:
            return self.cache[key]
        K = (self.L_sig if dt is None else self.L_eps / dt + self.L_sig).tocsr()
        P, S = self.P, self.S
        K_tt = (P @ K @ P.T).toarray()
        K_ti = (P @ K @ S.T).tocsr()
        K_ii = (S @ K @ S.T).tocsr()
        if K.nnz == 0 or float(abs(K).max()) == 0.0:
            entry = {"Y": np.zeros_like(K_tt), "solver": None, "K_ti": K_ti}
            self.asymmetry = 0.0
            self.cache[key] = entry
            return entry
        if K_ii.shape[0] == 0:
            Y, solver = K_tt, None
        else:
            solver = LinearSystemCPU(K_ii, method=self.method, tol=self.tol)
            K_it = K_ti.T.tocsc()
            W = np.column_stack([solver.solve(np.asarray(K_it[:, j].todense()).ravel())
                                 for j in range(K_it.shape[1])])
            Y = K_tt - K_ti @ W
        self.asymmetry = float(np.abs(Y - Y.T).max() / max(np.abs(Y).max(), 1e-300))
        entry = {"Y": 0.5 * (Y + Y.T), "solver": solver, "K_ti": K_ti}
        self.cache[key] = entry
        return entry

    def history(self, dt):
        if dt is None:
            return np.zeros(len(self.elec))
        entry = self.reduce(dt)
        f = (self.L_eps / dt) @ self.phi
        f_t = self.P @ f
        if entry["solver"] is None:
            return f_t
        return f_t - entry["K_ti"] @ entry["solver"].solve(self.S @ f)

    def accept(self, v, dt):
        entry = self.reduce(dt)
        v = np.asarray(v, float)
        phi = np.zeros(self.g.n_nodes)
        for k, e in enumerate(self.elec):
            phi[e] = v[k]
        if entry["solver"] is not None and dt is not None:
            f_i = self.S @ ((self.L_eps / dt) @ self.phi)
            phi[self.interior] = entry["solver"].solve(f_i - entry["K_ti"].T @ v)
        self.phi = phi


# ---------------------------------------------------------------------------
# Per-unit-length line parameters -- extraction.py:108-206
# ---------------------------------------------------------------------------
def rlgc_2d_matrices(g: Grid, eps_cell, sigma_cell, terminals, reference=-1,
                     method="direct", tol=1e-12, charge="csr"):
    """``C``, ``C_air``, ``G`` and ``L`` of a 2-D cross-section referenced to
    conductor ``reference`` (an index), as ``extraction.py:168-199``: three
    capacitance extractions (real permittivity, vacuum, conductivity floored
    at 1e-30) with every wall insulating, the reference row and column
    removed, and ``L = mu0 eps0 C_air^-1``."""
    nt = len(terminals)
    ref_i = int(reference) % nt
    keep = [i for i in range(nt) if i != ref_i]
    eps_cell = np.asarray(eps_cell, float)
    sigma_cell = np.asarray(sigma_cell, float)
    mu0 = 4e-7 * math.pi * 1.0000000000552

    def cap(prop):
        C, _ = capacitance_matrix(g, prop, terminals, method=method, tol=tol, charge=charge)
        return C[np.ix_(keep, keep)]
    C = cap(eps_cell)
    C_air = cap(np.full_like(eps_cell, EPS0))
    G = cap(np.maximum(sigma_cell, 1e-30)) if np.any(sigma_cell > 0) else np.zeros_like(C)
    return {"C": C, "C_air": C_air, "G": G, "L": mu0 * EPS0 * np.linalg.inv(C_air)}


# ---------------------------------------------------------------------------
# Harmonic EQS -- solvers/ac.py:34-181
# ---------------------------------------------------------------------------
def ac_system(g: Grid, eps_cell, sigma_cell, freq):
    """``K = L_sigma + j w (L_eps' + j L_eps'')`` as complex CSR (ac.py:79-95)."""
    eps = np.asarray(eps_cell)
    L_sig = nodal_laplacian(g, edge_mass_vector(g, cell_to_edge(g, np.asarray(sigma_cell, float))))
    L_eps = nodal_laplacian(g, edge_mass_vector(g, cell_to_edge(g, np.real(eps).astype(float))))
    L_eps = L_eps.astype(complex)
    if np.iscomplexobj(eps) and np.any(np.imag(eps) != 0.0):
        L_eps = L_eps + 1j * nodal_laplacian(
            g, edge_mass_vector(g, cell_to_edge(g, np.imag(eps).astype(float))))
    w = 2.0 * np.pi * float(freq)
    return sp.csr_matrix(L_sig.astype(complex) + 1j * w * L_eps)


def ac_potential(K, n, fixed, values):
    """Complex Dirichlet elimination and sparse LU (ac.py:166-181, :143)."""
    idx = np.asarray(fixed, np.intp)
    vals = np.asarray(values, complex)
    x0 = np.zeros(n, complex)
    x0[idx] = vals
    b = -(K @ x0)
    mask = np.ones(n, bool)
    mask[idx] = False
    Dm = sp.diags(mask.astype(float))
    A = sp.csr_matrix(Dm @ K @ Dm + sp.diags((~mask).astype(float)))
    b[idx] = vals
    return spla.spsolve(A.tocsc(), b)


def ac_admittance(g: Grid, eps_cell, sigma_cell, terminals, freqs):
    """``Y[k, i, j]`` by unit excitation (ac.py:123-148)."""
    terms = [np.asarray(t, np.intp) for t in terminals]
    fixed = np.concatenate(terms)
    nt = len(terms)
    freqs = np.atleast_1d(np.asarray(freqs, float))
    Y = np.zeros((freqs.size, nt, nt), complex)
    for k, f in enumerate(freqs):
        K = ac_system(g, eps_cell, sigma_cell, f)
        for j in range(nt):
            vals = np.concatenate([np.full(t.size, 1.0 if m == j else 0.0)
                                   for m, t in enumerate(terms)])
            cur = K @ ac_potential(K, g.n_nodes, fixed, vals)
            for i, t in enumerate(terms):
                Y[k, i, j] = cur[t].sum()
    return Y


def ac_schur(g: Grid, eps_cell, sigma_cell, terminals, omega):
    """The field region's frequency-domain stamp ``Y_eff = K_tt - K_ti
    K_ii^-1 K_it`` with ``K = L_sigma + j w L_eps`` (coupling.py:214-236),
    by unit excitation (the same matrix)."""
    return ac_admittance(g, eps_cell, sigma_cell, terminals, [omega / (2.0 * np.pi)])[0]


# ---------------------------------------------------------------------------
# Floating / charge-driven electrodes -- poisson.py:665-719, 1030-1063
# ---------------------------------------------------------------------------
def merged_potential(g: Grid, eps_cell, fixed, values, merge_groups, b_ext, mode="parallel"):
    """``phi = P x`` with every node set in ``merge_groups`` merged into one
    unknown (``P`` has one 1 per row), ``P^T L P x = P^T b`` with the Dirichlet
    rows eliminated and a direct solve (poisson.py:665-719, 1041-1058).
    ``b_ext``: node charges (free charge, a charge-driven electrode's charge
    on its first node).  Fixed nodes must not belong to a merged group.
    Returns ``(phi, L)``."""
    n = g.n_nodes
    Lm = nodal_laplacian(g, edge_mass_vector(g, cell_to_edge(g, np.asarray(eps_cell, float), mode)))
    label = np.arange(n)
    for grp in merge_groups:
        grp = np.asarray(grp, np.intp)
        label[grp] = grp[0]
    uniq, red = np.unique(label, return_inverse=True)
    P = sp.csr_matrix((np.ones(n), (np.arange(n), red)), shape=(n, uniq.size))
    A = sp.csr_matrix(P.T @ Lm @ P)
    b = P.T @ np.asarray(b_ext, float)
    fixed_r = red[np.asarray(fixed, np.intp)]
    A_bc, b_bc = apply_dirichlet(A, b, fixed_r, np.asarray(values, float))
    x = spla.spsolve(A_bc.tocsc(), b_bc)
    return P @ x, Lm


# ---------------------------------------------------------------------------
# Periodic walls -- boundaries.py:226-260 (pairs), poisson.py:665-719 (merge),
# 942-955, 1041-1058 (solve), 1196-1224 (capacitance)
# ---------------------------------------------------------------------------
def periodic_groups(g: Grid, axes):
    """The (lo, hi) node pairs identified by the periodic ``axes`` ("x", "y",
    "z"), one two-node group per pair."""
    shape = g.shape_nodes
    nid = np.arange(g.n_nodes).reshape(shape)
    groups = []
    for a in axes:
        ax = "xyz".index(a)
        lo = np.take(nid, 0, axis=ax).ravel()
        hi = np.take(nid, shape[ax] - 1, axis=ax).ravel()
        groups.extend(np.array([p, q]) for p, q in zip(lo, hi))
    return groups


def _merge_matrix(n, groups):
    """``P`` (n x n_reduced, one 1 per row) merging connected node groups."""
    a = [np.full(len(gp) - 1, gp[0]) for gp in groups if len(gp) > 1]
    b = [np.asarray(gp[1:]) for gp in groups if len(gp) > 1]
    if not a:
        return sp.identity(n, format="csr"), np.arange(n)
    from scipy.sparse.csgraph import connected_components
    adj = sp.coo_matrix((np.ones(sum(x.size for x in a)), (np.concatenate(a), np.concatenate(b))),
                        shape=(n, n))
    _, label = connected_components(adj, directed=False)
    P = sp.coo_matrix((np.ones(n), (np.arange(n), label)), shape=(n, label.max() + 1)).tocsr()
    return P, label


def periodic_capacitance(g: Grid, eps_cell, terminals, axes, dirichlet_walls=None):
    """Maxwell C with periodic ``axes``: unit excitations solved on ``P^T L P``
    (direct), charges ``L phi`` on the full grid (poisson.py:1196-1224);
    unsymmetrised."""
    Lm = nodal_laplacian(g, edge_mass_vector(g, cell_to_edge(g, np.asarray(eps_cell, float))))
    P, red = _merge_matrix(g.n_nodes, periodic_groups(g, axes))
    A_r = sp.csr_matrix(P.T @ Lm @ P)
    wall_idx, _ = dirichlet_nodes(g, dirichlet_walls or {})
    terms = [np.asarray(t, np.intp) for t in terminals]
    fixed = np.unique(np.concatenate([wall_idx] + terms))
    fixed_r = red[fixed]
    A_bc, _ = apply_dirichlet(A_r, np.zeros(A_r.shape[0]), fixed_r, np.zeros(fixed_r.size))
    lu = spla.splu(A_bc.tocsc())
    C = np.zeros((len(terms), len(terms)))
    for j, tj in enumerate(terms):
        x0 = np.zeros(A_r.shape[0])
        x0[red[tj]] = 1.0
        b = -(A_r @ x0)
        b[fixed_r] = x0[fixed_r]
        q = Lm @ (P @ lu.solve(b))
        for i, ti in enumerate(terms):
            C[i, j] = q[ti].sum()
    return C


def periodic_potential(g: Grid, eps_cell, fixed, values, axes, b_free):
    """Potential with periodic ``axes``, Dirichlet ``fixed``/``values`` and
    node charges ``b_free`` (poisson.py:1041-1058, direct solve); returns
    ``(phi, L)`` on the full grid."""
    Lm = nodal_laplacian(g, edge_mass_vector(g, cell_to_edge(g, np.asarray(eps_cell, float))))
    P, red = _merge_matrix(g.n_nodes, periodic_groups(g, axes))
    A_r = sp.csr_matrix(P.T @ Lm @ P)
    A_bc, b_bc = apply_dirichlet(A_r, P.T @ np.asarray(b_free, float), red[np.asarray(fixed)],
                                 np.asarray(values, float))
    return P @ spla.spsolve(A_bc.tocsc(), b_bc), Lm
