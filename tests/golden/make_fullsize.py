"""Full-size oracle run of the 256x256x128, 8-terminal extraction.

Runs the CPU oracle's Jacobi-preconditioned CG (SciPy's algorithm on the
equilibrated system, restated as an explicit loop so the residual history is
visible) to relres 1e-12 on every right-hand side, one process per RHS, and
records into ``layered_256x256x128_s0.json``:

* the iteration count at which relres first fell below 1e-10 (the
  reference's default tolerance) and 1e-12,
* the 8x8 capacitance matrix at relres 1e-12 (full-size golden result),
* the seconds per CG iteration on this host.

Usage: ``python tests/golden/make_fullsize.py`` (about 10-20 minutes).
"""

from __future__ import annotations

import json
import multiprocessing as mp
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

from oracle import fs_oracle as O  # noqa: E402

_STATE = {}


def _setup(shape, seed):
    from fieldspice_b200 import workloads as W
    w = W.layered_boxes(shape, nbox=8, seed=seed)
    g = O.Grid(w.x, w.y, w.z)
    m = O.edge_mass_vector(g, O.cell_to_edge(g, w.eps_cell))
    Lm = O.nodal_laplacian(g, m)
    wall = O.wall_nodes(g, "zlo")
    terms = [np.asarray(t, np.intp) for t in w.terminals]
    fixed = np.unique(np.concatenate([wall] + terms))
    A, _ = O.apply_dirichlet(Lm, np.zeros(g.n_nodes), fixed, 0.0)
    d = A.diagonal()
    import scipy.sparse as sp
    row_abs = np.asarray(abs(A).sum(axis=1)).ravel()
    solo = (row_abs <= np.abs(d)) & (d != 0)
    free = np.flatnonzero(~solo)
    Af = sp.csr_matrix(A[free][:, free])
    s = 1.0 / np.sqrt(Af.diagonal())
    Aeq = sp.csr_matrix(sp.diags(s) @ Af @ sp.diags(s))
    _STATE.update(Lm=Lm, A=A, Aeq=Aeq, s=s, free=free, solo=np.flatnonzero(solo),
                  fixed=fixed, terms=terms, n=g.n_nodes, wall=wall)


def _solve(j, tol=1e-12, tol_report=1e-10):
    Lm, A, Aeq, s, free = (_STATE[k] for k in ("Lm", "A", "Aeq", "s", "free"))
    terms, fixed, n = _STATE["terms"], _STATE["fixed"], _STATE["n"]
    x0 = np.zeros(n)
    x0[terms[j]] = 1.0
    b = -(Lm @ x0)
    b[fixed] = x0[fixed]
    bs = b[free] * s
    dd = Aeq.diagonal()
    # SciPy's cg loop (rtol=tol, atol=0, M=Jacobi), restated
    x = np.zeros_like(bs)
    r = bs.copy()
    bn = np.linalg.norm(bs)
    it_report = -1
    rho_prev = None
    p = None
    t0 = time.perf_counter()
    it = 0
    maxiter = max(500, int(10 * np.sqrt(bs.size)))
    while it < maxiter:
        rn = np.linalg.norm(r)
        if it_report < 0 and rn < tol_report * bn:
            it_report = it
        if rn < tol * bn:
            break
        z = r / dd
        rho = r @ z
        if it > 0:
            p *= rho / rho_prev
            p += z
        else:
            p = z.copy()
        q = Aeq @ p
        alpha = rho / (p @ q)
        x += alpha * p
        r -= alpha * q
        rho_prev = rho
        it += 1
    t_iter = (time.perf_counter() - t0) / max(it, 1)
    phi = x0.copy()
    phi[free] = x * s
    solo = _STATE["solo"]
    phi[solo] = b[solo] / A.diagonal()[solo]
    qn = Lm @ phi
    col = [float(qn[t].sum()) for t in terms]
    shield = float(qn[np.setdiff1d(_STATE["wall"], np.concatenate(terms))].sum())
    return j, it_report, it, t_iter, col, shield


def main(shape=(256, 256, 128), seed=0):
    t0 = time.perf_counter()
    _setup(shape, seed)
    t_setup = time.perf_counter() - t0
    ctx = mp.get_context("fork")  # CPU only: nothing here touches a GPU
    with ctx.Pool(8) as pool:
        res = pool.map(_solve, range(8))
    C = np.zeros((8, 8))
    out = {"shape": list(shape), "seed": seed, "setup_seconds": t_setup,
           "iterations_1e-10": [], "iterations_1e-12": [], "seconds_per_iteration": [],
           "shield_charge": []}
    for j, itr, it, ti, col, sh in sorted(res):
        C[:, j] = col
        out["iterations_1e-10"].append(itr)
        out["iterations_1e-12"].append(it)
        out["seconds_per_iteration"].append(ti)
        out["shield_charge"].append(sh)
    out["C_tol1e-12_unsymmetrised"] = C.tolist()
    out["host"] = "8-core Xeon, 8 concurrent single-threaded processes"
    tag = f"layered_{shape[0]}x{shape[1]}x{shape[2]}_s{seed}"
    (HERE / f"{tag}.json").write_text(json.dumps(out, indent=1))
    print(json.dumps({k: v for k, v in out.items() if not k.startswith("C_")}))


if __name__ == "__main__":
    main()
