"""Reference results at scale: the 64-geometry batch and the EQS transient.

Runs the reference fieldspice package (imported from ``$FIELDSPICE_REF``,
which must be set) with its Jacobi branch of ``LinearSystem`` forced and
``SolverConfig(linear_solver="cg", tol=1e-12)``:

* ``batch``: every geometry of ``workloads.batch_geometries(64, seed=0)``
  (32^3 .. 160x160x96 nodes, 2-16 conductor boxes, zlo grounded) through
  ``PoissonSolver.capacitance_matrix`` (``poisson.py:1100-1249``, what
  ``extraction.capacitance_matrix`` calls, ``extraction.py:41-56``).  One process per geometry, largest first.
  Writes ``batch64_s0.json`` (C per geometry, iterations, seconds).
* ``eqs``: the copper / oxide / doped-silicon interconnect of
  ``workloads.eqs_interconnect(shape, nbox=6, nports=2, seed=0)``, port 0
  driven by a 1 V ramp (10 ps rise), port 1 at 0 V, zlo at 0 V,
  dt = 1 ps, backward Euler, 200 steps, through ``EQSSolver.solve``
  (``eqs.py:229-323``); the port currents come from the reference's own
  ``_record_terminals`` (``eqs.py:360-375``).  Writes
  ``eqs_<nx>x<ny>x<nz>_s0.npz``.  The reference cold-starts CG at every
  step, so the cost grows with the grid as nodes x iterations; 96x96x48
  takes about 40 minutes on one core here.

Usage::

    FIELDSPICE_REF=/path/to/fieldspice python tests/golden/make_scale.py batch
    FIELDSPICE_REF=/path/to/fieldspice python tests/golden/make_scale.py eqs 96,96,48

Only tests read the outputs: the GPU path never imports the reference.
"""

from __future__ import annotations

import contextlib
import json
import multiprocessing as mp
import os
import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))


def _import_reference():
    ref = os.environ.get("FIELDSPICE_REF")
    if not ref:
        raise SystemExit("set FIELDSPICE_REF to the reference fieldspice source tree")
    if ref not in sys.path:
        sys.path.insert(0, ref)


@contextlib.contextmanager
def jacobi_forced():
    """Make ``spilu`` raise so ``LinearSystem`` takes its Jacobi-CG branch
    (``poisson.py:472-484``); the incomplete-LU branch stalls here."""
    import scipy.sparse.linalg as spla
    orig = spla.spilu

    def _raise(*a, **k):
        raise MemoryError("incomplete LU disabled: Jacobi branch forced")
    spla.spilu = _raise
    try:
        yield
    finally:
        spla.spilu = orig


def _batch_one(i):
    _import_reference()
    from threadpoolctl import threadpool_limits
    from fieldspice.boundaries import BoundarySpec, Dirichlet
    from fieldspice.grid import RectilinearGrid
    from fieldspice.solvers.poisson import PoissonSolver
    from fieldspice.solvers.base import SolverConfig, Terminal
    from fieldspice_b200 import workloads as W
    w = W.batch_geometries(64, seed=0)[i]
    g = RectilinearGrid(w.x, w.y, w.z)
    terms = [Terminal(n, t) for n, t in zip(w.names, w.terminals)]
    rep = {}
    t0 = time.perf_counter()
    with threadpool_limits(limits=1), jacobi_forced():
        # extraction.capacitance_matrix is this call (extraction.py:54-56);
        # the solver object is made here to keep its report
        ps = PoissonSolver(g, w.eps_cell, SolverConfig(linear_solver="cg", tol=1e-12))
        C = ps.capacitance_matrix(terms, BoundarySpec(zlo=Dirichlet(0.0)), report=rep)
    lin = rep.get("linear", {})
    return {"index": i, "name": w.name, "shape": list(w.shape_nodes),
            "nterm": len(terms), "C": np.asarray(C).tolist(),
            "asymmetry_rel": float(rep.get("asymmetry_rel", float("nan"))),
            "iterations": lin.get("iterations"),
            "seconds": time.perf_counter() - t0}


def batch(procs=8):
    from fieldspice_b200 import workloads as W
    ws = W.batch_geometries(64, seed=0)
    order = sorted(range(len(ws)), key=lambda i: -np.prod(ws[i].shape_nodes) * len(ws[i].terminals))
    out = {"workload": "batch_geometries(64, seed=0), zlo grounded",
           "solver": "reference extraction.capacitance_matrix, Jacobi-forced CG, tol 1e-12",
           "geometries": [None] * len(ws)}
    t0 = time.perf_counter()
    ctx = mp.get_context("spawn")
    with ctx.Pool(procs) as pool:
        for r in pool.imap_unordered(_batch_one, order):
            out["geometries"][r["index"]] = r
            print(f"geometry {r['index']} {r['shape']} k={r['nterm']} "
                  f"{r['seconds']:.1f} s", flush=True)
    out["seconds"] = time.perf_counter() - t0
    out["host"] = f"{procs} single-threaded processes"
    (HERE / "batch64_s0.json").write_text(json.dumps(out))


def eqs(shape, steps=200):
    _import_reference()
    from threadpoolctl import threadpool_limits
    from fieldspice.boundaries import BoundarySpec, Dirichlet
    from fieldspice.grid import RectilinearGrid
    from fieldspice.solvers.base import SolverConfig, Terminal
    from fieldspice.solvers.eqs import EQSSolver
    from fieldspice_b200 import workloads as W
    w = W.eqs_interconnect(shape, nbox=6, nports=2, seed=0)
    g = RectilinearGrid(w.x, w.y, w.z)
    ramp = W.ramp(0.0, 0.0, 1.0, 10e-12)
    terms = [Terminal("port0", w.terminals[0], voltage=ramp),
             Terminal("port1", w.terminals[1], voltage=0.0)]
    t0 = time.perf_counter()
    with threadpool_limits(limits=1), jacobi_forced():
        s = EQSSolver(g, w.eps_cell, w.sigma_cell, SolverConfig(linear_solver="cg", tol=1e-12))
        r = s.solve(terms, t_end=steps * 1e-12, dt=1e-12, bc=BoundarySpec(zlo=Dirichlet(0.0)))
    tag = f"eqs_{shape[0]}x{shape[1]}x{shape[2]}_s0"
    np.savez_compressed(HERE / f"{tag}.npz", shape=np.asarray(shape), steps=steps, dt=1e-12,
                        t=np.asarray(r.t), i0=np.asarray(r.i("port0")),
                        i1=np.asarray(r.i("port1")), v0=np.asarray(r.v("port0")),
                        energy=np.asarray(r.scalars["energy_electric"]),
                        dissipation=np.asarray(r.scalars["dissipation"]),
                        seconds=time.perf_counter() - t0)
    print(f"{tag}: {time.perf_counter() - t0:.1f} s", flush=True)


if __name__ == "__main__":
    what = sys.argv[1] if len(sys.argv) > 1 else "batch"
    if what == "batch":
        batch(int(sys.argv[2]) if len(sys.argv) > 2 else 8)
    elif what == "eqs":
        eqs(tuple(int(v) for v in sys.argv[2].split(",")))
    else:
        raise SystemExit("usage: make_scale.py batch [procs] | eqs nx,ny,nz")
