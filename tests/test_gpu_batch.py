"""Batched extraction of uneven geometries (needs a B200).

A seeded batch of the uneven-geometry family (2-16 terminals, eps_r drawn
from {2.5, 3.9, 7.0, 11.7}, log-uniform node counts) at sizes the oracle
factorises in seconds: every C matrix must match the oracle to 1e-9 of its
largest diagonal entry (relres 1e-10), and equal the one-at-a-time GPU path.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _batch(count=6, seed=1):
    from fieldspice_b200 import workloads as W
    from fieldspice_b200.boundaries import BoundarySpec, Dirichlet
    from fieldspice_b200.solvers.base import Terminal
    ws = W.batch_geometries(count, seed=seed, lo=(24, 24, 20), hi=(44, 44, 28))
    bc = BoundarySpec(zlo=Dirichlet(0.0))
    probs = [(w.grid(), w.eps_cell, [Terminal(n, t) for n, t in zip(w.names, w.terminals)], bc)
             for w in ws]
    return ws, probs


@pytest.mark.parametrize("preconditioner", ["mg", "jacobi"])
def test_batch_matches_oracle_and_single_path(cuda, preconditioner):
    from oracle import fs_oracle as O
    from fieldspice_b200 import extraction as EX
    from fieldspice_b200.batch import capacitance_matrices
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig
    ws, probs = _batch()
    cfg = SolverConfig(tol=1e-10)
    gcfg = GPUConfig(preconditioner=preconditioner)
    reps = [None] * len(probs)
    Cs = capacitance_matrices(probs, cfg, gpu=gcfg, streams=4, reports=reps)
    assert len(Cs) == len(probs)
    for w, (grid, eps, terms, bc), C, rep in zip(ws, probs, Cs, reps):
        g = O.Grid(grid.xn, grid.yn, grid.zn)
        Cref, _ = O.capacitance_matrix(g, eps, [t.nodes for t in terms], {"zlo": 0.0},
                                       method="direct")
        scale = np.abs(np.diag(Cref)).max()
        assert C.shape == (len(terms), len(terms))
        assert np.abs(C - Cref).max() / scale <= 1e-9, w.name
        assert max(rep["linear"]["relres_fp64"]) < 1e-10
        C1 = EX.capacitance_matrix(grid, eps, terms, bc, cfg, gpu=gcfg)
        assert np.abs(C - C1).max() / scale <= 1e-12


def test_batch_rejects_bad_geometry_before_solving(cuda):
    from fieldspice_b200.batch import capacitance_matrices
    _, probs = _batch(2)
    grid, eps, terms, bc = probs[1]
    with pytest.raises(ValueError, match="RELATIVE"):
        capacitance_matrices([probs[0], (grid, eps / 8.8541878128e-12, terms, bc)])


def test_batch64_matches_reference_at_scale(cuda):
    """The 64-geometry batch (32^3 .. 160x160x96 nodes, 2-16 terminals) with
    the default path (mixed precision, multigrid, relres 1e-10): every C
    matrix against the reference's own extraction of the same geometry
    (Jacobi-CG forced, tol 1e-12; tests/golden/batch64_s0.json, made by
    tests/golden/make_scale.py) to 1e-9 of its largest diagonal entry."""
    import json
    from pathlib import Path

    from fieldspice_b200 import workloads as W
    from fieldspice_b200.batch import capacitance_matrices
    from fieldspice_b200.boundaries import BoundarySpec, Dirichlet
    from fieldspice_b200.solvers.base import SolverConfig, Terminal
    ref = json.loads((Path(__file__).parent / "golden" / "batch64_s0.json").read_text())
    ws = W.batch_geometries(64, seed=0)
    bc = BoundarySpec(zlo=Dirichlet(0.0))
    probs = [(w.grid(), w.eps_cell, [Terminal(n, t) for n, t in zip(w.names, w.terminals)], bc)
             for w in ws]
    reps = [None] * len(probs)
    Cs = capacitance_matrices(probs, SolverConfig(tol=1e-10), reports=reps)
    errs = []
    for w, C, r, rep in zip(ws, Cs, ref["geometries"], reps):
        assert r["shape"] == list(w.shape_nodes) and r["nterm"] == len(w.terminals)
        Cref = np.asarray(r["C"])
        errs.append(float(np.abs(C - Cref).max() / np.abs(np.diag(Cref)).max()))
        assert max(rep["linear"]["relres_fp64"]) < 1e-10
    assert max(errs) <= 1e-9, (int(np.argmax(errs)), max(errs))
