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


def test_nonblocking_solve_equals_blocking_solve(cuda):
    """fs_pcg_plan_solve_begin / _poll: the same iterates, stats and status
    as fs_pcg_plan_solve on the same plan and inputs (bit-identical phi), with
    poll returning at once while the plan runs; a second begin while one is
    in flight and a poll of an idle plan are refused."""
    import ctypes

    import torch

    from fieldspice_b200 import _lib as L
    from fieldspice_b200.device import DeviceOperator, EliminatedSystem
    ws, probs = _batch(1, seed=3)
    grid, eps, terms, _ = probs[0]
    op = DeviceOperator(grid, eps)
    label = torch.zeros(op.N, dtype=torch.uint8, device=op.dev)
    nid = np.arange(op.N).reshape(grid.shape_nodes)
    label[torch.as_tensor(nid[:, :, 0].ravel(), device=op.dev)] = L.LABEL_FIXED
    k = len(terms)
    for t in terms:
        label[torch.as_tensor(np.asarray(t.nodes), device=op.dev)] = L.LABEL_FIXED
    system = EliminatedSystem(op, label, k, precision="mixed", preconditioner="mg")
    phi0 = torch.zeros_like(system.phi)
    view = phi0.view(op.N, system.k)
    for c, t in enumerate(terms):
        view[torch.as_tensor(np.asarray(t.nodes), device=op.dev), c] = 1.0
    # (terminal columns past the last terminal stay 0: padded RHS)
    lib = L.lib()
    system.phi.copy_(phi0)
    st_b = (L.FsRhsStats * system.k)()
    s_blocking = lib.fs_pcg_plan_solve(system.plan, 0, 1e-10, 0, st_b, L.stream_ptr())
    phi_b = system.phi.clone()
    system.phi.copy_(phi0)
    torch.cuda.synchronize()
    done = ctypes.c_int()
    assert lib.fs_pcg_plan_solve_poll(system.plan, None, ctypes.byref(done)) == L.FS_BAD_ARG
    st_a = (L.FsRhsStats * system.k)()
    L.check("begin", lib.fs_pcg_plan_solve_begin(system.plan, 0, 1e-10, 0, L.stream_ptr()))
    assert lib.fs_pcg_plan_solve_begin(system.plan, 0, 1e-10, 0, L.stream_ptr()) == L.FS_BAD_ARG
    polls = 0
    while True:
        s_async = lib.fs_pcg_plan_solve_poll(system.plan, st_a, ctypes.byref(done))
        polls += 1
        if done.value:
            break
        assert s_async == L.FS_OK
        assert polls < 10_000_000
    torch.cuda.synchronize()
    assert s_async == s_blocking == L.FS_OK
    assert polls > 2
    for a, b in zip(st_a, st_b):
        assert (a.iterations, a.status, a.reliable_updates) == (b.iterations, b.status,
                                                               b.reliable_updates)
        assert a.relres == b.relres
    assert torch.equal(system.phi, phi_b)
    system.close()
