"""Multigrid on grids with short axes (needs a B200).

Axes of fewer than 5 nodes are kept while the others are halved: a 2-D
cross-section (two node planes, collapsed z) and a thin 3-D slab get a full
V-cycle instead of the single coarsest-level polynomial.  Checked against the
oracle's direct solve, plus an iteration bound that only a working hierarchy
meets.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _c_err(C, Cref):
    return float(np.abs(C - Cref).max() / np.abs(np.diag(Cref)).max())


def test_cross_section_capacitance_uses_semicoarsened_multigrid(cuda):
    from fieldspice_b200 import extraction as EX
    from fieldspice_b200 import workloads as W
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig, Terminal
    from oracle import fs_oracle as O
    w = W.cross_section(301, 201, nlines=2, seed=3)
    g = w.grid()
    terms = [Terminal(n, t) for n, t in zip(w.names, w.terminals)]
    rep = {}
    C = EX.capacitance_matrix(g, w.eps_cell, terms, config=SolverConfig(tol=1e-11),
                              report=rep, gpu=GPUConfig(preconditioner="mg"))
    Cref, _ = O.capacitance_matrix(O.Grid(w.x, w.y, w.z), w.eps_cell, w.terminals,
                                   method="direct")
    assert _c_err(C, Cref) <= 1e-9
    # the V-cycle reaches 1e-11 in a few tens of iterations on 121k nodes
    assert max(rep["linear"]["iterations"]) <= 60, rep["linear"]["iterations"]


def test_thin_slab_semicoarsening(cuda):
    from fieldspice_b200 import extraction as EX
    from fieldspice_b200 import workloads as W
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig, Terminal
    from oracle import fs_oracle as O
    w = W.layered_boxes((96, 96, 8), nbox=3, seed=2)
    g = w.grid()
    terms = [Terminal(n, t) for n, t in zip(w.names, w.terminals)]
    rep = {}
    C = EX.capacitance_matrix(g, w.eps_cell, terms, w.boundary_spec(),
                              SolverConfig(tol=1e-11), report=rep,
                              gpu=GPUConfig(preconditioner="mg"))
    Cref, _ = O.capacitance_matrix(O.Grid(w.x, w.y, w.z), w.eps_cell, w.terminals,
                                   w.dirichlet_walls, method="direct")
    assert _c_err(C, Cref) <= 1e-9
    assert max(rep["linear"]["iterations"]) <= 60, rep["linear"]["iterations"]


def test_plan_levels_keep_short_axes(cuda):
    """The hierarchy of a 2-D grid halves x and y and keeps the z planes."""
    import ctypes

    import torch

    from fieldspice_b200 import _lib as L
    from fieldspice_b200.device import DeviceOperator, EliminatedSystem
    from fieldspice_b200 import workloads as W
    w = W.cross_section(301, 201, nlines=1, seed=0)
    op = DeviceOperator(w.grid(), w.eps_cell)
    label = torch.zeros(op.N, dtype=torch.uint8, device=op.dev)
    label[torch.as_tensor(w.terminals[-1], device=op.dev)] = L.LABEL_FIXED
    sys_ = EliminatedSystem(op, label, 1, preconditioner="mg")
    nlev = ctypes.c_int()
    dims = (ctypes.c_int * 36)()
    L.check("levels", L.lib().fs_pcg_plan_levels(sys_.plan, ctypes.byref(nlev), dims))
    got = [tuple(dims[3 * l:3 * l + 3]) for l in range(nlev.value)]
    assert got[0] == (301, 201, 2)
    assert got[1] == (151, 101, 2)
    assert all(d[2] == 2 for d in got)
    assert got[-1][0] * got[-1][1] * 2 <= 4096
    sys_.close()
