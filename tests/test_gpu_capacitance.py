"""GPU capacitance extraction against the reference's recorded results.

Tolerances (the reference's own, ``tests/test_core.py:236-311`` and
``tests/test_solvers.py:24-45``): the README capacitor to 1e-12 of eps*A/d;
the layered 8-terminal extractions to 1e-9 of max|diag C| against the
reference's FP64 Jacobi-CG at tol 1e-12; relres <= 1e-10 on every RHS.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PRECISIONS = ["mixed", "fp64", "auto"]


def _layered(d):
    from fieldspice_b200.grid import RectilinearGrid
    from fieldspice_b200.solvers.base import Terminal
    g = RectilinearGrid(d["x"], d["y"], d["z"])
    nid = np.arange(int(np.prod(g.shape_nodes))).reshape(g.shape_nodes)
    terms = [Terminal(f"box{i}", nid[a0:a1 + 1, b0:b1 + 1, c0:c1 + 1].ravel())
             for i, (a0, b0, c0, a1, b1, c1) in enumerate(d["boxes"])]
    return g, terms


@pytest.mark.parametrize("preconditioner", ["jacobi", "mg"])
@pytest.mark.parametrize("precision", PRECISIONS)
def test_readme_capacitor(cuda, golden, precision, preconditioner):
    from fieldspice_b200 import extraction as EX
    from fieldspice_b200 import workloads as W
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig, Terminal
    w = W.parallel_plate()
    terms = [Terminal("top", w.terminals[0], voltage=1.0),
             Terminal("bottom", w.terminals[1], voltage=0.0)]
    rep = {}
    C = EX.capacitance_matrix(w.grid(), w.eps_cell, terms,
                              config=SolverConfig(tol=1e-13), report=rep,
                              gpu=GPUConfig(precision=precision,
                                            preconditioner=preconditioner))
    assert C[0, 0] == pytest.approx(w.meta["C_ref"], rel=1e-12)
    assert np.allclose(C, golden("readme")["C"], rtol=1e-12, atol=0)
    assert rep["asymmetry_rel"] < 1e-9 and rep["row_sum_rel"] < 1e-9
    assert rep["linear"]["symmetric"] is True
    assert max(rep["linear"]["relres_fp64"]) < 1e-13


@pytest.mark.parametrize("preconditioner", ["jacobi", "mg"])
@pytest.mark.parametrize("precision", PRECISIONS)
@pytest.mark.parametrize("tag", ["layered_32x32x16_s0", "layered_48x48x24_s1"])
def test_layered_matches_reference(cuda, golden, tag, precision, preconditioner):
    from fieldspice_b200.boundaries import BoundarySpec, Dirichlet
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig
    from fieldspice_b200.solvers.poisson import PoissonSolver
    d = golden(tag)
    g, terms = _layered(d)
    ps = PoissonSolver(g, d["eps_cell"], SolverConfig(tol=1e-10),
                       gpu=GPUConfig(precision=precision, preconditioner=preconditioner))
    rep = {}
    C = ps.capacitance_matrix(terms, BoundarySpec(zlo=Dirichlet(0.0)), report=rep)
    ref = d["C"]
    scale = np.abs(np.diag(ref)).max()
    assert np.abs(C - ref).max() / scale <= 1e-9
    # the shield charge is a sum of cancelling surface terms: 1e-8
    assert np.abs(rep["shield_charge"] - d["shield"]).max() / scale <= 1e-8
    assert max(rep["linear"]["relres_fp64"]) < 1e-10
    assert rep["max_offdiag"] <= 0.0
    assert rep["asymmetry_rel"] < 1e-8


def test_multigrid_cuts_iterations(cuda, golden):
    """The multigrid V-cycle must pay for itself: >5x fewer iterations than
    Jacobi CG on the same system, same answer."""
    from fieldspice_b200.boundaries import BoundarySpec, Dirichlet
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig
    from fieldspice_b200.solvers.poisson import PoissonSolver
    d = golden("layered_48x48x24_s1")
    g, terms = _layered(d)
    its = {}
    for pc in ("jacobi", "mg"):
        ps = PoissonSolver(g, d["eps_cell"], SolverConfig(tol=1e-10),
                           gpu=GPUConfig(preconditioner=pc))
        rep = {}
        ps.capacitance_matrix(terms, BoundarySpec(zlo=Dirichlet(0.0)), report=rep)
        its[pc] = max(rep["linear"]["iterations"])
    assert its["mg"] * 5 < its["jacobi"], its


@pytest.mark.parametrize("params", [(3, 0.3, 24, 0.03, 512, -1), (1, 0.5, 8, 0.05, 64, 0),
                                    (2, 0.3, 32, 0.03, 4096, 2)])
def test_multigrid_parameters(cuda, golden, params):
    """Non-default smoothing degrees (the plain Chebyshev pre-smoothing path,
    not the degree-2 residual form), coarsest sizes and stencil kinds, given
    per solver, give the same C; a solver with the defaults created next to
    it is not affected (no process-wide setting)."""
    import ctypes

    import torch

    from fieldspice_b200 import _lib as L
    from fieldspice_b200.boundaries import BoundarySpec, Dirichlet
    from fieldspice_b200.device import DeviceOperator, EliminatedSystem
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig
    from fieldspice_b200.solvers.poisson import PoissonSolver
    d = golden("layered_48x48x24_s1")
    g, terms = _layered(d)
    names = ("smooth_deg", "smooth_lo", "coarse_deg", "coarse_lo", "coarsest_nodes",
             "stencil_kind")
    opts = dict(zip(names, params))
    ps = PoissonSolver(g, d["eps_cell"], SolverConfig(tol=1e-10),
                       gpu=GPUConfig(preconditioner="mg", mg_params=opts))
    rep = {}
    C = ps.capacitance_matrix(terms, BoundarySpec(zlo=Dirichlet(0.0)), report=rep)
    scale = np.abs(np.diag(d["C"])).max()
    assert np.abs(C - d["C"]).max() / scale <= 1e-9
    assert max(rep["linear"]["relres_fp64"]) < 1e-10
    assert max(rep["linear"]["iterations"]) < 100
    # two live plans, one with the options and one without: each keeps its own
    op = DeviceOperator(g, d["eps_cell"])
    label = torch.zeros(op.N, dtype=torch.uint8, device=op.dev)
    label[:g.shape_nodes[1] * g.shape_nodes[2]] = L.LABEL_FIXED
    a = EliminatedSystem(op, label, 8, precision="mixed", preconditioner="mg",
                         coarsening="geometric", mg_params=opts)
    b = EliminatedSystem(op, label, 8, precision="mixed", preconditioner="mg",
                         coarsening="geometric")
    coarsest = {}
    for name, s in (("opt", a), ("default", b)):
        n = ctypes.c_int()
        dims = (ctypes.c_int * 48)()
        L.check("levels", L.lib().fs_pcg_plan_levels(s.plan, ctypes.byref(n), dims))
        coarsest[name] = int(np.prod(dims[3 * (n.value - 1):3 * n.value]))
    assert coarsest["opt"] <= params[4]
    assert coarsest["default"] == 864  # 48x48x24 -> 24x24x12 -> 12x12x6
    if params[5] >= 0:
        assert L.lib().fs_pcg_plan_stencil_kind(a.plan) in (params[5], 1)
    a.close()
    b.close()


def test_many_terminals_and_padding(cuda):
    """19 terminals: one 16-RHS block plus a padded 4-RHS block; matches the
    oracle run on the same inputs."""
    from fieldspice_b200 import workloads as W
    from fieldspice_b200.boundaries import BoundarySpec, Dirichlet
    from fieldspice_b200.solvers.base import SolverConfig
    from fieldspice_b200.solvers.poisson import PoissonSolver
    from oracle import fs_oracle as O
    w = W.layered_boxes((40, 40, 24), nbox=19, seed=11, ext_xy=(8, 40), ext_z=(4, 10))
    ps = PoissonSolver(w.grid(), w.eps_cell, SolverConfig(tol=1e-11))
    C = ps.capacitance_matrix(w.terminal_objects(), BoundarySpec(zlo=Dirichlet(0.0)))
    Cref, _ = O.capacitance_matrix(O.Grid(w.x, w.y, w.z), w.eps_cell, w.terminals,
                                   {"zlo": 0.0}, method="cg", tol=1e-12)
    scale = np.abs(np.diag(Cref)).max()
    assert C.shape == (19, 19)
    assert np.abs(C - Cref).max() / scale <= 1e-9


def test_isolated_terminal_and_solo_nodes(cuda):
    """A terminal enclosed by a grounded shell has no free neighbour: its RHS
    is zero (SciPy returns x = 0), free nodes inside the shell are decoupled
    ("solo") rows solved directly, and its capacitance row is exact."""
    from fieldspice_b200.grid import RectilinearGrid
    from fieldspice_b200.solvers.base import Terminal
    from fieldspice_b200.solvers.poisson import PoissonSolver
    from oracle import fs_oracle as O
    g = RectilinearGrid.uniform([(0, 1e-6)] * 3, [10, 10, 10])
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    eps = np.full(g.shape_cells, 3.9 * O.EPS0)
    shell = np.setdiff1d(nid[1:8, 1:8, 1:8].ravel(), nid[2:7, 2:7, 2:7].ravel())
    center = nid[4, 4, 4]
    core = np.setdiff1d(nid[2:7, 2:7, 2:7].ravel(), [center])  # encloses one free node
    far = nid[8:10, 8:10, 8:10].ravel()
    terms = [Terminal("shell", shell), Terminal("core", core), Terminal("far", far)]
    ps = PoissonSolver(g, eps)
    rep = {}
    C = ps.capacitance_matrix(terms, report=rep)
    Cref, _ = O.capacitance_matrix(O.Grid(g.xn, g.yn, g.zn), eps,
                                   [shell, core, far], method="direct")
    scale = np.abs(np.diag(Cref)).max()
    assert np.abs(C - Cref).max() / scale <= 1e-9
    assert rep["linear"]["n_solo"] > 0


def test_all_neumann_solve_pins_and_warns(cuda):
    from fieldspice_b200.grid import RectilinearGrid
    from fieldspice_b200.solvers.poisson import PoissonSolver
    from oracle import fs_oracle as O
    g = RectilinearGrid.uniform([(0, 1e-6)] * 3, [6, 5, 4])
    ps = PoissonSolver(g, np.full(g.shape_cells, O.EPS0))
    rho = np.zeros(g.shape_nodes)
    rho[1, 1, 1], rho[4, 3, 2] = 1.0, -1.0
    with pytest.warns(RuntimeWarning, match="pinned"):
        res = ps.solve(rho_node=rho)
    phi = res.fields["phi"].ravel()
    q = ps.node_charge(phi)
    vn = g.node_volumes().ravel()
    assert np.abs(q - rho.ravel() * vn).max() <= 1e-8 * np.abs(rho.ravel() * vn).max()


def test_solve_potential_and_energy_match_reference(cuda, golden):
    from fieldspice_b200 import workloads as W
    from fieldspice_b200.solvers.base import SolverConfig, Terminal
    from fieldspice_b200.solvers.poisson import PoissonSolver
    d = golden("readme")
    w = W.parallel_plate()
    terms = [Terminal("top", w.terminals[0], voltage=1.0),
             Terminal("bottom", w.terminals[1], voltage=0.0)]
    ps = PoissonSolver(w.grid(), w.eps_cell, SolverConfig(tol=1e-13))
    res = ps.solve(terms)
    assert np.abs(res.fields["phi"].ravel() - d["phi"]).max() < 1e-12
    assert res.scalars["energy"][0] == pytest.approx(float(d["energy"][0]), rel=1e-11)
    assert res.terminals["top"]["q"][0] == pytest.approx(float(d["q_top"][0]), rel=1e-11)
    assert ps.energy(res.fields["phi"][0]) == pytest.approx(float(d["energy"][0]), rel=1e-11)


def test_maxiter_raises_convergence_error(cuda):
    from fieldspice_b200 import workloads as W
    from fieldspice_b200.boundaries import BoundarySpec, Dirichlet
    from fieldspice_b200.solvers.base import ConvergenceError, GPUConfig
    from fieldspice_b200.solvers.poisson import PoissonSolver
    w = W.layered_boxes((32, 32, 16), seed=0)
    ps = PoissonSolver(w.grid(), w.eps_cell, gpu=GPUConfig(maxiter=3))
    with pytest.raises(ConvergenceError):
        ps.capacitance_matrix(w.terminal_objects(), BoundarySpec(zlo=Dirichlet(0.0)))


def test_input_rejection(cuda):
    from fieldspice_b200.grid import RectilinearGrid
    from fieldspice_b200.solvers.base import Terminal
    from fieldspice_b200.solvers.poisson import PoissonSolver
    g = RectilinearGrid.uniform([(0, 1e-6)] * 3, [4, 4, 4])
    with pytest.raises(ValueError, match="RELATIVE"):
        PoissonSolver(g, np.full(g.shape_cells, 3.9))
    with pytest.raises(ValueError, match="positive"):
        PoissonSolver(g, np.full(g.shape_cells, -1e-11))
    ps = PoissonSolver(g, np.full(g.shape_cells, 1e-11))
    with pytest.raises(ValueError, match="at least one"):
        ps.capacitance_matrix([])
    with pytest.raises(ValueError, match="share node"):
        ps.capacitance_matrix([Terminal("a", [0, 1]), Terminal("b", [1, 2])])


def test_one_call_extraction_rejects_like_the_solver(cuda):
    """extraction.capacitance_matrix checks eps while the host checks the
    terminals: the same errors, a bad eps reported before bad terminals, and
    page-locked inputs give the same C as pageable ones."""
    import torch
    from fieldspice_b200 import extraction as EX
    from fieldspice_b200 import workloads as W
    from fieldspice_b200.boundaries import BoundarySpec, Dirichlet
    from fieldspice_b200.grid import RectilinearGrid
    from fieldspice_b200.solvers.base import Terminal
    g = RectilinearGrid.uniform([(0, 1e-6)] * 3, [4, 4, 4])
    good = [Terminal("a", [0, 1])]
    bad_terms = [Terminal("a", [0, 1]), Terminal("b", [1, 2])]
    nan = np.full(g.shape_cells, 1e-11)
    nan[1, 2, 0] = np.nan
    for eps, match in ((np.full(g.shape_cells, 3.9), "RELATIVE"),
                       (np.full(g.shape_cells, -1e-11), "positive"), (nan, "non-finite")):
        with pytest.raises(ValueError, match=match):
            EX.capacitance_matrix(g, eps, good)
        with pytest.raises(ValueError, match=match):
            EX.capacitance_matrix(g, eps, bad_terms)
    with pytest.raises(ValueError, match="share node"):
        EX.capacitance_matrix(g, np.full(g.shape_cells, 1e-11), bad_terms)
    w = W.layered_boxes((32, 32, 16), seed=2)
    bc = BoundarySpec(zlo=Dirichlet(0.0))
    C = EX.capacitance_matrix(w.grid(), w.eps_cell, w.terminal_objects(), bc)
    pinned = torch.from_numpy(np.ascontiguousarray(w.eps_cell)).pin_memory().numpy()
    C_p = EX.capacitance_matrix(w.grid(), pinned, w.terminal_objects(), bc)
    assert np.array_equal(C, C_p)


@pytest.mark.slow
def test_full_size_extraction_properties(cuda):
    """256x256x128 nodes, 8 terminals: size-independent properties of the
    exact answer (reciprocity, signs, grounded-shield balance) plus FP64 vs
    mixed-precision agreement to 1e-9."""
    from fieldspice_b200 import workloads as W
    from fieldspice_b200.boundaries import BoundarySpec, Dirichlet
    from fieldspice_b200.solvers.base import GPUConfig
    from fieldspice_b200.solvers.poisson import PoissonSolver
    w = W.layered_boxes()
    bc = BoundarySpec(zlo=Dirichlet(0.0))
    out = {}
    for prec in ("mixed", "fp64"):
        ps = PoissonSolver(w.grid(), w.eps_cell, gpu=GPUConfig(precision=prec))
        rep = {}
        C = ps.capacitance_matrix(w.terminal_objects(), bc, report=rep)
        out[prec] = (C, rep)
        scale = np.abs(np.diag(C)).max()
        assert np.all(np.diag(C) > 0)
        assert rep["max_offdiag"] <= 0.0
        assert rep["asymmetry_rel"] < 1e-8
        assert max(rep["linear"]["relres_fp64"]) < 1e-10
        # Gauss: every field line from terminal j ends on a terminal or on
        # the grounded plane, so column sums balance the shield charge.
        bal = np.abs(C.sum(axis=0) + rep["shield_charge"]).max()
        assert bal <= 1e-7 * scale
    Cm, Cf = out["mixed"][0], out["fp64"][0]
    assert np.abs(Cm - Cf).max() / np.abs(np.diag(Cf)).max() <= 1e-9
