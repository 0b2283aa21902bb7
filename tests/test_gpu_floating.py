"""Floating and charge-driven electrodes in ``PoissonSolver.solve`` (needs a B200).

The reference merges each such electrode into one unknown (``poisson.py:665-719``);
the GPU path solves the same problem by superposition of Dirichlet solves (one
block) and a small capacitance system.  Recorded reference run:
``tests/golden/floating.npz`` (a driven electrode, a floating conductor, a
charge-driven conductor, a grounded floor and a point of free charge).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("preconditioner", ["mg", "jacobi"])
def test_floating_and_charge_driven_match_reference(cuda, golden, preconditioner):
    from fieldspice_b200.boundaries import BoundarySpec, Dirichlet
    from fieldspice_b200.grid import RectilinearGrid
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig, Terminal
    from fieldspice_b200.solvers.poisson import PoissonSolver
    d = golden("floating")
    g = RectilinearGrid(d["x"], d["y"], d["z"])
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    nodes = [nid[a0:a1 + 1, b0:b1 + 1, c0:c1 + 1].ravel() for a0, b0, c0, a1, b1, c1 in d["boxes"]]
    terms = [Terminal("drv", nodes[0], voltage=1.0), Terminal("flt", nodes[1]),
             Terminal("chg", nodes[2], current=2e-17)]
    ps = PoissonSolver(g, d["eps"], SolverConfig(tol=1e-12),
                       gpu=GPUConfig(preconditioner=preconditioner))
    r = ps.solve(terms, BoundarySpec(zlo=Dirichlet(0.0)), rho_node=d["rho"])
    phi = r.fields["phi"][0].ravel()
    assert np.abs(phi - d["phi"]).max() <= 1e-9
    qscale = abs(float(d["q_drv"][0]))
    for t in terms:
        assert abs(r.terminals[t.name]["v"][0] - d[f"v_{t.name}"][0]) <= 1e-9
        assert abs(r.terminals[t.name]["q"][0] - d[f"q_{t.name}"][0]) <= 1e-8 * qscale
    # the floating conductor is an equipotential carrying no net charge
    assert np.ptp(phi[nodes[1]]) == 0.0
    assert abs(r.terminals["flt"]["q"][0]) <= 1e-8 * qscale


def test_floating_without_reference_raises(cuda):
    from fieldspice_b200.grid import RectilinearGrid
    from fieldspice_b200.solvers.base import Terminal
    from fieldspice_b200.solvers.poisson import PoissonSolver
    g = RectilinearGrid.uniform([(0, 1e-6), (0, 1e-6), (0, 1e-6)], [6, 6, 6])
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    ps = PoissonSolver(g, np.full(g.shape_cells, 3.9 * 8.854e-12))
    with pytest.raises(NotImplementedError, match="reference"):
        ps.solve([Terminal("f", nid[2:4, 2:4, 2:4].ravel())])


@pytest.mark.parametrize("preconditioner", ["mg", "jacobi"])
def test_twenty_floating_electrodes_match_reference(cuda, golden, preconditioner):
    """20 floating and charge-driven conductors and a driven electrode
    (``tests/golden/floating_many.npz``): 21 columns, more than one block of
    right-hand sides (8 per block in mixed precision), solved block after
    block on one system."""
    from fieldspice_b200.boundaries import BoundarySpec, Dirichlet
    from fieldspice_b200.grid import RectilinearGrid
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig, Terminal
    from fieldspice_b200.solvers.poisson import PoissonSolver
    d = golden("floating_many")
    g = RectilinearGrid(d["x"], d["y"], d["z"])
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    nodes = [nid[a0:a1 + 1, b0:b1 + 1, c0:c1 + 1].ravel() for a0, b0, c0, a1, b1, c1 in d["boxes"]]
    terms = [Terminal("drv", nodes[0], voltage=1.0)]
    for i, nd in enumerate(nodes[1:]):
        terms.append(Terminal(f"c{i}", nd, current=1e-18 * (i - 9)) if i % 3 == 2
                     else Terminal(f"f{i}", nd))
    assert [t.name for t in terms] == list(d["names"])
    ps = PoissonSolver(g, d["eps"], SolverConfig(tol=1e-12),
                       gpu=GPUConfig(preconditioner=preconditioner))
    r = ps.solve(terms, BoundarySpec(zlo=Dirichlet(0.0)))
    assert r.meta["linear"]["blocks"] == 3  # 21 columns in blocks of 7
    phi = r.fields["phi"][0].ravel()
    assert np.abs(phi - d["phi"]).max() <= 1e-9
    qscale = abs(float(d["q"][0]))
    for i, t in enumerate(terms):
        assert abs(r.terminals[t.name]["v"][0] - d["v"][i]) <= 1e-9, t.name
        assert abs(r.terminals[t.name]["q"][0] - d["q"][i]) <= 1e-8 * qscale, t.name
