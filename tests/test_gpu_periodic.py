"""Periodic walls on the GPU path (needs a B200).

The reference merges the two node planes of a periodic axis into one unknown
(``P^T L P``, ``poisson.py:665-719``); here the solve runs on the wrap-around
grid (the last plane of each periodic axis merged into the first, a wrap edge
joining them) with Jacobi PCG, and the charges are integrated on the full
grid as the reference does.  Recorded reference runs:
``tests/golden/periodic.npz`` (periodic in x, and in x and y; a grounded
floor; three electrodes, one crossing the x wrap; free charge in the solve).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(d):
    from fieldspice_b200.grid import RectilinearGrid
    from fieldspice_b200.solvers.base import Terminal
    g = RectilinearGrid(d["x"], d["y"], d["z"])
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    terms = [Terminal(f"b{i}", nid[a0:a1 + 1, b0:b1 + 1, c0:c1 + 1].ravel())
             for i, (a0, b0, c0, a1, b1, c1) in enumerate(d["boxes"])]
    terms.append(Terminal("wrap", d["wrap_nodes"]))
    return g, terms


def _bc(axes):
    from fieldspice_b200.boundaries import BoundarySpec, Dirichlet, Periodic
    kw = {"zlo": Dirichlet(0.0)}
    for a in axes:
        kw[f"{a}lo"] = Periodic()
        kw[f"{a}hi"] = Periodic()
    return BoundarySpec(**kw)


@pytest.mark.parametrize("precision", ["mixed", "fp64"])
@pytest.mark.parametrize("tag,axes", [("x", ("x",)), ("xy", ("x", "y"))])
def test_periodic_capacitance_and_potential_match_reference(cuda, golden, tag, axes,
                                                              precision):
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig, Terminal
    from fieldspice_b200.solvers.poisson import PoissonSolver
    d = golden("periodic")
    g, terms = _setup(d)
    ps = PoissonSolver(g, d["eps"], SolverConfig(tol=1e-12), gpu=GPUConfig(precision=precision))
    C = ps.capacitance_matrix(terms, _bc(axes))
    want = d[f"C_{tag}"]
    assert np.abs(C - want).max() <= 1e-9 * np.abs(np.diag(want)).max()
    drive = [Terminal(t.name, t.nodes, voltage=v) for t, v in zip(terms, (1.0, -0.5, 0.25))]
    r = ps.solve(drive, _bc(axes), rho_node=d["rho"])
    assert np.abs(r.fields["phi"][0].ravel() - d[f"phi_{tag}"]).max() <= 1e-9
    q = np.array([r.terminals[t.name]["q"][0] for t in drive])
    assert np.abs(q - d[f"q_{tag}"]).max() <= 1e-8 * np.abs(d[f"q_{tag}"]).max()
    # the merged planes carry one potential
    phi = r.fields["phi"][0]
    assert np.array_equal(phi[0], phi[-1])
    if "y" in axes:
        assert np.array_equal(phi[:, 0], phi[:, -1])


def test_periodic_rejections(cuda, golden):
    from fieldspice_b200.boundaries import BoundarySpec, Periodic
    from fieldspice_b200.solvers.base import Terminal
    from fieldspice_b200.solvers.poisson import PoissonSolver
    d = golden("periodic")
    g, terms = _setup(d)
    ps = PoissonSolver(g, d["eps"])
    with pytest.raises(ValueError, match="both walls"):
        ps.capacitance_matrix(terms, BoundarySpec(xlo=Periodic()))
    with pytest.raises(ValueError, match="offset"):
        ps.capacitance_matrix(terms, BoundarySpec(xlo=Periodic(offset=0.1),
                                                  xhi=Periodic(offset=0.1)))
    with pytest.raises(NotImplementedError, match="floating"):
        ps.solve([Terminal("f", terms[0].nodes)] + terms[1:2], _bc(("x",)))


@pytest.mark.parametrize("axes", [("x",), ("x", "y")])
def test_periodic_multigrid_matches_oracle(cuda, axes):
    """Multigrid on wrapping node aggregates: the Galerkin coarse levels keep
    each periodic axis periodic (the last aggregate's crossing to aggregate 0
    is a coarse wrap edge).  Same C as the oracle's direct solve on
    ``P^T L P``, in a quarter of the Jacobi iterations."""
    import oracle.fs_oracle as O
    from fieldspice_b200 import workloads as W
    from fieldspice_b200.grid import RectilinearGrid
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig, Terminal
    from fieldspice_b200.solvers.poisson import PoissonSolver
    w = W.layered_boxes((41, 29, 18), nbox=3, seed=5)
    g = RectilinearGrid(w.x, w.y, w.z)
    terms = [Terminal(n, t) for n, t in zip(w.names, w.terminals)]
    want = O.periodic_capacitance(O.Grid(w.x, w.y, w.z), w.eps_cell, w.terminals, axes,
                                  {"zlo": 0.0})
    want = 0.5 * (want + want.T)
    its = {}
    for pre in ("mg", "jacobi"):
        rep = {}
        C = PoissonSolver(g, w.eps_cell, SolverConfig(tol=1e-12),
                          gpu=GPUConfig(precision="fp64", preconditioner=pre)
                          ).capacitance_matrix(terms, _bc(axes), report=rep)
        assert np.abs(C - want).max() <= 1e-9 * np.abs(np.diag(want)).max(), pre
        its[pre] = max(rep["linear"]["iterations"])
        if pre == "mg":
            assert rep["linear"]["coarsening"] == "galerkin"
    assert its["mg"] * 4 <= its["jacobi"], its
