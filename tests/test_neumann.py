"""Driven Neumann walls: the flux load and the potential it drives.

``tests/golden/neumann.npz`` was recorded from the reference
(``tests/golden/make_golden.py neumann``): a constant D.n on the xhi wall, a
time-dependent one on yhi, a grounded floor and one driven box, direct
solve.  The load vector (``BoundarySpec.neumann_load``,
``boundaries.py:1031-1085``) is host arithmetic and must agree to the last
bit; the GPU potential (``poisson.py:957-964``: the load joins the free
charge) to 1e-9 of its largest value.
"""

import numpy as np
import pytest


def _case(golden):
    from fieldspice_b200.boundaries import BoundarySpec, Dirichlet, Neumann
    from fieldspice_b200.grid import RectilinearGrid
    from fieldspice_b200.solvers.base import Terminal
    d = golden("neumann")
    g = RectilinearGrid(d["x"], d["y"], d["z"])

    def ramp_flux(t):
        return 2e-4 * (1.0 + t * 1e9)
    bc = BoundarySpec(zlo=Dirichlet(0.0), xhi=Neumann(flux=-3e-4), yhi=Neumann(flux=ramp_flux))
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    box = Terminal("box", nid[4:8, 3:6, 4:6].ravel(), voltage=0.7)
    return d, g, bc, box


def test_neumann_load_matches_reference(golden):
    from fieldspice_b200.boundaries import BoundarySpec, neumann_load
    d, g, bc, _ = _case(golden)
    load = neumann_load(bc, g, float(d["t"]))
    assert np.array_equal(load, d["load"])
    assert neumann_load(BoundarySpec(), g) is None


@pytest.mark.gpu
def test_driven_neumann_potential_matches_reference(cuda, golden):
    from fieldspice_b200.solvers.base import SolverConfig
    from fieldspice_b200.solvers.poisson import PoissonSolver
    d, g, bc, box = _case(golden)
    r = PoissonSolver(g, d["eps"], SolverConfig(tol=1e-12)).solve([box], bc, t=float(d["t"]))
    phi = r.fields["phi"][0].ravel()
    assert np.abs(phi - d["phi"]).max() <= 1e-9 * np.abs(d["phi"]).max()
    assert r.terminals["box"]["q"][0] == pytest.approx(float(d["q_box"][0]), rel=1e-8)
    assert r.scalars["energy"][0] == pytest.approx(float(d["energy"][0]), rel=1e-9)
