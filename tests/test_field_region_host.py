"""Host-side checks of the GPU field region that need no device: the eager
argument validation of ``circuit/coupling.py:88-125`` runs before any upload."""

import numpy as np
import pytest


def _setup():
    from fieldspice_b200.grid import RectilinearGrid
    from fieldspice_b200.solvers.base import Terminal
    g = RectilinearGrid(np.linspace(0, 2e-6, 6), np.linspace(0, 5e-6, 4), np.linspace(0, 4e-6, 3))
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    terms = [Terminal("a", nid[0].ravel()), Terminal("b", nid[-1].ravel())]
    return g, terms


def test_overlapping_terminals_are_rejected():
    from fieldspice_b200.circuit import FieldRegion
    from fieldspice_b200.solvers.base import Terminal
    g, terms = _setup()
    bad = [terms[0], Terminal("dup", terms[0].nodes)]
    eps = np.full(g.shape_cells, 3.9e-11)
    with pytest.raises(ValueError, match="overlap"):
        FieldRegion("FR", g, eps, np.zeros(g.shape_cells), bad, circuit_nodes=["a", "b"])


def test_bad_arguments_are_rejected():
    from fieldspice_b200.circuit import FieldRegion
    g, terms = _setup()
    eps = np.full(g.shape_cells, 3.9e-11)
    sig = np.zeros(g.shape_cells)
    with pytest.raises(ValueError, match="at least one terminal"):
        FieldRegion("FR", g, eps, sig, [])
    with pytest.raises(ValueError, match="circuit_nodes"):
        FieldRegion("FR", g, eps, sig, terms, circuit_nodes=["a"])
    with pytest.raises(ValueError, match="shape"):
        FieldRegion("FR", g, eps[:-1], sig, terms)
    with pytest.raises(ValueError, match="shape"):
        FieldRegion("FR", g, eps, sig[:, :-1], terms)

