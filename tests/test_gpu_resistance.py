"""GPU resistance extraction against the reference (needs a B200).

``extraction.resistance_matrix`` (``extraction.py:59-87``) on a seeded
copper-on-silicon network with insulating regions, recorded from the
reference in ``tests/golden/resistance.npz``.  NumPy's pseudo-inverse keeps
the all-ones direction of ``Y``, which is null only to round-off, so the
comparison is on ``P R P`` (``P = I - 11^T/n``): the resistance differences.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _projected(R):
    n = R.shape[0]
    P = np.eye(n) - np.ones((n, n)) / n
    return P @ R @ P


@pytest.mark.parametrize("preconditioner", ["jacobi", "mg"])
@pytest.mark.parametrize("precision", ["auto", "fp64"])
def test_resistance_matrix_matches_reference(cuda, golden, precision, preconditioner):
    from fieldspice_b200 import extraction as EX
    from fieldspice_b200.grid import RectilinearGrid
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig, Terminal
    d = golden("resistance")
    g = RectilinearGrid(d["x"], d["y"], d["z"])
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    terms = [Terminal(f"t{i}", nid[a0:a1 + 1, b0:b1 + 1, c0:c1 + 1].ravel())
             for i, (a0, b0, c0, a1, b1, c1) in enumerate(d["boxes"])]
    rep = {}
    with pytest.warns(RuntimeWarning, match="coupled to nothing"):
        R = EX.resistance_matrix(g, d["sigma"], terms, config=SolverConfig(tol=1e-14),
                                 report=rep,
                                 gpu=GPUConfig(precision=precision,
                                               preconditioner=preconditioner))
    # the conductances themselves against the oracle (pinned to the reference
    # in tests/test_oracle_golden.py); copper next to silicon makes the system
    # stiff (contrast 6e5), so the solve runs to relres 1e-14 for 1e-9 here
    from oracle import fs_oracle as O
    og = O.Grid(d["x"], d["y"], d["z"])
    _, Yo = O.resistance_matrix(og, d["sigma"], [t.nodes for t in terms], method="direct")
    Yo = 0.5 * (Yo + Yo.T)
    Y = rep["Y"]
    assert np.abs(Y - Yo).max() <= 1e-9 * np.abs(np.diag(Yo)).max()
    assert rep["row_sum_rel"] < 1e-9
    assert np.all(np.diag(Y) > 0) and np.all(Y - np.diag(np.diag(Y)) <= 0)
    # R itself is NumPy's pinv of the symmetrised Y, as in the reference.
    # Y's all-ones direction is null only to round-off, so R carries
    # 1/lambda_min (1e12 and more, different for every solve) along it and
    # cannot be compared entry by entry; its physical part is Y, checked above.
    assert np.all(np.isfinite(R))
    assert np.array_equal(R, np.linalg.pinv(Y))


def test_resistance_rejects_bad_input(cuda):
    from fieldspice_b200 import extraction as EX
    from fieldspice_b200.grid import RectilinearGrid
    from fieldspice_b200.solvers.base import Terminal
    g = RectilinearGrid(np.linspace(0, 1, 5), np.linspace(0, 1, 4), np.linspace(0, 1, 3))
    sig = np.ones(g.shape_cells)
    with pytest.raises(ValueError, match="two terminals"):
        EX.resistance_matrix(g, sig, [Terminal("a", np.array([0]))])
    with pytest.raises(ValueError, match="non-negative"):
        EX.resistance_matrix(g, -sig, [Terminal("a", np.array([0])), Terminal("b", np.array([5]))])
