"""GPU per-unit-length line parameters against the reference (needs a B200).

``extraction.rlgc_2d`` (``extraction.py:108-206``) on a seeded coupled
microstrip (two copper lines on a lossy FR-4-like substrate over a ground
plane, air above, collapsed z), recorded from the reference in
``tests/golden/rlgc.npz``: the return conductor by default, by name and by
index, at dc and at 1 GHz.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(d):
    from fieldspice_b200.grid import RectilinearGrid
    from fieldspice_b200.solvers.base import Terminal
    g = RectilinearGrid(d["x"], d["y"], None)
    terms = [Terminal(n, d[f"term{i}"]) for i, n in enumerate(("s1", "s2", "gnd"))]
    return g, terms


@pytest.mark.parametrize("tag,kw", [("dc", {}), ("ghz", {"freq": 1e9}),
                                    ("name", {"reference": "gnd"}), ("ref0", {"reference": 0})])
def test_rlgc_2d_matches_reference(cuda, golden, tag, kw):
    from fieldspice_b200 import extraction as EX
    from fieldspice_b200.solvers.base import SolverConfig
    d = golden("rlgc")
    g, terms = _problem(d)
    r = EX.rlgc_2d(g, d["eps"], d["sigma"], terms, config=SolverConfig(tol=1e-12), **kw)
    assert r["reference"] == str(d[f"{tag}_reference"])
    for k in ("C", "C_air", "L", "eps_eff", "Z0", "v_p"):
        want = d[f"{tag}_{k}"]
        assert np.abs(r[k] - want).max() <= 1e-9 * np.abs(want).max(), k
    # G: the reference integrates L @ phi with the assembled CSR; on the copper
    # traces (5.8e7 S/m inside the electrodes) the diagonal d ~ 1e8 cancels
    # against its off-diagonals and leaves ~5e-8 of round-off in G (3e-5
    # relative; its rows no longer sum to zero).  The GPU and the oracle's
    # edge-by-edge integration G^T (m * G phi) do not cancel: they agree to
    # 1e-9, and the reference within its round-off.
    from oracle import fs_oracle as O
    og = O.Grid(d["x"], d["y"], np.array([0.0, 1.0]))
    ref = kw.get("reference", -1)
    ref = {"gnd": 2}.get(ref, ref)
    Go = O.rlgc_2d_matrices(og, d["eps"], d["sigma"], [t.nodes for t in terms], reference=ref,
                            charge="edges")["G"]
    assert np.abs(r["G"] - Go).max() <= 1e-9 * np.abs(Go).max()
    # the reference's CSR round-off: up to ~eps * d_n on every electrode node
    sig = np.maximum(d["sigma"], 1e-30)
    Lm = O.nodal_laplacian(og, O.edge_mass_vector(og, O.cell_to_edge(og, sig)))
    dn = np.abs(Lm.diagonal())
    keep = [i for i in range(3) if i != ref % 3]
    D = np.array([dn[terms[i].nodes].sum() for i in keep])
    floor = 4 * 2.2e-16 * np.maximum(D[:, None], D[None, :])
    assert np.all(np.abs(r["G"] - d[f"{tag}_G"]) <= 1e-9 * np.abs(Go).max() + floor)
    assert np.array_equal(r["R"], d[f"{tag}_R"])
    # the TEM identity holds for the vacuum matrices
    assert EX.check_lc_identity({"L": r["L"], "C": r["C_air"]}) < 1e-9


def test_rlgc_2d_rejects_bad_input(cuda, golden):
    from fieldspice_b200 import extraction as EX
    from fieldspice_b200.grid import RectilinearGrid
    d = golden("rlgc")
    g, terms = _problem(d)
    with pytest.raises(ValueError, match="at least two conductors"):
        EX.rlgc_2d(g, d["eps"], d["sigma"], terms[:1])
    with pytest.raises(ValueError, match="not among"):
        EX.rlgc_2d(g, d["eps"], d["sigma"], terms, reference="nope")
    g3 = RectilinearGrid(d["x"], d["y"], np.array([0.0, 1.0, 2.0]))
    with pytest.raises(ValueError, match="2D cross-section"):
        EX.rlgc_2d(g3, np.zeros(g3.shape_cells), np.zeros(g3.shape_cells), terms)
