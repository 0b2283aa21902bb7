"""Pin the CPU oracle to the reference's recorded outputs (CPU only).

The fixtures in ``tests/golden`` were produced by running the reference
fieldspice package (``tests/golden/make_golden.py``).  The oracle restates
the reference's algorithm; here it must reproduce every fixture: masses
bit-for-bit, Laplacian applies to FP64 round-off, and the capacitance
matrices and EQS currents to the tolerances the reference's own tests use.
"""

import numpy as np
import pytest
import scipy.sparse as sp

from oracle import fs_oracle as O

GRIDS = ("graded", "uniform", "collapsed", "wide")


def _grid(d, name):
    return O.Grid(d[f"{name}_xn"], d[f"{name}_yn"], d[f"{name}_zn"])


@pytest.mark.parametrize("name", GRIDS)
def test_masses_bit_exact(golden, name):
    d = golden("masses")
    g = _grid(d, name)
    prop = d[f"{name}_prop"]
    pe = O.cell_to_edge(g, prop, "parallel")
    assert np.array_equal(pe, d[f"{name}_eps_edge"])
    assert np.array_equal(O.edge_mass_vector(g, pe), d[f"{name}_mass_parallel"])
    ph = O.cell_to_edge(g, prop, "harmonic")
    assert np.array_equal(O.edge_mass_vector(g, ph), d[f"{name}_mass_harmonic"])


@pytest.mark.parametrize("name", GRIDS)
def test_incidence_and_laplacian_match_reference(golden, name):
    d = golden("masses")
    g = _grid(d, name)
    G = O.grad_node_edge(g)
    assert np.array_equal(G.indptr, d[f"{name}_G_indptr"])
    assert np.array_equal(G.indices, d[f"{name}_G_indices"])
    assert np.array_equal(G.data, d[f"{name}_G_data"])
    m = O.edge_mass_vector(g, O.cell_to_edge(g, d[f"{name}_prop"]))
    L = O.nodal_laplacian(g, m)
    Lref = sp.csr_matrix((d[f"{name}_L_data"], d[f"{name}_L_indices"],
                          d[f"{name}_L_indptr"]), shape=L.shape)
    assert abs(L - Lref).max() <= 1e-15 * abs(Lref).max()
    y = L @ d[f"{name}_x"]
    assert np.abs(y - d[f"{name}_Lx"]).max() <= 1e-14 * np.abs(d[f"{name}_Lx"]).max()


@pytest.mark.parametrize("name", GRIDS)
def test_topology_identities_exact(golden, name):
    # tests/test_core.py:132-180 of the reference: C@G == 0 and D@C == 0
    # exactly, entries are +-1.
    g = _grid(golden("masses"), name)
    G, C, D = O.grad_node_edge(g), O.curl_edge_face(g), O.div_face_cell(g)
    CG, DC = C @ G, D @ C
    assert CG.nnz == 0 or np.abs(CG.data).max() == 0.0
    assert DC.nnz == 0 or np.abs(DC.data).max() == 0.0
    for M in (G, C, D):
        assert set(np.unique(M.data)).issubset({-1.0, 1.0})
    assert np.abs(G @ np.ones(g.n_nodes)).max() == 0.0


def test_readme_capacitor(golden):
    from fieldspice_b200 import workloads as W
    d = golden("readme")
    w = W.parallel_plate()
    g = O.Grid(w.x, w.y, w.z)
    C, rep = O.capacitance_matrix(g, w.eps_cell, w.terminals, method="direct")
    assert np.allclose(C, d["C"], rtol=1e-12, atol=0)
    assert C[0, 0] == pytest.approx(w.meta["C_ref"], rel=1e-12)
    # CG path too (Jacobi), at the README's 1e-12 requirement
    C2, _ = O.capacitance_matrix(g, w.eps_cell, w.terminals, method="cg", tol=1e-13)
    assert C2[0, 0] == pytest.approx(w.meta["C_ref"], rel=1e-12)


@pytest.mark.parametrize("tag", ["layered_32x32x16_s0", "layered_48x48x24_s1"])
def test_layered_capacitance_matches_reference(golden, tag):
    d = golden(tag)
    g = O.Grid(d["x"], d["y"], d["z"])
    nx, ny, nz = g.shape_nodes
    nid = np.arange(g.n_nodes).reshape(nx, ny, nz)
    terms = [nid[a0:a1 + 1, b0:b1 + 1, c0:c1 + 1].ravel() for a0, b0, c0, a1, b1, c1 in d["boxes"]]
    C, rep = O.capacitance_matrix(g, d["eps_cell"], terms, {"zlo": 0.0},
                                  method="cg", tol=float(d["tol"]))
    scale = np.abs(np.diag(d["C"])).max()
    assert np.abs(C - d["C"]).max() / scale < 1e-11
    assert np.abs(rep["shield_charge"] - d["shield"]).max() / scale < 1e-11


def test_closed_forms(golden):
    d = golden("closed_forms")
    assert d["series_C"][0, 0] == pytest.approx(float(d["series_ref"]), rel=1e-10)
    assert d["graded_C"][0, 0] == pytest.approx(float(d["graded_ref"]), rel=1e-10)
    g = O.Grid(d["graded_xn"], d["graded_yn"], d["graded_zn"])
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    eps = np.full(g.shape_cells, 3.9 * O.EPS0)
    C, _ = O.capacitance_matrix(g, eps, [nid[0].ravel(), nid[-1].ravel()], method="direct")
    assert np.allclose(C, d["graded_C"], rtol=1e-12, atol=0)


def test_eqs_interconnect_matches_reference(golden):
    from fieldspice_b200 import workloads as W
    d = golden("eqs")
    g = O.Grid(d["ic_x"], d["ic_y"], d["ic_z"])
    nx, ny, nz = g.shape_nodes
    nid = np.arange(g.n_nodes).reshape(nx, ny, nz)
    boxes = d["ic_boxes"]
    ports = [nid[a0:a1 + 1, b0:b1 + 1, c0:c1 + 1].ravel() for a0, b0, c0, a1, b1, c1 in boxes[:2]]
    ramp = W.ramp(0.0, 0.0, 1.0, 10e-12)
    # terminals first, then the zlo wall: the wall wins on shared nodes
    phis, cur = O.eqs_transient(g, d["ic_eps"], d["ic_sig"], ports,
                                lambda t: (ramp(t), 0.0), 1e-12, 20, tol=1e-12,
                                dirichlet_walls={"zlo": 0.0})
    scale = np.abs(d["ic_i0"]).max()
    assert np.abs(cur[:, 0] - d["ic_i0"]).max() / scale < 1e-8
    assert np.abs(cur[:, 1] - d["ic_i1"]).max() / scale < 1e-8
    assert np.abs(phis[-1] - d["ic_phi_last"]).max() < 1e-9


def test_eqs_rc_stack_matches_reference(golden):
    d = golden("eqs")
    g = O.Grid(d["xn"], d["yn"], d["zn"])
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    tau = float(d["tau"])
    phis, cur = O.eqs_transient(g, d["eps"], d["sig"], [nid[0].ravel(), nid[-1].ravel()],
                                lambda t: (1.0, 0.0), tau / 50, 400, method="direct")
    vm = np.array([p[nid[30, 1, 1]] for p in phis])
    assert np.abs(vm - d["spt50_vm"]).max() < 1e-10
    scale = np.abs(d["spt50_i_hi"]).max()
    assert np.abs(cur[:, 0] - d["spt50_i_hi"]).max() / scale < 1e-8


def _projected(R):
    n = R.shape[0]
    P = np.eye(n) - np.ones((n, n)) / n
    return P @ R @ P


def test_resistance_matrix_matches_reference(golden):
    # extraction.py:59-87: pinv keeps the round-off-null all-ones direction,
    # so only P R P (resistance differences) is reproducible
    d = golden("resistance")
    g = O.Grid(d["x"], d["y"], d["z"])
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    terms = [nid[a0:a1 + 1, b0:b1 + 1, c0:c1 + 1].ravel() for a0, b0, c0, a1, b1, c1 in d["boxes"]]
    R, Y = O.resistance_matrix(g, d["sigma"], terms, method="direct")
    want = _projected(d["R"])
    assert np.abs(_projected(R) - want).max() <= 1e-9 * np.abs(want).max()
    assert np.abs(Y.sum(axis=1)).max() <= 1e-9 * np.abs(np.diag(Y)).max()


def test_thermal_matches_reference(golden):
    # solvers/thermal.py:200-300: steady with a Dirichlet sink and convective
    # walls, theta-scheme transients (theta 1 and 1/2), direct solves
    d = golden("thermal")
    g = O.Grid(d["x"], d["y"], d["z"])
    conv = {"zhi": (2e4, 310.0), "xlo": (5e3, 295.0)}
    T = O.thermal_steady(g, d["kappa"], d["q"], {"zlo": 300.0}, conv, method="direct")
    assert np.abs(T - d["T_steady"]).max() <= 1e-9 * np.abs(d["T_steady"] - 300.0).max()
    for theta in (1.0, 0.5):
        Ts = O.thermal_transient(g, d["kappa"], d["rho_cp"], d["q"], 2e-5, 1e-6, 300.0,
                                 {"zlo": 300.0}, conv, theta=theta, method="direct")
        want = d[f"T_transient_theta{theta:g}"]
        assert len(Ts) == want.shape[0]
        assert np.abs(np.array(Ts) - want).max() <= 1e-9 * np.abs(want - 300.0).max()


def field_region_terminals(d, g):
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    return [nid[a0:a1 + 1, b0:b1 + 1, c0:c1 + 1].ravel() for a0, b0, c0, a1, b1, c1 in d["boxes"]]


def test_field_region_matches_reference(golden):
    """coupling.py: reduced admittances and the recorded MNA call sequence
    (every history current and every accepted field) replayed through the
    oracle's restatement."""
    d = golden("field_region")
    g = O.Grid(d["x"], d["y"], d["z"])
    fr = O.FieldRegionCPU(g, d["eps"], d["sigma"], field_region_terminals(d, g))
    for key, dt in (("Y_dc", None), ("Y_dt1e-13", 1e-13), ("Y_dt2e-12", 2e-12)):
        Y = fr.reduce(dt)["Y"]
        assert np.abs(Y - d[key]).max() <= 1e-12 * np.abs(d[key]).max(), key
    fr = O.FieldRegionCPU(g, d["eps"], d["sigma"], field_region_terminals(d, g))
    phis = dict(zip(d["phi_at"].tolist(), d["phi"]))
    for i, kind in enumerate(d["ev_kind"]):
        dt = None if kind == 0 else float(d["ev_dt"][i])
        if kind in (0, 1):
            Y = fr.reduce(dt)["Y"]
            assert np.abs(Y - d["ev_Y"][i]).max() <= 1e-12 * np.abs(Y).max()
        if kind == 1:
            f = fr.history(dt)
            want = d["ev_vec"][i]
            assert np.abs(f - want).max() <= 1e-10 * max(np.abs(want).max(), 1e-30)
        if kind == 2:
            fr.accept(d["ev_vec"][i], dt)
            if i in phis:
                assert np.abs(fr.phi - phis[i]).max() <= 1e-12


def test_rlgc_matrices_match_reference(golden):
    """extraction.py:108-206 on a coupled-microstrip cross-section: the
    oracle's three capacitance extractions reproduce the reference's C,
    C_air, G and L with the ground and with the first line as the return."""
    d = golden("rlgc")
    g = O.Grid(d["x"], d["y"], np.array([0.0, 1.0]))
    terms = [d["term0"], d["term1"], d["term2"]]
    for tag, ref in (("dc", -1), ("ref0", 0)):
        got = O.rlgc_2d_matrices(g, d["eps"], d["sigma"], terms, reference=ref)
        for k in ("C", "C_air", "G", "L"):
            want = d[f"{tag}_{k}"]
            assert np.abs(got[k] - want).max() <= 1e-10 * np.abs(want).max(), (tag, k)


def test_ac_matches_reference(golden):
    """solvers/ac.py: admittance matrices of a lossy three-terminal structure
    at four frequencies, the currents of a complex-driven solve, and the
    field region's frequency-domain stamp (coupling.py:214-236)."""
    d = golden("ac")
    g = O.Grid(d["x"], d["y"], d["z"])
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    terms = [nid[a0:a1 + 1, b0:b1 + 1, c0:c1 + 1].ravel() for a0, b0, c0, a1, b1, c1 in d["boxes"]]
    Y = O.ac_admittance(g, d["eps"], d["sigma"], terms, d["freqs"])
    for k in range(d["freqs"].size):
        assert np.abs(Y[k] - d["Y"][k]).max() <= 1e-9 * np.abs(d["Y"][k]).max(), k
    # a driven solve is Y times the drive vector
    v = np.array([1.0, 0.5, 0.0])
    for k in range(1, d["freqs"].size):
        want = d["solve_i"][:, k - 1]
        assert np.abs(Y[k] @ v - want).max() <= 1e-9 * np.abs(want).max()
    f = golden("field_region")
    g2 = O.Grid(f["x"], f["y"], f["z"])
    t2 = field_region_terminals(f, g2)
    Ys = O.ac_schur(g2, f["eps"], f["sigma"], t2, 2 * np.pi * 1e9)
    want = d["fr_stamp_ac"]
    assert np.abs(Ys[1:, 1:] - want).max() <= 1e-9 * np.abs(want).max()


def test_floating_electrodes_match_reference(golden):
    """poisson.py: a floating and a charge-driven conductor merged into single
    unknowns next to a driven electrode, a grounded floor and free charge."""
    d = golden("floating")
    g = O.Grid(d["x"], d["y"], d["z"])
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    nodes = [nid[a0:a1 + 1, b0:b1 + 1, c0:c1 + 1].ravel() for a0, b0, c0, a1, b1, c1 in d["boxes"]]
    wall = nid[:, :, 0].ravel()
    fixed = np.concatenate([wall, nodes[0]])
    vals = np.concatenate([np.zeros(wall.size), np.ones(nodes[0].size)])
    b_free = d["rho"].ravel() * g.node_volumes().ravel()
    b_ext = b_free.copy()
    b_ext[nodes[2][0]] += 2e-17
    phi, Lm = O.merged_potential(g, d["eps"], fixed, vals, [nodes[1], nodes[2]], b_ext)
    assert np.abs(phi - d["phi"]).max() <= 1e-10
    q = Lm @ phi - b_free
    for name, nd in zip(("drv", "flt", "chg"), nodes):
        assert abs(q[nd].sum() - d[f"q_{name}"][0]) <= 1e-9 * abs(d["q_drv"][0])
        assert abs(phi[nd[0]] - d[f"v_{name}"][0]) <= 1e-10


def _periodic_terms(d, g):
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    t = [nid[a0:a1 + 1, b0:b1 + 1, c0:c1 + 1].ravel() for a0, b0, c0, a1, b1, c1 in d["boxes"]]
    return t + [d["wrap_nodes"]]


@pytest.mark.parametrize("tag,axes", [("x", ("x",)), ("xy", ("x", "y"))])
def test_periodic_walls_match_reference(golden, tag, axes):
    """poisson.py with Periodic walls: capacitance (symmetrised) and a driven
    potential with free charge, through the oracle's node merge."""
    d = golden("periodic")
    g = O.Grid(d["x"], d["y"], d["z"])
    terms = _periodic_terms(d, g)
    C = O.periodic_capacitance(g, d["eps"], terms, axes, {"zlo": 0.0})
    C = 0.5 * (C + C.T)
    assert np.abs(C - d[f"C_{tag}"]).max() <= 1e-10 * np.abs(np.diag(C)).max()
    wall = np.arange(g.n_nodes).reshape(g.shape_nodes)[:, :, 0].ravel()
    fixed = np.concatenate([wall] + terms)
    vals = np.concatenate([np.zeros(wall.size)] + [np.full(t.size, v)
                                                  for t, v in zip(terms, (1.0, -0.5, 0.25))])
    fixed, vals = O.unique_last(fixed, vals)
    b_free = d["rho"].ravel() * g.node_volumes().ravel()
    phi, Lm = O.periodic_potential(g, d["eps"], fixed, vals, axes, b_free)
    assert np.abs(phi - d[f"phi_{tag}"]).max() <= 1e-10
