"""GPU field region (``circuit/coupling.py``) against the reference (needs a B200).

* The reduced admittances of a seeded three-electrode region (doped silicon,
  leaky oxide, two copper straps) at dc and at two step sizes, and the whole
  call sequence the reference's own MNA transient made on it (every history
  current, every accepted field), recorded in ``tests/golden/field_region.npz``
  and replayed here through the GPU region.
* The closed forms of the reference's tests (``tests/test_quasistatic.py``):
  a uniform resistor's ``1/Y`` is ``d/(sigma W H)``, an insulating slab's
  ``Y dt`` is ``eps A/d``, a capacitive region is open at dc, and the region
  driven through a resistor by a step follows ``1 - exp(-t/RC)`` to first
  order in ``dt`` (a minimal backward-Euler nodal analysis stands in for the
  reference's MNA solver).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS0 = 8.8541878188e-12


def _terminals(d, g):
    from fieldspice_b200.solvers.base import Terminal
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    return [Terminal(f"e{i}", nid[a0:a1 + 1, b0:b1 + 1, c0:c1 + 1].ravel())
            for i, (a0, b0, c0, a1, b1, c1) in enumerate(d["boxes"])]


@pytest.mark.parametrize("precision,preconditioner",
                         [("auto", "mg"), ("fp64", "mg"), ("auto", "jacobi")])
def test_field_region_replays_reference_mna_run(cuda, golden, precision, preconditioner):
    from fieldspice_b200.circuit import FieldRegion
    from fieldspice_b200.grid import RectilinearGrid
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig
    d = golden("field_region")
    g = RectilinearGrid(d["x"], d["y"], d["z"])
    cfg = SolverConfig(tol=1e-13)
    gcfg = GPUConfig(precision=precision, preconditioner=preconditioner)
    fr = FieldRegion("FR", g, d["eps"], d["sigma"], _terminals(d, g),
                     circuit_nodes=["0", "a", "b"], config=cfg, gpu=gcfg)
    for key, dt in (("Y_dc", None), ("Y_dt1e-13", 1e-13), ("Y_dt2e-12", 2e-12)):
        Y = fr.terminal_admittance(dt)
        assert np.abs(Y - d[key]).max() <= 1e-9 * np.abs(d[key]).max(), key
        assert fr.asymmetry < 1e-9
    fr.close()
    fr = FieldRegion("FR", g, d["eps"], d["sigma"], _terminals(d, g),
                     circuit_nodes=["0", "a", "b"], config=cfg, gpu=gcfg)
    nmap = {"a": 0, "b": 1}
    phis = dict(zip(d["phi_at"].tolist(), d["phi"]))
    checked = 0
    for i, kind in enumerate(d["ev_kind"]):
        dt = float(d["ev_dt"][i])
        if kind == 0:
            G = np.zeros((3, 3))
            fr.stamp_dc(G, np.zeros(3), None, nmap)
            want = d["ev_Y"][i][1:, 1:]
            assert np.abs(G[:2, :2] - want).max() <= 1e-9 * np.abs(want).max()
        elif kind == 1:
            G, I = np.zeros((3, 3)), np.zeros(3)
            fr.stamp_tran(G, I, None, None, dt, nmap)
            want_Y = d["ev_Y"][i][1:, 1:]
            assert np.abs(G[:2, :2] - want_Y).max() <= 1e-9 * np.abs(want_Y).max()
            want_f = d["ev_vec"][i]
            scale = max(np.abs(want_f).max(), 1e-30)
            # ground row dropped: I holds f_eff for the electrodes "a" and "b"
            assert np.abs(I[:2] - want_f[1:]).max() <= 1e-8 * scale, i
        else:
            v = d["ev_vec"][i]
            x = np.array([v[1], v[2], 0.0])
            fr.accept_timestep(x, None, dt, nmap)
            if i in phis:
                assert np.abs(fr.phi - phis[i]).max() <= 1e-8, i
                checked += 1
    assert checked == len(phis)
    fr.close()


def _slab(n=16):
    from fieldspice_b200.grid import RectilinearGrid
    from fieldspice_b200.solvers.base import Terminal
    d, W, H = 2e-6, 5e-6, 4e-6
    g = RectilinearGrid(np.linspace(0, d, n), np.linspace(0, W, 6), np.linspace(0, H, 5))
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    terms = [Terminal("a", nid[0].ravel()), Terminal("b", nid[-1].ravel())]
    return g, terms, d, W, H


def test_reduced_admittance_reproduces_field_resistance(cuda):
    from fieldspice_b200.circuit import FieldRegion
    g, terms, d, W, H = _slab()
    sigma = 1e4
    fr = FieldRegion("FR", g, np.full(g.shape_cells, 3.9 * EPS0),
                     np.full(g.shape_cells, sigma), terms, circuit_nodes=["a", "b"])
    Y = fr.terminal_admittance(None)
    assert 1.0 / Y[0, 0] == pytest.approx(d / (sigma * W * H), rel=1e-9)
    assert fr.asymmetry < 1e-9
    assert abs(Y.sum(axis=1)).max() <= 1e-9 * Y[0, 0]


def test_reduced_admittance_reproduces_field_capacitance(cuda):
    from fieldspice_b200.circuit import FieldRegion
    g, terms, d, W, H = _slab()
    er, dt = 3.9, 1e-12
    fr = FieldRegion("FR", g, np.full(g.shape_cells, er * EPS0),
                     np.zeros(g.shape_cells), terms, circuit_nodes=["a", "b"])
    Y = fr.terminal_admittance(dt)
    assert Y[0, 0] * dt == pytest.approx(er * EPS0 * W * H / d, rel=1e-9)


def test_capacitive_region_is_open_at_dc(cuda):
    from fieldspice_b200.circuit import FieldRegion
    from fieldspice_b200.grid import RectilinearGrid
    from fieldspice_b200.solvers.base import Terminal
    g = RectilinearGrid.uniform([(0, 2e-6), (0, 5e-6), (0, 4e-6)], [8, 4, 3])
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    terms = [Terminal("a", nid[0].ravel()), Terminal("b", nid[-1].ravel())]
    fr = FieldRegion("FR", g, np.full(g.shape_cells, 3.9 * EPS0),
                     np.zeros(g.shape_cells), terms, circuit_nodes=["a", "b"])
    assert np.abs(fr.terminal_admittance(None)).max() == 0.0
    G = np.zeros((2, 2))
    fr.stamp_dc(G, np.zeros(2), None, {"a": 0, "b": 1})
    assert np.abs(G).max() == 0.0


def test_reset_state_keeps_integration_history(cuda):
    from fieldspice_b200.circuit import FieldRegion
    g, terms, *_ = _slab()
    fr = FieldRegion("FR", g, np.full(g.shape_cells, 3.9 * EPS0),
                     np.full(g.shape_cells, 1e4), terms, circuit_nodes=["a", "b"])
    fr.phi = np.ones(g.n_nodes) * 0.25
    fr.reset_state()
    assert np.allclose(fr.phi, 0.25)
    fr.reset_history()
    assert np.allclose(fr.phi, 0.0)


def test_electrodes_only_region(cuda):
    """Every node an electrode: ``Y = K_tt`` with no interior solve
    (coupling.py:169-172); a 2x2x2-node cube split into two faces."""
    from fieldspice_b200.circuit import FieldRegion
    from fieldspice_b200.grid import RectilinearGrid
    from fieldspice_b200.solvers.base import Terminal
    from oracle import fs_oracle as O
    g = RectilinearGrid(np.array([0, 1e-6]), np.array([0, 2e-6]), np.array([0, 3e-6]))
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    terms = [Terminal("a", nid[0].ravel()), Terminal("b", nid[1].ravel())]
    eps = np.full(g.shape_cells, 2.0 * EPS0)
    sig = np.full(g.shape_cells, 3.0)
    fr = FieldRegion("FR", g, eps, sig, terms, circuit_nodes=["a", "b"])
    og = O.Grid(g.xn, g.yn, g.zn)
    ofr = O.FieldRegionCPU(og, eps, sig, [t.nodes for t in terms])
    for dt in (None, 1e-9):
        want = ofr.reduce(dt)["Y"]
        assert np.abs(fr.terminal_admittance(dt) - want).max() <= 1e-12 * np.abs(want).max()
    nmap = {"a": 0, "b": 1}
    fr.stamp_tran(np.zeros((2, 2)), np.zeros(2), None, None, 1e-9, nmap)
    fr.accept_timestep(np.array([0.7, -0.2]), None, 1e-9, nmap)
    ofr.accept(np.array([0.7, -0.2]), 1e-9)
    assert np.array_equal(fr.phi, ofr.phi)
    I = np.zeros(2)
    fr.stamp_tran(np.zeros((2, 2)), I, None, None, 1e-9, nmap)
    want = ofr.history(1e-9)
    assert np.abs(I - want).max() <= 1e-12 * np.abs(want).max()


def _be_rc(fr, R, t0, dt, n):
    """Backward-Euler nodal analysis of V(step at t0) -R- out, with the field
    region between ``out`` and ground; unknowns [v_in, v_out, i_V]."""
    nmap = {"out": 1}
    x = np.zeros(3)
    ts, vs = [0.0], [0.0]
    for k in range(1, n + 1):
        t = k * dt
        G = np.zeros((3, 3))
        I = np.zeros(3)
        g = 1.0 / R
        G[0, 0] += g
        G[1, 1] += g
        G[0, 1] -= g
        G[1, 0] -= g
        G[0, 2] += 1.0
        G[2, 0] += 1.0
        I[2] = 1.0 if t >= t0 * (1 - 1e-12) else 0.0
        fr.stamp_tran(G, I, x, x, dt, nmap, t)
        x_new = np.linalg.solve(G, I)
        fr.accept_timestep(x_new, x, dt, nmap)
        x = x_new
        ts.append(t)
        vs.append(x[1])
    return np.array(ts), np.array(vs)


def test_coupled_rc_transient_matches_analytic(cuda):
    from fieldspice_b200.circuit import FieldRegion
    g, terms, d, W, H = _slab()
    er = 3.9
    Cf = er * EPS0 * W * H / d
    R = 1e6
    tau = R * Cf
    t0 = 2 * tau
    errs = []
    for spt in (25, 100, 400):
        fr = FieldRegion("FR", g, np.full(g.shape_cells, er * EPS0),
                         np.zeros(g.shape_cells), terms, circuit_nodes=["out", "0"])
        dt = tau / spt
        t, v = _be_rc(fr, R, t0, dt, int(np.ceil((t0 + 8 * tau) / dt)))
        m = t >= t0 * (1 - 1e-12)
        errs.append(np.abs(v[m] - (1.0 - np.exp(-(t[m] - t0) / tau))).max())
        fr.close()
    assert errs[-1] < 6e-3
    for lo, hi in zip(errs[:-1], errs[1:]):
        assert 3.0 < lo / hi < 5.0
