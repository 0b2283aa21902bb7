"""Generate the golden fixtures by running the reference fieldspice package.

Run in a container where the reference source tree is available:

    FIELDSPICE_REF=/path/to/fieldspice python tests/golden/make_golden.py

The reference is imported from that path and executed on small seeded
inputs; its outputs are written next to this script as ``.npz`` files.  The
tests never import the reference: they compare the CPU oracle and the GPU
library against these recorded outputs.

Iterative reference solves force SciPy's Jacobi branch of ``LinearSystem``
(``fieldspice/solvers/poisson.py:472-484``) by making ``spilu`` raise: the
default incomplete-LU branch stalls on these systems.
"""

from __future__ import annotations

import contextlib
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REF = os.environ.get("FIELDSPICE_REF")
if not REF:
    raise SystemExit("set FIELDSPICE_REF to the reference fieldspice source tree")
sys.path.insert(0, REF)
sys.path.insert(0, str(HERE.parents[1]))

import scipy.sparse.linalg as spla  # noqa: E402

import fieldspice as fs  # noqa: E402
from fieldspice import operators as ops  # noqa: E402
from fieldspice.boundaries import BoundarySpec, Dirichlet  # noqa: E402
from fieldspice.grid import RectilinearGrid, graded_1d  # noqa: E402
from fieldspice.solvers.base import SolverConfig, Terminal  # noqa: E402
from fieldspice.solvers.eqs import EQSSolver  # noqa: E402
from fieldspice.solvers.poisson import PoissonSolver  # noqa: E402
from fieldspice.units import eps0  # noqa: E402

from fieldspice_b200 import workloads as W  # noqa: E402  (input generator only)


@contextlib.contextmanager
def jacobi_forced():
    orig = spla.spilu

    def _raise(*a, **k):
        raise MemoryError("incomplete LU disabled: Jacobi branch forced")
    spla.spilu = _raise
    try:
        yield
    finally:
        spla.spilu = orig


def graded_grid():
    # the awkward grid of tests/test_core.py:25-36 ("3d_graded")
    return RectilinearGrid(graded_1d(0, 1e-3, 7, 1.3), graded_1d(0, 2e-3, 5, 0.8),
                           graded_1d(0, 3e-4, 4, 1.5))


def masses_fixture():
    out = {}
    rng = np.random.default_rng(1234)
    for name, g in {"graded": graded_grid(),
                    "uniform": RectilinearGrid.uniform([(0, 1), (0, 1), (0, 1)], [4, 3, 2]),
                    "collapsed": RectilinearGrid(graded_1d(0, 1e-3, 7, 1.3),
                                                 graded_1d(0, 2e-3, 5, 0.8), None),
                    "wide": RectilinearGrid(np.sort(rng.uniform(0, 1, 12)),
                                            np.sort(rng.uniform(0, 1, 9)),
                                            np.sort(rng.uniform(0, 1, 7)))}.items():
        prop = rng.uniform(1.0, 12.0, g.shape_cells) * eps0
        pe = ops.cell_to_edge(g, prop, "parallel")
        ph = ops.cell_to_edge(g, prop, "harmonic")
        mp = ops.edge_mass(g, pe).diagonal()
        mh = ops.edge_mass(g, ph).diagonal()
        Lm = ops.nodal_laplacian(g, pe)
        x = rng.standard_normal((g.n_nodes, 3))
        y = Lm @ x
        G = ops.grad_node_edge(g)
        out.update({f"{name}_xn": g.xn, f"{name}_yn": g.yn, f"{name}_zn": g.zn,
                    f"{name}_prop": prop, f"{name}_eps_edge": pe,
                    f"{name}_mass_parallel": mp, f"{name}_mass_harmonic": mh,
                    f"{name}_x": x, f"{name}_Lx": y,
                    f"{name}_L_indptr": Lm.indptr, f"{name}_L_indices": Lm.indices,
                    f"{name}_L_data": Lm.data,
                    f"{name}_G_indptr": G.indptr, f"{name}_G_indices": G.indices,
                    f"{name}_G_data": G.data})
    np.savez_compressed(HERE / "masses.npz", **out)


def readme_fixture():
    w = W.parallel_plate()
    g = RectilinearGrid(w.x, w.y, w.z)
    terms = [Terminal("top", w.terminals[0], voltage=1.0),
             Terminal("bottom", w.terminals[1], voltage=0.0)]
    ps = PoissonSolver(g, w.eps_cell)
    rep = {}
    C = ps.capacitance_matrix(terms, report=rep)
    res = ps.solve(terms)
    np.savez_compressed(HERE / "readme.npz", C=C, asym=rep["asymmetry_rel"],
                        row_sum_rel=rep["row_sum_rel"],
                        phi=res.fields["phi"].ravel(),
                        energy=res.scalars["energy"], q_top=res.terminals["top"]["q"])


def layered_fixture(shape, seed, tol):
    w = W.layered_boxes(shape, nbox=8, seed=seed)
    g = RectilinearGrid(w.x, w.y, w.z)
    terms = [Terminal(n, t) for n, t in zip(w.names, w.terminals)]
    bc = BoundarySpec(zlo=Dirichlet(0.0))
    rep = {}
    with jacobi_forced():
        ps = PoissonSolver(g, w.eps_cell, SolverConfig(linear_solver="cg", tol=tol))
        C = ps.capacitance_matrix(terms, bc, report=rep)
    tag = f"layered_{shape[0]}x{shape[1]}x{shape[2]}_s{seed}"
    np.savez_compressed(HERE / f"{tag}.npz", C=C, x=w.x, y=w.y, z=w.z,
                        eps_cell=w.eps_cell.astype(np.float64),
                        boxes=np.asarray(w.boxes), shield=rep["shield_charge"],
                        asym=rep["asymmetry_rel"], tol=tol,
                        iterations=rep["linear"].get("iterations", -1))


def resistance_fixture():
    """extraction.py:59-87 on a seeded conductor network: a doped-silicon
    slab, two copper straps on it, insulating oxide (sigma = 0) above, three
    terminals; small enough that the reference factorises it directly."""
    from fieldspice.extraction import resistance_matrix
    rng = np.random.default_rng(7)
    g = RectilinearGrid(np.sort(rng.uniform(0, 4e-6, 22)), np.linspace(0, 3e-6, 17),
                        np.linspace(0, 1e-6, 11))
    sig = np.zeros(g.shape_cells)
    sig[:, :, :4] = 1e2
    sig[2:19, 3:6, 4:6] = 5.8e7
    sig[2:19, 10:13, 4:6] = 5.8e7
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    boxes = [(0, 0, 0, 21, 16, 0), (2, 3, 5, 3, 6, 6), (18, 10, 5, 19, 13, 6)]
    terms = [Terminal(f"t{i}", nid[a0:a1 + 1, b0:b1 + 1, c0:c1 + 1].ravel())
             for i, (a0, b0, c0, a1, b1, c1) in enumerate(boxes)]
    R = resistance_matrix(g, sig, terms)
    np.savez_compressed(HERE / "resistance.npz", R=R, x=g.xn, y=g.yn, z=g.zn,
                        sigma=sig, boxes=np.asarray(boxes))


def thermal_fixture():
    """solvers/thermal.py: steady (Dirichlet heat sink + convective top),
    theta-scheme transients (theta 1 and 0.5) and a thermal resistance, on a
    seeded graded grid with silicon/oxide conductivities."""
    from fieldspice.solvers.thermal import ThermalSolver
    rng = np.random.default_rng(11)
    g = RectilinearGrid(np.sort(rng.uniform(0, 20e-6, 15)), np.sort(rng.uniform(0, 16e-6, 12)),
                        np.sort(rng.uniform(0, 8e-6, 10)))
    kappa = np.where(rng.random(g.shape_cells) < 0.5, 150.0, 1.4)
    rho_cp = rng.uniform(1.6e6, 2.1e6, g.shape_cells)
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    src = nid[5:9, 4:7, 7:9].ravel()
    q = np.zeros(g.n_nodes)
    q[src] = 2e-4
    bc = BoundarySpec(zlo=Dirichlet(300.0))
    conv = {"zhi": (2e4, 310.0), "xlo": (5e3, 295.0)}
    th = ThermalSolver(g, kappa, rho_cp)
    steady = th.steady(q, bc=bc, convection=conv).fields["T"][0]
    out = {"x": g.xn, "y": g.yn, "z": g.zn, "kappa": kappa, "rho_cp": rho_cp, "q": q,
           "src": src, "T_steady": steady}
    for theta in (1.0, 0.5):
        r = th.transient(q, t_end=2e-5, dt=1e-6, T0=300.0, bc=bc, convection=conv,
                         theta=theta, store=True)
        out[f"T_transient_theta{theta:g}"] = r.fields["T"]
    out["R_th"] = th.thermal_resistance(src, bc=bc, convection=conv, power=1e-3)
    np.savez_compressed(HERE / "thermal.npz", **out)


class _StampRecorder:
    """Wraps a reference device; logs every stamp and accept with their inputs
    and outputs (duck-typed: the MNA reads everything else through it)."""

    def __init__(self, dev):
        self.dev = dev
        self.log = []

    def __getattr__(self, name):
        return getattr(self.dev, name)

    def _own(self, nmap, stamp):
        idx = [nmap.get(n, -1) for n in self.dev.nodes]
        return idx, stamp

    def stamp_dc(self, G, I, x, nmap, t=None):
        self.dev.stamp_dc(G, I, x, nmap, t)
        self.log.append(("dc", None, self.dev.terminal_admittance(None).copy(), None, None))

    def stamp_tran(self, G, I, x, x_prev, dt, nmap, t=None):
        self.dev.stamp_tran(G, I, x, x_prev, dt, nmap, t)
        entry = self.dev._reduce(dt)
        f = self.dev._history(entry, dt)
        self.log.append(("tran", dt, entry["Y"].copy(), np.array(f, float), None))

    def accept_timestep(self, x, x_prev, dt, nmap):
        v = np.array([0.0 if nmap.get(n, -1) < 0 else float(x[nmap[n]])
                      for n in self.dev.nodes])
        self.dev.accept_timestep(x, x_prev, dt, nmap)
        self.log.append(("accept", dt, None, v, self.dev.phi.copy()))


def field_region_geometry():
    """Doped-silicon slab under oxide with two copper straps on it: a
    substrate contact on the bottom plane and the two straps are the
    electrodes (seeded graded x axis)."""
    rng = np.random.default_rng(21)
    g = RectilinearGrid(np.sort(rng.uniform(0, 4e-6, 18)), np.linspace(0, 3e-6, 13),
                        np.linspace(0, 1e-6, 9))
    sig = np.full(g.shape_cells, 1e-4)          # leaky oxide
    sig[:, :, :3] = 1e2                         # doped silicon
    eps = np.full(g.shape_cells, 3.9 * eps0)
    eps[:, :, :3] = 11.7 * eps0
    sig[2:15, 2:5, 3:5] = 5.8e7                 # copper straps
    sig[3:16, 8:11, 3:5] = 5.8e7
    eps[2:15, 2:5, 3:5] = eps0
    eps[3:16, 8:11, 3:5] = eps0
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    boxes = [(0, 0, 0, 17, 12, 0), (2, 2, 3, 15, 5, 5), (3, 8, 3, 16, 11, 5)]
    return g, eps, sig, boxes, nid


def field_region_fixture():
    """circuit/coupling.py:55-275: the reduced admittance of a three-electrode
    region at dc and at two step sizes, then the region inside the reference's
    own backward-Euler MNA transient (a stepped source through a resistor into
    one strap, the other strap terminated): every stamp and accept the MNA
    made is recorded with its inputs and outputs, so that another region
    implementation can be replayed through the same call sequence."""
    from fieldspice import sources as S
    from fieldspice.circuit.coupling import FieldRegion
    from fieldspice.circuit.mna import MNASolver, Netlist
    g, eps, sig, boxes, nid = field_region_geometry()
    terms = [Terminal(f"e{i}", nid[a0:a1 + 1, b0:b1 + 1, c0:c1 + 1].ravel())
             for i, (a0, b0, c0, a1, b1, c1) in enumerate(boxes)]
    cfg = SolverConfig(tol=1e-12)
    fr = FieldRegion("FR", g, eps, sig, terms, circuit_nodes=["0", "a", "b"], config=cfg)
    out = {"x": g.xn, "y": g.yn, "z": g.zn, "eps": eps, "sigma": sig,
           "boxes": np.asarray(boxes)}
    out["Y_dc"] = fr.terminal_admittance(None).copy()
    for dt in (1e-13, 2e-12):
        out[f"Y_dt{dt:g}"] = fr.terminal_admittance(dt).copy()
    rec = _StampRecorder(FieldRegion("FR", g, eps, sig, terms,
                                     circuit_nodes=["0", "a", "b"], config=cfg))
    net = Netlist()
    net.add_vsource("V1", "in", "0", S.step(0.5e-12, 0.0, 1.0, trise=0.4e-12))
    net.add_resistor("R1", "in", "a", 2e3)
    net.add_resistor("R2", "b", "0", 5e3)
    net.add_device(rec)
    solver = MNASolver(net)
    res = solver.transient(t_end=6e-12, dt=0.2e-12, method="be")
    out["t"] = res.t
    out["v_a"] = res.fields["x"][:, solver.index("a")]
    out["v_b"] = res.fields["x"][:, solver.index("b")]
    kinds = {"dc": 0, "tran": 1, "accept": 2}
    out["ev_kind"] = np.array([kinds[e[0]] for e in rec.log])
    out["ev_dt"] = np.array([0.0 if e[1] is None else e[1] for e in rec.log])
    nE = len(terms)
    out["ev_Y"] = np.array([e[2] if e[2] is not None else np.zeros((nE, nE))
                            for e in rec.log])
    out["ev_vec"] = np.array([e[3] if e[3] is not None else np.zeros(nE) for e in rec.log])
    acc = [i for i, e in enumerate(rec.log) if e[0] == "accept"]
    keep = acc[:: max(1, len(acc) // 4)] + acc[-1:]
    out["phi_at"] = np.array(keep)
    out["phi"] = np.array([rec.log[i][4] for i in keep])
    out["asymmetry"] = fr.asymmetry
    np.savez_compressed(HERE / "field_region.npz", **out)


def rlgc_fixture():
    """extraction.py:108-233: per-unit-length R, L, G, C of a coupled
    microstrip cross-section (two copper lines on a lossy substrate over a
    ground plane, air above; seeded graded x axis, collapsed z) at dc and at
    1 GHz, with the reference conductor given by index and by name."""
    from fieldspice.extraction import rlgc_2d
    rng = np.random.default_rng(5)
    x = np.unique(np.concatenate([np.linspace(0, 40e-6, 41),
                                  rng.uniform(12e-6, 28e-6, 10)]))
    y = np.linspace(0, 30e-6, 31)
    g = RectilinearGrid(x, y, None)
    xc = 0.5 * (x[:-1] + x[1:])
    yc = 0.5 * (y[:-1] + y[1:])
    X, Y = np.meshgrid(xc, yc, indexing="ij")
    eps = np.full(g.shape_cells, eps0)
    sig = np.zeros(g.shape_cells)
    sub = Y < 10e-6
    eps[sub] = 4.4 * eps0
    sig[sub] = 1e-3
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    xn, yn = g.xn, g.yn

    tol = 1e-12  # node coordinates carry round-off (linspace)

    def box(x0, x1, y0, y1):
        i = np.flatnonzero((xn >= x0 - tol) & (xn <= x1 + tol))
        j = np.flatnonzero((yn >= y0 - tol) & (yn <= y1 + tol))
        return nid[i[0]:i[-1] + 1, j[0]:j[-1] + 1, :].ravel()
    # copper exactly on the cells between each line's electrode nodes: a
    # copper cell touching a free node would carry the substrate current
    # through a 5.8e7 S/m edge, a difference of nearly equal potentials that
    # no solver resolves beyond ~1e-5 relative
    for x0, x1 in ((12e-6, 17e-6), (22e-6, 27e-6)):
        i = np.flatnonzero((xn >= x0 - tol) & (xn <= x1 + tol))
        j = np.flatnonzero((yn >= 10e-6 - tol) & (yn <= 12e-6 + tol))
        sig[i[0]:i[-1], j[0]:j[-1], :] = 5.8e7
    terms = [Terminal("s1", box(12e-6, 17e-6, 10e-6, 12e-6)),
             Terminal("s2", box(22e-6, 27e-6, 10e-6, 12e-6)),
             Terminal("gnd", box(0, 40e-6, 0, 0))]
    out = {"x": x, "y": y, "eps": eps, "sigma": sig}
    for i, t in enumerate(terms):
        out[f"term{i}"] = t.nodes
    for tag, kw in (("dc", {}), ("ghz", {"freq": 1e9}), ("name", {"reference": "gnd"}),
                    ("ref0", {"reference": 0})):
        r = rlgc_2d(g, eps, sig, terms, **kw)
        for k in ("R", "L", "G", "C", "C_air", "eps_eff", "Z0", "v_p"):
            out[f"{tag}_{k}"] = np.asarray(r[k])
        out[f"{tag}_reference"] = np.array(r["reference"])
    np.savez_compressed(HERE / "rlgc.npz", **out)


def ac_fixture():
    """solvers/ac.py:34-164: admittance matrices of a seeded three-terminal
    structure (graded grid; a lossy dielectric eps' - j eps'' over doped
    silicon, two copper pads) at four frequencies, the terminal currents of
    ``solve`` with complex drive values, and the complex Schur complement of
    the field region of ``field_region_fixture`` (``FieldRegion.stamp_ac``,
    coupling.py:214-236) at 1 GHz."""
    from fieldspice.circuit.coupling import FieldRegion
    from fieldspice.solvers.ac import ACSolver
    rng = np.random.default_rng(33)
    g = RectilinearGrid(np.sort(rng.uniform(0, 6e-6, 16)), np.sort(rng.uniform(0, 4e-6, 12)),
                        np.linspace(0, 2e-6, 10))
    eps = np.full(g.shape_cells, 3.9 * eps0, dtype=complex)
    eps[:, :, 4:] = (4.2 - 0.08j) * eps0           # lossy dielectric (tan d ~ 0.02)
    sig = np.zeros(g.shape_cells)
    sig[:, :, :3] = 10.0                            # doped silicon
    eps[:, :, :3] = 11.7 * eps0
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    boxes = [(2, 2, 6, 5, 5, 7), (9, 6, 6, 13, 9, 8), (0, 0, 0, 15, 11, 0)]
    terms = [Terminal(f"t{i}", nid[a0:a1 + 1, b0:b1 + 1, c0:c1 + 1].ravel())
             for i, (a0, b0, c0, a1, b1, c1) in enumerate(boxes)]
    # the pads are electrodes: no copper conductivity inside them, whose
    # 5.8e7 S/m edges would carry the LU's round-off on the fixed rows
    # (|phi - v| ~ 1e-16) into the terminal currents at the 1e-5 level
    freqs = np.array([1e3, 1e6, 1e9, 1e11])
    ac = ACSolver(g, eps, sig)
    out = {"x": g.xn, "y": g.yn, "z": g.zn, "eps": eps, "sigma": sig,
           "boxes": np.asarray(boxes), "freqs": freqs}
    out["Y"] = ac.admittance_matrix(terms, freqs)
    drive = [Terminal("t0", terms[0].nodes, voltage=1.0),
             Terminal("t1", terms[1].nodes, voltage=0.5),
             Terminal("t2", terms[2].nodes, voltage=0.0)]
    r = ac.solve(drive, freqs[1:])
    out["solve_i"] = np.array([r.terminals[t.name]["i"] for t in drive])
    out["solve_v"] = np.array([r.terminals[t.name]["v"] for t in drive])
    # the field region of field_region_fixture, small-signal at 1 GHz
    g2, eps2, sig2, boxes2, nid2 = field_region_geometry()
    t2 = [Terminal(f"e{i}", nid2[a0:a1 + 1, b0:b1 + 1, c0:c1 + 1].ravel())
          for i, (a0, b0, c0, a1, b1, c1) in enumerate(boxes2)]
    fr = FieldRegion("FR", g2, eps2, sig2, t2, circuit_nodes=["0", "a", "b"])
    Ym = np.zeros((2, 2), dtype=complex)
    fr.stamp_ac(Ym, np.zeros(2, dtype=complex), None, 2 * np.pi * 1e9, {"a": 0, "b": 1})
    out["fr_stamp_ac"] = Ym
    np.savez_compressed(HERE / "ac.npz", **out)


def floating_fixture():
    """poisson.py:967-1063 with the node-merging reduction (:665-719): a
    grounded-bottom layered box with a driven electrode, a floating conductor
    and a charge-driven conductor, plus free charge; potential, terminal
    voltages and charges."""
    rng = np.random.default_rng(41)
    g = RectilinearGrid(np.sort(rng.uniform(0, 3e-6, 14)), np.linspace(0, 2e-6, 11),
                        np.linspace(0, 1.5e-6, 9))
    eps = np.full(g.shape_cells, 3.9 * eps0)
    eps[:, :, :3] = 7.0 * eps0
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    boxes = [(2, 2, 4, 4, 4, 5), (7, 3, 3, 9, 6, 5), (10, 6, 5, 12, 8, 6)]
    nodes = [nid[a0:a1 + 1, b0:b1 + 1, c0:c1 + 1].ravel() for a0, b0, c0, a1, b1, c1 in boxes]
    terms = [Terminal("drv", nodes[0], voltage=1.0), Terminal("flt", nodes[1]),
             Terminal("chg", nodes[2], current=2e-17)]
    rho = np.zeros(g.shape_nodes)
    rho[5, 5, 6] = 1e3
    bc = BoundarySpec(zlo=Dirichlet(0.0))
    ps = PoissonSolver(g, eps, SolverConfig(linear_solver="direct", tol=1e-12))
    r = ps.solve(terms, bc, rho_node=rho)
    out = {"x": g.xn, "y": g.yn, "z": g.zn, "eps": eps, "boxes": np.asarray(boxes),
           "rho": rho, "phi": r.fields["phi"][0].ravel()}
    for t in terms:
        out[f"v_{t.name}"] = r.terminals[t.name]["v"]
        out[f"q_{t.name}"] = r.terminals[t.name]["q"]
    np.savez_compressed(HERE / "floating.npz", **out)


def floating_many_fixture():
    """The floating-electrode solve of floating_fixture with 20 floating and
    charge-driven conductors (a 5 x 4 array of small boxes, every third one
    charge-driven) and one driven electrode: more electrodes than one block
    of right-hand sides holds on the GPU path."""
    rng = np.random.default_rng(43)
    g = RectilinearGrid(np.linspace(0, 4e-6, 23), np.linspace(0, 3e-6, 19),
                        np.sort(rng.uniform(0, 1.2e-6, 10)))
    eps = np.full(g.shape_cells, 3.9 * eps0)
    eps[:, :, :3] = 11.7 * eps0
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    boxes = [(1, 1, 6, 3, 17, 7)]
    for a in range(5):
        for b in range(4):
            boxes.append((5 + 3 * a, 2 + 4 * b, 4, 6 + 3 * a, 3 + 4 * b, 5))
    nodes = [nid[a0:a1 + 1, b0:b1 + 1, c0:c1 + 1].ravel() for a0, b0, c0, a1, b1, c1 in boxes]
    terms = [Terminal("drv", nodes[0], voltage=1.0)]
    for i, nd in enumerate(nodes[1:]):
        terms.append(Terminal(f"c{i}", nd, current=1e-18 * (i - 9)) if i % 3 == 2
                     else Terminal(f"f{i}", nd))
    bc = BoundarySpec(zlo=Dirichlet(0.0))
    ps = PoissonSolver(g, eps, SolverConfig(linear_solver="direct", tol=1e-12))
    r = ps.solve(terms, bc)
    out = {"x": g.xn, "y": g.yn, "z": g.zn, "eps": eps, "boxes": np.asarray(boxes),
           "phi": r.fields["phi"][0].ravel(),
           "names": np.array([t.name for t in terms]),
           "v": np.array([r.terminals[t.name]["v"][0] for t in terms]),
           "q": np.array([r.terminals[t.name]["q"][0] for t in terms])}
    np.savez_compressed(HERE / "floating_many.npz", **out)


def periodic_fixture():
    """poisson.py:942-955, 1041-1058, 1196-1224 with Periodic walls: a layered
    unit cell periodic in x (and one periodic in x and y), grounded floor,
    three box electrodes (one crossing the x wrap); the capacitance matrix and
    a driven potential with free charge."""
    from fieldspice.boundaries import Periodic
    rng = np.random.default_rng(51)
    g = RectilinearGrid(np.linspace(0, 3e-6, 17), np.sort(rng.uniform(0, 2e-6, 11)),
                        np.linspace(0, 1e-6, 9))
    eps = np.full(g.shape_cells, 3.9 * eps0)
    eps[:, :, :3] = 7.0 * eps0
    eps[:, 6:, 5:] = 2.5 * eps0
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    boxes = [(3, 2, 4, 6, 5, 5), (9, 5, 3, 12, 8, 5)]
    terms = [Terminal(f"b{i}", nid[a0:a1 + 1, b0:b1 + 1, c0:c1 + 1].ravel())
             for i, (a0, b0, c0, a1, b1, c1) in enumerate(boxes)]
    # a strip across the x wrap: both boundary planes belong to it
    wrap = np.concatenate([nid[14:, 3:7, 6:8].ravel(), nid[:2, 3:7, 6:8].ravel()])
    terms.append(Terminal("wrap", wrap))
    cfg = SolverConfig(linear_solver="direct", tol=1e-12)
    out = {"x": g.xn, "y": g.yn, "z": g.zn, "eps": eps, "boxes": np.asarray(boxes),
           "wrap_nodes": wrap}
    for tag, walls in (("x", ("x",)), ("xy", ("x", "y"))):
        kw = {"zlo": Dirichlet(0.0)}
        for a in walls:
            kw[f"{a}lo"] = Periodic()
            kw[f"{a}hi"] = Periodic()
        bc = BoundarySpec(**kw)
        ps = PoissonSolver(g, eps, cfg)
        out[f"C_{tag}"] = ps.capacitance_matrix(terms, bc)
        drive = [Terminal(t.name, t.nodes, voltage=v) for t, v in zip(terms, (1.0, -0.5, 0.25))]
        rho = np.zeros(g.shape_nodes)
        rho[7, 7, 6] = 2e3
        r = ps.solve(drive, bc, rho_node=rho)
        out[f"phi_{tag}"] = r.fields["phi"][0].ravel()
        out[f"q_{tag}"] = np.array([r.terminals[t.name]["q"][0] for t in drive])
        out["rho"] = rho
    np.savez_compressed(HERE / "periodic.npz", **out)


def neumann_fixture():
    """boundaries.py:1031-1085 and poisson.py:957-964: a driven Neumann flux
    on two walls (a constant D.n on xhi, a time-dependent one on yhi)
    feeding PoissonSolver.solve, with a grounded floor and one driven box;
    direct solve.  Records the reference's load vector and the solution."""
    from fieldspice.boundaries import Neumann
    rng = np.random.default_rng(61)
    g = RectilinearGrid(np.sort(rng.uniform(0, 3e-6, 15)), np.linspace(0, 2e-6, 11),
                        np.linspace(0, 1e-6, 9))
    eps = rng.uniform(2.5, 7.0, g.shape_cells) * eps0
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    box = Terminal("box", nid[4:8, 3:6, 4:6].ravel(), voltage=0.7)

    def ramp_flux(t):
        return 2e-4 * (1.0 + t * 1e9)
    bc = BoundarySpec(zlo=Dirichlet(0.0), xhi=Neumann(flux=-3e-4), yhi=Neumann(flux=ramp_flux))
    t = 0.5e-9
    ps = PoissonSolver(g, eps, SolverConfig(linear_solver="direct"))
    r = ps.solve([box], bc, t=t)
    out = {"x": g.xn, "y": g.yn, "z": g.zn, "eps": eps, "t": t,
           "load": bc.neumann_load(g, t), "phi": r.fields["phi"][0].ravel(),
           "q_box": r.terminals["box"]["q"], "energy": r.scalars["energy"]}
    np.savez_compressed(HERE / "neumann.npz", **out)


def rc_stack(n=60):
    d, Wd, H = 4e-6, 3e-6, 2e-6
    sigma1, er1, er2 = 1e3, 4.0, 2.0
    g = RectilinearGrid(np.linspace(0, d, n + 1), np.linspace(0, Wd, 4),
                        np.linspace(0, H, 3))
    left = g.xc < d / 2
    sig = np.zeros(g.shape_cells)
    sig[left] = sigma1
    eps = np.empty(g.shape_cells)
    eps[left] = er1 * eps0
    eps[~left] = er2 * eps0
    return g, eps, sig


def eqs_fixture():
    # the RC stack of tests/test_quasistatic.py:24-59, direct path
    g, eps, sig = rc_stack()
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    out = {"xn": g.xn, "yn": g.yn, "zn": g.zn, "eps": eps, "sig": sig}
    from fieldspice import reference as ref
    A = 3e-6 * 2e-6
    R1 = 2e-6 / (1e3 * A)
    C1 = ref.parallel_plate_capacitance(A, 2e-6, 4.0)
    C2 = ref.parallel_plate_capacitance(A, 2e-6, 2.0)
    tau = R1 * (C1 + C2)
    out["tau"] = tau
    for spt in (50, 100):
        s = EQSSolver(g, eps, sig, SolverConfig(verbose=0))
        hi = Terminal("hi", nid[0].ravel(), voltage=1.0)
        lo = Terminal("lo", nid[-1].ravel(), voltage=0.0)
        r = s.solve([hi, lo], t_end=8 * tau, dt=tau / spt, store=True)
        out[f"spt{spt}_i_hi"] = r.i("hi")
        out[f"spt{spt}_i_lo"] = r.i("lo")
        out[f"spt{spt}_vm"] = r.fields["phi"][:, nid[30, 1, 1]]
        out[f"spt{spt}_t"] = r.scalars["t_stored"]
        out[f"spt{spt}_energy"] = r.scalars["energy_electric"]
    # a small interconnect transient (CG path, Jacobi forced, tight tol)
    w = W.eqs_interconnect((24, 24, 16), nbox=3, nports=2, seed=3, si_cells=4)
    g2 = RectilinearGrid(w.x, w.y, w.z)
    ramp = W.ramp(0.0, 0.0, 1.0, 10e-12)
    terms = [Terminal("port0", w.terminals[0], voltage=ramp),
             Terminal("port1", w.terminals[1], voltage=0.0)]
    with jacobi_forced():
        s2 = EQSSolver(g2, w.eps_cell, w.sigma_cell,
                       SolverConfig(linear_solver="cg", tol=1e-12))
        r2 = s2.solve(terms, t_end=20e-12, dt=1e-12,
                      bc=BoundarySpec(zlo=Dirichlet(0.0)), store=True)
    out.update({"ic_x": w.x, "ic_y": w.y, "ic_z": w.z, "ic_eps": w.eps_cell,
                "ic_sig": w.sigma_cell, "ic_boxes": np.asarray(w.boxes),
                "ic_i0": r2.i("port0"), "ic_i1": r2.i("port1"),
                "ic_v0": r2.v("port0"), "ic_phi_last": r2.fields["phi"][-1],
                "ic_energy": r2.scalars["energy_electric"],
                "ic_dissipation": r2.scalars["dissipation"]})
    np.savez_compressed(HERE / "eqs.npz", **out)


def closed_forms():
    # tests/test_core.py:236-297: series stack and graded plate, direct solves
    from fieldspice import reference as ref
    out = {}
    er1, er2, d, Wd, H = 4.0, 2.0, 4e-6, 3e-6, 2e-6
    g = RectilinearGrid(np.linspace(0, d, 41), np.linspace(0, Wd, 5), np.linspace(0, H, 4))
    e = np.empty(g.shape_cells)
    left = g.xc < d / 2
    e[left] = er1 * eps0
    e[~left] = er2 * eps0
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    C = PoissonSolver(g, e).capacitance_matrix(
        [Terminal("lo", nid[0].ravel()), Terminal("hi", nid[-1].ravel())])
    out["series_C"] = C
    C1 = ref.parallel_plate_capacitance(Wd * H, d / 2, er1)
    C2 = ref.parallel_plate_capacitance(Wd * H, d / 2, er2)
    out["series_ref"] = C1 * C2 / (C1 + C2)
    x = graded_1d(0, 2e-6, 30, 1.25)
    g = RectilinearGrid(x, graded_1d(0, 5e-6, 9, 0.85), np.linspace(0, 4e-6, 7))
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    C = PoissonSolver(g, np.full(g.shape_cells, 3.9 * eps0)).capacitance_matrix(
        [Terminal("lo", nid[0].ravel()), Terminal("hi", nid[-1].ravel())])
    out["graded_C"] = C
    out["graded_xn"], out["graded_yn"], out["graded_zn"] = g.xn, g.yn, g.zn
    out["graded_ref"] = ref.parallel_plate_capacitance(20e-12, 2e-6, 3.9)
    np.savez_compressed(HERE / "closed_forms.npz", **out)


FIXTURES = {
    "masses": masses_fixture,
    "readme": readme_fixture,
    "closed_forms": closed_forms,
    "layered": lambda: (layered_fixture((32, 32, 16), 0, 1e-12),
                        layered_fixture((48, 48, 24), 1, 1e-12)),
    "eqs": eqs_fixture,
    "resistance": resistance_fixture,
    "thermal": thermal_fixture,
    "field_region": field_region_fixture,
    "rlgc": rlgc_fixture,
    "ac": ac_fixture,
    "floating": floating_fixture,
    "periodic": periodic_fixture,
    "neumann": neumann_fixture,
    "floating_many": floating_many_fixture,
}

if __name__ == "__main__":
    # with names on the command line only those fixtures are regenerated
    for name in (sys.argv[1:] or list(FIXTURES)):
        FIXTURES[name]()
    print("golden fixtures written to", HERE)
