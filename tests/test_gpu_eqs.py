"""GPU electroquasistatic transient against the reference's results.

The RC stack of the reference's ``tests/test_quasistatic.py:24-112`` (lossy
left half, insulating right half) and a seeded copper/oxide/silicon
interconnect driven by a 10 ps ramp, recorded from the reference in
``tests/golden/eqs.npz``.  Tolerances: the reference's own (IC divider 1e-9,
analytic RC 2e-4, first-order ratios 1.8-2.2, current conservation 1e-8,
slab resistance 1e-9); recorded currents to 1e-7 of their peak.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

EPS0 = 8.8541878128e-12


def _rc_stack(n=60):
    from fieldspice_b200.grid import RectilinearGrid
    from oracle import fs_oracle as O
    d, W, H = 4e-6, 3e-6, 2e-6
    sigma1, er1, er2 = 1e3, 4.0, 2.0
    g = RectilinearGrid(np.linspace(0, d, n + 1), np.linspace(0, W, 4), np.linspace(0, H, 3))
    left = g.xc < d / 2
    sig = np.zeros(g.shape_cells)
    sig[left] = sigma1
    eps = np.empty(g.shape_cells)
    eps[left] = er1 * O.EPS0
    eps[~left] = er2 * O.EPS0
    A = W * H
    R1 = (d / 2) / (sigma1 * A)
    C1 = er1 * O.EPS0 * A / (d / 2)
    C2 = er2 * O.EPS0 * A / (d / 2)
    return g, eps, sig, R1, C1, C2, n


def _run(steps_per_tau, tol=1e-12, precision="mixed"):
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig, Terminal
    from fieldspice_b200.solvers.eqs import EQSSolver
    g, eps, sig, R1, C1, C2, n = _rc_stack()
    tau = R1 * (C1 + C2)
    v0 = C1 / (C1 + C2)
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    s = EQSSolver(g, eps, sig, SolverConfig(tol=tol), gpu=GPUConfig(precision=precision))
    hi = Terminal("hi", nid[0].ravel(), voltage=1.0)
    lo = Terminal("lo", nid[-1].ravel(), voltage=0.0)
    r = s.solve([hi, lo], t_end=8 * tau, dt=tau / steps_per_tau, store=True)
    vm = r.fields["phi"][:, nid[n // 2, 1, 1]]
    ts = r.scalars["t_stored"]
    ana = 1.0 - (1.0 - v0) * np.exp(-ts / (R1 * (C1 + C2)))
    return r, vm, ana, tau, v0


def test_initial_condition_is_the_capacitive_divider(cuda):
    _, vm, _, _, v0 = _run(50)
    assert v0 == pytest.approx(2.0 / 3.0, rel=1e-12)
    assert vm[0] == pytest.approx(v0, rel=1e-9)


def test_matches_reference_rc_transient(cuda, golden):
    # the reference factorises this small system (exact solve); the GPU
    # iterates to relres 1e-13 so that 400 steps of accumulated solver error
    # stay inside 1e-9 V
    d = golden("eqs")
    r, vm, ana, _, _ = _run(50, tol=1e-13)
    assert np.abs(vm - d["spt50_vm"]).max() < 1e-9
    scale = np.abs(d["spt50_i_hi"]).max()
    assert np.abs(r.i("hi") - d["spt50_i_hi"]).max() / scale < 1e-7
    assert np.abs(r.i("lo") - d["spt50_i_lo"]).max() / scale < 1e-7
    e = d["spt50_energy"]
    assert np.abs(r.scalars["energy_electric"] - e).max() / np.abs(e).max() < 1e-8
    assert r.meta["n_factorisations"] == 1


def test_backward_euler_is_first_order_and_matches_analytic(cuda):
    errs = [np.abs(v - a).max() for _, v, a, _, _ in (_run(s) for s in (50, 100, 200, 400))]
    assert errs[0] == pytest.approx(1.216e-3, rel=0.05)
    assert errs[-1] < 2e-4
    for lo, hi in zip(errs[:-1], errs[1:]):
        assert 1.8 < lo / hi < 2.2


@pytest.mark.parametrize("precision", ["auto", "fp64"])
def test_terminal_currents_conserve(cuda, precision):
    # The imbalance equals the summed free-node residual, so it tracks the
    # CG tolerance (the reference factorises this case directly): with the
    # step's right-hand side ~1e5 x the current, tol 1e-14 keeps it < 1e-8.
    r, *_ = _run(100, tol=1e-14, precision=precision)
    total = r.i("hi") + r.i("lo")
    scale = max(np.abs(r.i("hi")).max(), 1e-30)
    assert np.abs(total).max() / scale < 1e-8


@pytest.mark.parametrize("preconditioner", ["mg", "jacobi"])
@pytest.mark.parametrize("precision", ["auto", "fp64"])
def test_interconnect_ramp_matches_reference(cuda, golden, precision, preconditioner):
    """Copper next to oxide: the floating copper box is an eigenvalue of
    1.5e-7 of the equilibrated operator, below FP32 resolution, so "auto"
    must notice the stall and finish in FP64."""
    from fieldspice_b200 import workloads as W
    from fieldspice_b200.boundaries import BoundarySpec, Dirichlet
    from fieldspice_b200.grid import RectilinearGrid
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig, Terminal
    from fieldspice_b200.solvers.eqs import EQSSolver
    d = golden("eqs")
    g = RectilinearGrid(d["ic_x"], d["ic_y"], d["ic_z"])
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    ports = [nid[a0:a1 + 1, b0:b1 + 1, c0:c1 + 1].ravel()
             for a0, b0, c0, a1, b1, c1 in d["ic_boxes"][:2]]
    ramp = W.ramp(0.0, 0.0, 1.0, 10e-12)
    terms = [Terminal("port0", ports[0], voltage=ramp), Terminal("port1", ports[1], voltage=0.0)]
    s = EQSSolver(g, d["ic_eps"], d["ic_sig"], SolverConfig(tol=1e-12),
                  gpu=GPUConfig(precision=precision, preconditioner=preconditioner))
    r = s.solve(terms, t_end=20e-12, dt=1e-12, bc=BoundarySpec(zlo=Dirichlet(0.0)), store=True)
    scale = np.abs(d["ic_i0"]).max()
    assert np.abs(r.i("port0") - d["ic_i0"]).max() / scale < 1e-7
    assert np.abs(r.i("port1") - d["ic_i1"]).max() / scale < 1e-7
    assert np.abs(r.v("port0") - d["ic_v0"]).max() < 1e-12
    assert np.abs(r.fields["phi"][-1] - d["ic_phi_last"]).max() < 1e-9
    en = d["ic_energy"]
    assert np.abs(r.scalars["energy_electric"] - en).max() / np.abs(en).max() < 1e-8
    di = d["ic_dissipation"]
    assert np.abs(r.scalars["dissipation"] - di).max() / np.abs(di).max() < 1e-6


def test_steady_state_is_the_resistive_solution(cuda):
    from fieldspice_b200.grid import RectilinearGrid
    from fieldspice_b200.solvers.base import Terminal
    from fieldspice_b200.solvers.eqs import EQSSolver
    d, W, H, sigma = 2e-6, 5e-6, 4e-6, 1e4
    g = RectilinearGrid(np.linspace(0, d, 16), np.linspace(0, W, 6), np.linspace(0, H, 5))
    s = EQSSolver(g, np.full(g.shape_cells, 3.9 * EPS0), np.full(g.shape_cells, sigma))
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    hi = Terminal("hi", nid[0].ravel(), voltage=1.0)
    lo = Terminal("lo", nid[-1].ravel(), voltage=0.0)
    r = s.steady_state([hi, lo])
    R = 1.0 / abs(float(r.i("hi")[0]))
    assert R == pytest.approx(d / (sigma * W * H), rel=1e-9)


def test_rejects_bad_materials(cuda):
    from fieldspice_b200.grid import RectilinearGrid
    from fieldspice_b200.solvers.eqs import EQSSolver
    g = RectilinearGrid.uniform([(0, 1e-6), (0, 1e-6)], [4, 4])
    with pytest.raises(ValueError):
        EQSSolver(g, np.full(g.shape_cells, 3.9), np.zeros(g.shape_cells))
    with pytest.raises(ValueError):
        EQSSolver(g, np.full(g.shape_cells, EPS0), np.full(g.shape_cells, -1.0))


@pytest.mark.parametrize("coarsening", ["auto", "geometric"])
def test_interconnect_transient_at_scale_matches_reference(cuda, coarsening):
    """The copper/oxide/doped-silicon interconnect (two ports, a 1 V ramp of
    10 ps on port 0, dt 1 ps, 200 steps) at the largest grid the reference
    itself finished here (tests/golden/eqs_<shape>_s0.npz, made by
    tests/golden/make_scale.py: the reference's EQSSolver, Jacobi-CG forced,
    tol 1e-12).  Port currents at every step to 1e-7 of their peak."""
    from pathlib import Path

    from fieldspice_b200 import workloads as W
    from fieldspice_b200.boundaries import BoundarySpec, Dirichlet
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig, Terminal
    from fieldspice_b200.solvers.eqs import EQSSolver
    fx = sorted((Path(__file__).parent / "golden").glob("eqs_*x*x*_s0.npz"),
                key=lambda p: int(np.prod(np.load(p)["shape"])))
    d = np.load(fx[-1])
    shape = tuple(int(v) for v in d["shape"])
    steps = int(d["steps"])
    w = W.eqs_interconnect(shape, nbox=6, nports=2, seed=0)
    ramp = W.ramp(0.0, 0.0, 1.0, 10e-12)
    terms = [Terminal("port0", w.terminals[0], voltage=ramp),
             Terminal("port1", w.terminals[1], voltage=0.0)]
    s = EQSSolver(w.grid(), w.eps_cell, w.sigma_cell, SolverConfig(tol=1e-12),
                  gpu=GPUConfig(preconditioner="mg", coarsening=coarsening))
    r = s.solve(terms, t_end=steps * 1e-12, dt=1e-12, bc=BoundarySpec(zlo=Dirichlet(0.0)))
    if coarsening == "auto":
        assert r.meta["coarsening"] == "galerkin"
    scale = max(np.abs(d["i0"]).max(), np.abs(d["i1"]).max())
    assert np.abs(r.i("port0") - d["i0"]).max() / scale < 1e-7
    assert np.abs(r.i("port1") - d["i1"]).max() / scale < 1e-7


class _ProbeSet:
    """A monitor set in the reference's protocol (``record(state, t)``,
    ``finalize()``, ``monitors.py:1607-1720``): the potential at one node and
    the state keys the solver hands over."""

    def __init__(self, node, fail_at=None):
        self.node, self.fail_at = node, fail_at
        self.t, self.v, self.keys = [], [], set()

    def record(self, state, t):
        self.keys |= set(state)
        if self.fail_at is not None and len(self.t) == self.fail_at:
            self.t.append(t)
            raise RuntimeError("a monitor that fails once")
        self.t.append(t)
        self.v.append(float(state["phi"][self.node]))

    def finalize(self):
        return {"t": np.asarray(self.t), "v": np.asarray(self.v)}


def test_monitors_see_every_step(cuda, golden):
    """A monitor set receives the potential at t0 and after every step
    (``eqs.py:287-319``, ``:377-386``), equal to the stored fields; its
    result lands in ``meta["monitors"]``; a monitor that raises does not end
    the solve."""
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig, Terminal
    from fieldspice_b200.solvers.eqs import EQSSolver
    d = golden("eqs")
    g, eps, sig, R1, C1, C2, n = _rc_stack()
    tau = R1 * (C1 + C2)
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    probe = _ProbeSet(int(nid[n // 2, 1, 1]))
    s = EQSSolver(g, eps, sig, SolverConfig(tol=1e-12), gpu=GPUConfig(precision="mixed"))
    hi = Terminal("hi", nid[0].ravel(), voltage=1.0)
    lo = Terminal("lo", nid[-1].ravel(), voltage=0.0)
    r = s.solve([hi, lo], t_end=8 * tau, dt=tau / 50, monitors=probe, store=True)
    m = r.meta["monitors"]
    assert np.allclose(m["t"], r.t, rtol=0, atol=1e-30)
    assert np.array_equal(m["v"], r.fields["phi"][:, probe.node])
    assert np.abs(m["v"] - d["spt50_vm"]).max() < 2e-9
    assert {"phi", "grid", "ops", "eps_edge", "sigma_edge", "step", "dt"} <= probe.keys
    bad = _ProbeSet(int(nid[n // 2, 1, 1]), fail_at=3)
    r2 = s.solve([hi, lo], t_end=8 * tau, dt=tau / 50, monitors=bad)
    assert len(bad.t) == len(r2.t) and len(bad.v) == len(r2.t) - 1
