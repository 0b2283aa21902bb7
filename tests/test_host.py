"""Host-side logic of the drop-in boundary (CPU only)."""

import numpy as np
import pytest

from fieldspice_b200 import boundaries as B
from fieldspice_b200 import workloads as W
from fieldspice_b200.grid import RectilinearGrid, axis_metric
from fieldspice_b200.solvers.base import SolverConfig, Terminal
from fieldspice_b200.solvers.poisson import (as_cell_array, check_terminals,
                                             prepare_bc, raise_on_status)
from oracle import fs_oracle as O


def test_grid_metric_matches_oracle(golden):
    d = golden("masses")
    for name in ("graded", "uniform", "collapsed", "wide"):
        g = RectilinearGrid(d[f"{name}_xn"], d[f"{name}_yn"], d[f"{name}_zn"])
        o = O.Grid(d[f"{name}_xn"], d[f"{name}_yn"], d[f"{name}_zn"])
        for a, b in ((g.hx, o.hx), (g.hyd, o.hyd), (g.hzd, o.hzd)):
            assert np.array_equal(a, b)
        assert g.shape_nodes == o.shape_nodes
        assert np.array_equal(g.node_volumes(), o.node_volumes())


def test_collapsed_axis_has_two_node_planes():
    g = RectilinearGrid(np.linspace(0, 1, 137))
    assert g.shape_nodes == (137, 2, 2)
    h, hd = axis_metric([0.0, 1.0])
    assert np.array_equal(hd, [0.5, 0.5])


def test_wall_nodes_and_precedence():
    g = RectilinearGrid.uniform([(0, 1), (0, 2), (0, 3)], [4, 5, 6])
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    for wall, sl in (("xlo", nid[0]), ("xhi", nid[-1]), ("ylo", nid[:, 0]),
                     ("yhi", nid[:, -1]), ("zlo", nid[:, :, 0]), ("zhi", nid[:, :, -1])):
        assert np.array_equal(np.sort(B.wall_nodes(g, wall)), np.sort(sl.ravel()))
        assert np.array_equal(B.wall_nodes(g, wall), O.wall_nodes(O.Grid(g.xn, g.yn, g.zn), wall))
    spec = B.BoundarySpec(xlo=B.Dirichlet(1.0), zlo=B.Dirichlet(2.0))
    idx, val = B.dirichlet_nodes(spec, g)
    # the shared x=0, z=0 edge belongs to the later wall (zlo)
    shared = nid[0, :, 0]
    pos = np.searchsorted(idx, shared)
    assert np.all(val[pos] == 2.0)
    assert np.all(np.diff(idx) > 0)


def test_unsupported_walls_raise():
    @__import__("dataclasses").dataclass(frozen=True)
    class Periodic:
        is_dirichlet_like = False
        is_natural = False
    spec = B.BoundarySpec(xlo=Periodic(), xhi=Periodic())
    with pytest.raises(NotImplementedError):
        B.check_supported(spec)
    # a driven Neumann flux is supported (a right-hand-side load)
    B.check_supported(B.BoundarySpec(xlo=B.Neumann(flux=3.0)))
    B.check_supported(B.BoundarySpec(zlo=B.Dirichlet(0.0)))

    @__import__("dataclasses").dataclass(frozen=True)
    class Absorbing:
        is_dirichlet_like = False
        is_natural = False
    with pytest.raises(NotImplementedError):
        B.check_supported(B.BoundarySpec(xlo=Absorbing()))


def test_terminal_checks():
    g = RectilinearGrid.uniform([(0, 1), (0, 1), (0, 1)], [3, 3, 3])
    a = Terminal("a", [0, 1, 2])
    b = Terminal("b", [2, 3])
    with pytest.raises(ValueError, match="share node 2"):
        check_terminals([a, b], g)
    with pytest.raises(ValueError, match="bare Terminal"):
        check_terminals(a, g)
    with pytest.raises(ValueError, match="no nodes"):
        check_terminals([Terminal("e", [])], g)
    with pytest.raises(ValueError, match="outside"):
        check_terminals([Terminal("o", [10_000])], g)
    with pytest.raises(ValueError, match="duplicate"):
        check_terminals([Terminal("a", [0]), Terminal("a", [5])], g)
    assert Terminal("u", [3, 1, 3, 2]).nodes.tolist() == [1, 2, 3]
    with pytest.raises(ValueError):
        Terminal("x", [0], voltage=1.0, current=1.0)


def test_cell_array_checks():
    g = RectilinearGrid.uniform([(0, 1), (0, 1), (0, 1)], [3, 3, 3])
    with pytest.raises(ValueError, match="shape"):
        as_cell_array(np.ones((2, 2, 2)), g, "eps_cell")
    bad = np.ones(g.shape_cells)
    bad[0, 0, 0] = np.nan
    with pytest.raises(ValueError, match="non-finite"):
        as_cell_array(bad, g, "eps_cell")
    assert as_cell_array(2.0, g, "eps").shape == g.shape_cells


def test_status_mapping():
    from fieldspice_b200.solvers.base import ConvergenceError
    ok = {"status": 0, "relres": 5e-11, "iterations": 10}
    raise_on_status([ok], 1e-10, "cg")
    with pytest.raises(ConvergenceError):
        raise_on_status([{"status": 1, "relres": 1e-3, "iterations": 1}], 1e-10, "cg")
    with pytest.raises(ConvergenceError, match="NaN"):
        raise_on_status([{"status": 4, "relres": float("nan"), "iterations": 3}], 1e-10, "cg")
    with pytest.warns(RuntimeWarning):
        raise_on_status([{"status": 1, "relres": 1e-8, "iterations": 9}], 1e-10, "cg")


def test_workloads_are_deterministic_and_valid():
    a = W.layered_boxes((64, 64, 32), seed=5)
    b = W.layered_boxes((64, 64, 32), seed=5)
    assert a.boxes == b.boxes and np.array_equal(a.eps_cell, b.eps_cell)
    g = a.grid()
    check_terminals(a.terminal_objects(), g)          # disjoint, in range
    for (x0, y0, z0, x1, y1, z1) in a.boxes:
        assert z0 >= 1                                 # never on the grounded plane
    full = W.layered_boxes()
    assert full.shape_nodes == (256, 256, 128) and len(full.terminals) == 8
    z1, z2 = full.meta["z_interfaces"]
    assert z1 >= 8 and z2 - z1 >= 8 and 127 - z2 >= 8
    batch = W.batch_geometries(count=64, seed=0)
    assert len(batch) == 64
    assert all(2 <= len(w.terminals) <= 16 for w in batch)
    n = [w.n_nodes for w in batch]
    assert min(n) >= 24 ** 3 * 0.8 and max(n) <= 160 * 160 * 96 * 1.05


def test_prepare_bc_defaults_to_neumann():
    g = RectilinearGrid.uniform([(0, 1), (0, 1), (0, 1)], [3, 3, 3])
    bc = prepare_bc(None, g)
    idx, _ = B.dirichlet_nodes(bc, g)
    assert idx.size == 0


def test_solver_config_defaults_match_reference():
    c = SolverConfig()
    assert c.tol == 1e-10 and c.linear_solver == "auto"


def test_preconditioner_follows_linear_solver():
    from fieldspice_b200.solvers.base import GPUConfig, resolve_preconditioner
    assert resolve_preconditioner(SolverConfig(linear_solver="cg"), None) == "jacobi"
    for ls in ("auto", "amg", "direct"):
        assert resolve_preconditioner(SolverConfig(linear_solver=ls), None) == "mg"
    assert resolve_preconditioner(SolverConfig(linear_solver="cg"),
                                  GPUConfig(preconditioner="mg")) == "mg"
    with pytest.raises(ValueError):
        resolve_preconditioner(SolverConfig(linear_solver="lu"), None)


def test_metric_cache_hits_and_refreshes(monkeypatch):
    """metric_dev: one upload per grid while its values are unchanged, a new
    upload after an in-place change or for another device (uploads counted
    through a stand-in for the device copy)."""
    import torch
    from fieldspice_b200 import device as D
    calls = []

    def fake_h2d(a, dtype, dev):
        calls.append(dev)
        return torch.as_tensor(np.array(a, copy=True), dtype=dtype)

    monkeypatch.setattr(D, "h2d", fake_h2d)
    g = RectilinearGrid(np.linspace(0, 1, 6), np.linspace(0, 2, 5), np.linspace(0, 3, 4))
    a = D.metric_dev(g, "dev0")
    assert len(calls) == 6 and float(a[0][0]) == float(g.hx[0])
    b = D.metric_dev(g, "dev0")
    assert len(calls) == 6 and all(x is y for x, y in zip(a, b))
    g.hx[1] *= 3.0
    c = D.metric_dev(g, "dev0")
    assert len(calls) == 12 and float(c[0][1]) == float(g.hx[1])
    D.metric_dev(g, "dev1")
    assert len(calls) == 18
    g2 = RectilinearGrid(np.linspace(0, 1, 6), np.linspace(0, 2, 5), np.linspace(0, 3, 4))
    D.metric_dev(g2, "dev1")
    assert len(calls) == 24  # another grid object: its own entry
