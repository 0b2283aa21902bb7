"""GPU parity of the edge masses and the stencil apply (needs a B200).

The masses are compared BIT-FOR-BIT with the reference's
``edge_mass(cell_to_edge(...))`` recorded in ``tests/golden/masses.npz``;
the FP64 stencil with the reference's CSR ``L @ x`` to FP64 round-off
(relative 1e-14 of max|L x|), the FP32 stencil to FP32 round-off (1e-5).
"""

import ctypes

import numpy as np
import pytest

from oracle import fs_oracle as O

pytestmark = pytest.mark.gpu

GRIDS = ("graded", "uniform", "collapsed", "wide")


def _grid(d, name):
    from fieldspice_b200.grid import RectilinearGrid
    return RectilinearGrid(d[f"{name}_xn"], d[f"{name}_yn"], d[f"{name}_zn"])


@pytest.mark.parametrize("name", GRIDS)
@pytest.mark.parametrize("mode", ["parallel", "harmonic"])
def test_masses_bit_exact_vs_reference(cuda, golden, name, mode):
    from fieldspice_b200.device import DeviceOperator
    d = golden("masses")
    g = _grid(d, name)
    op = DeviceOperator(g, d[f"{name}_prop"], mode=mode)
    got = op.edge_vector()
    want = d[f"{name}_mass_{mode}"]
    assert got.shape == want.shape
    assert np.array_equal(got, want), np.abs(got - want).max()


@pytest.mark.parametrize("name", GRIDS)
def test_fp64_apply_matches_reference_csr(cuda, golden, name):
    import torch
    from fieldspice_b200.device import DeviceOperator
    d = golden("masses")
    g = _grid(d, name)
    op = DeviceOperator(g, d[f"{name}_prop"])
    x = d[f"{name}_x"]                      # (n_nodes, 3)
    y = np.zeros_like(x)
    for c in range(3):
        xd = torch.as_tensor(np.ascontiguousarray(x[:, c]), device=cuda)
        y[:, c] = op.apply(xd).cpu().numpy()
    want = d[f"{name}_Lx"]
    assert np.abs(y - want).max() <= 1e-14 * np.abs(want).max()


@pytest.mark.parametrize("k", [1, 2, 4, 8, 16])
@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_stencil_apply_masked_multi_rhs(cuda, k, dtype):
    """fs_stencil_apply with a Dirichlet label equals the eliminated CSR
    operator of operators.py:362-407 restricted to the free rows."""
    import torch
    from fieldspice_b200 import _lib as L
    from fieldspice_b200.device import DeviceOperator
    rng = np.random.default_rng(k)
    w_shape = (13, 11, 9)
    from fieldspice_b200.grid import RectilinearGrid
    g = RectilinearGrid(*[np.sort(rng.uniform(0, 1e-6, n)) for n in w_shape])
    eps = rng.uniform(1, 10, g.shape_cells) * O.EPS0
    op = DeviceOperator(g, eps)
    og = O.Grid(g.xn, g.yn, g.zn)
    m = O.edge_mass_vector(og, O.cell_to_edge(og, eps))
    Lm = O.nodal_laplacian(og, m)
    N = g.n_nodes
    fixed = rng.random(N) < 0.2
    A, _ = O.apply_dirichlet(Lm, np.zeros(N), fixed, 0.0)
    x = rng.standard_normal((N, k))
    x[fixed] = 0.0
    want = A @ x
    want[fixed] = 0.0
    tdt = torch.float64 if dtype == "f64" else torch.float32
    xd = torch.as_tensor(x, dtype=tdt, device=cuda).contiguous()
    yd = torch.empty_like(xd)
    md = op.m.to(tdt)
    lab = torch.as_tensor(fixed.astype(np.uint8), device=cuda)
    st = L.lib().fs_stencil_apply(L.ptr(xd), L.ptr(yd), L.ptr(md[0]), L.ptr(md[1]),
                                  L.ptr(md[2]), L.ptr(lab), *g.shape_nodes, k,
                                  L.DTYPE_F64 if dtype == "f64" else L.DTYPE_F32,
                                  L.stream_ptr())
    L.check("fs_stencil_apply", st)
    got = yd.cpu().double().numpy()
    tol = 1e-14 if dtype == "f64" else 2e-6
    assert np.abs(got - want).max() <= tol * np.abs(want).max()


def test_quadform_and_group_sums(cuda, golden):
    import torch
    from fieldspice_b200.device import DeviceOperator
    d = golden("masses")
    g = _grid(d, "graded")
    op = DeviceOperator(g, d["graded_prop"])
    og = O.Grid(g.xn, g.yn, g.zn)
    Lm = O.nodal_laplacian(og, d["graded_mass_parallel"])
    x = d["graded_x"][:, :2].copy()
    xd = torch.as_tensor(x, device=cuda).contiguous()
    q = op.quadform(xd.view(-1), nrhs=2)
    want = np.einsum("nk,nk->k", x, Lm @ x)
    assert np.allclose(q, want, rtol=1e-12, atol=0)
    groups = [np.arange(0, 40), np.arange(100, 180), np.array([5, 7, 230])]
    s = op.group_sums(xd.view(-1), groups, nrhs=2)
    y = Lm @ x
    for gi, gr in enumerate(groups):
        assert np.allclose(s[gi], y[gr].sum(axis=0), rtol=1e-12, atol=1e-12 * np.abs(y).max())


def test_grid_metric_cache_reuses_and_refreshes(cuda, golden):
    """The device copy of a grid's metric is reused while the grid's values
    are unchanged and uploaded again (with the masses following) once they
    change in place."""
    from fieldspice_b200.device import DeviceOperator, metric_dev
    d = golden("masses")
    g = _grid(d, "graded")
    dev = DeviceOperator(g, np.full(g.shape_cells, 1e-11)).dev
    a = metric_dev(g, dev)
    assert all(x is y for x, y in zip(a, metric_dev(g, dev)))
    m0 = DeviceOperator(g, np.full(g.shape_cells, 1e-11)).m.cpu().numpy()
    g.hx[0] *= 2.0  # changed in place: a new upload, and masses that follow it
    b = metric_dev(g, dev)
    assert b[0] is not a[0]
    assert float(b[0][0]) == float(g.hx[0])
    m1 = DeviceOperator(g, np.full(g.shape_cells, 1e-11)).m.cpu().numpy()
    assert not np.array_equal(m0, m1)
