"""The allocation-free charge integration matches the allocating one.

``fs_group_apply_noalloc`` serves callers that cannot let the library
allocate device memory (a host binding that owns every device buffer in its
own pool, or a stepping loop that must not stall on an allocation): its
scratch is a static array inside the library instead of a caller workspace.
This test calls both entry points through the C ABI on the same inputs and
requires the same per-terminal sums on two calls in a row, since the static
array keeps the previous call's contents; the sums are also checked against
the CPU oracle's assembled ``L_A u - L_B w`` summed over each node group.  It
sits in a file collected last.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(dev, k, seed):
    import torch
    from fieldspice_b200.device import DeviceOperator
    from fieldspice_b200.grid import RectilinearGrid
    rng = np.random.default_rng(seed)
    g = RectilinearGrid(*[np.sort(rng.uniform(0, 1e-6, n)) for n in (21, 17, 13)])
    propA = rng.uniform(1, 12, g.shape_cells) * 8.854e-12
    propB = rng.uniform(0, 5, g.shape_cells)
    opA = DeviceOperator(g, propA)
    opB = DeviceOperator(g, propB)
    N = g.n_nodes
    u = torch.as_tensor(rng.standard_normal(N * k), device=dev)
    w = torch.as_tensor(rng.standard_normal(N * k), device=dev)
    perm = rng.permutation(N)
    cuts = np.sort(rng.choice(np.arange(1, 900), 6, replace=False))
    groups = [np.sort(c) for c in np.split(perm[:900], cuts)]
    offsets = np.zeros(len(groups) + 1, np.int64)
    offsets[1:] = np.cumsum([gr.size for gr in groups])
    nodes = torch.as_tensor(np.concatenate(groups).astype(np.int64), device=dev)
    offs = torch.as_tensor(offsets, device=dev)
    return g, opA, opB, u, w, nodes, offs, len(groups), (propA, propB, groups)


def _oracle_sums(g, k, u, w, host):
    """sum over each group of (L_A u - L_B w), the CSR operators assembled by
    the CPU oracle from the cell properties (operators.py:302-351)."""
    from oracle import fs_oracle as O
    propA, propB, groups = host
    og = O.Grid(g.xn, g.yn, g.zn)
    LA = O.nodal_laplacian(og, O.edge_mass_vector(og, O.cell_to_edge(og, propA)))
    LB = O.nodal_laplacian(og, O.edge_mass_vector(og, O.cell_to_edge(og, propB)))
    uh = u.cpu().numpy().reshape(-1, k)
    wh = w.cpu().numpy().reshape(-1, k)
    y = LA @ uh - LB @ wh
    mag = np.abs(LA @ uh) + np.abs(LB @ wh)
    sums = np.stack([y[gr].sum(axis=0) for gr in groups])
    scale = max(float(mag[gr].sum(axis=0).max()) for gr in groups)
    return sums.reshape(-1), scale


@pytest.mark.parametrize("k", [1, 8])
def test_noalloc_matches_allocating_entry_point(cuda, k):
    import torch
    from fieldspice_b200 import _lib as L
    lib = L.lib()
    g, opA, opB, u, w, nodes, offs, ng, host = _problem(cuda, k, seed=k)
    nx, ny, nz = g.shape_nodes
    pA = [L.ptr(t) for t in (opA.mx, opA.my, opA.mz)]
    pB = [L.ptr(t) for t in (opB.mx, opB.my, opB.mz)]

    nb = ctypes.c_size_t()
    L.check("ws", lib.fs_group_apply_workspace_bytes(ng, k, ctypes.byref(nb)))
    ws = torch.empty(nb.value, dtype=torch.uint8, device=cuda)
    want = torch.empty(ng * k, dtype=torch.float64, device=cuda)
    L.check("fs_group_apply", lib.fs_group_apply(
        *pA, L.ptr(u), *pB, L.ptr(w), L.ptr(nodes), L.ptr(offs), ng, nx, ny, nz, k,
        L.ptr(want), L.ptr(ws), nb.value, L.stream_ptr()))
    want = want.cpu().numpy()
    scale = np.abs(want).max()
    oracle, oscale = _oracle_sums(g, k, u, w, host)
    # FP64 sums of ~1e3 terms in a different order: 1e-13 of the summed magnitudes
    assert np.abs(want - oracle).max() <= 1e-13 * oscale

    for call in range(2):
        got = torch.full((ng * k,), np.nan, dtype=torch.float64, device=cuda)
        st = lib.fs_group_apply_noalloc(*pA, L.ptr(u), *pB, L.ptr(w), L.ptr(nodes),
                                        L.ptr(offs), ng, nx, ny, nz, k, L.ptr(got),
                                        L.stream_ptr())
        L.check("fs_group_apply_noalloc", st)
        got = got.cpu().numpy()
        assert np.all(np.isfinite(got)), call
        assert np.abs(got - want).max() <= 1e-12 * scale, call
        assert np.abs(got - oracle).max() <= 1e-13 * oscale, call


def test_noalloc_rejects_sizes_beyond_its_static_scratch(cuda):
    import torch
    from fieldspice_b200 import _lib as L
    lib = L.lib()
    g, opA, _, u, _, nodes, offs, ng, _ = _problem(cuda, 16, seed=3)
    nx, ny, nz = g.shape_nodes
    out = torch.zeros(200 * 16, dtype=torch.float64, device=cuda)
    # 200 groups x 16 RHS = 3200 > 2048: refused before any device work
    st = lib.fs_group_apply_noalloc(L.ptr(opA.mx), L.ptr(opA.my), L.ptr(opA.mz),
                                    L.ptr(u), None, None, None, None, L.ptr(nodes),
                                    L.ptr(offs), 200, nx, ny, nz, 16, L.ptr(out),
                                    L.stream_ptr())
    assert st == L.FS_BAD_ARG
    assert "static scratch limit" in lib.fs_last_error().decode()


def test_noalloc_rejects_unsupported_rhs_width(cuda):
    """nrhs must be 1, 2, 4, 8 or 16; anything else is refused with a reason
    before the shared array or the output is touched."""
    import torch
    from fieldspice_b200 import _lib as L
    lib = L.lib()
    g, opA, _, u, _, nodes, offs, ng, _ = _problem(cuda, 4, seed=5)
    nx, ny, nz = g.shape_nodes
    out = torch.full((ng * 3,), 7.0, dtype=torch.float64, device=cuda)
    st = lib.fs_group_apply_noalloc(L.ptr(opA.mx), L.ptr(opA.my), L.ptr(opA.mz),
                                    L.ptr(u), None, None, None, None, L.ptr(nodes),
                                    L.ptr(offs), ng, nx, ny, nz, 3, L.ptr(out),
                                    L.stream_ptr())
    assert st == L.FS_BAD_ARG
    assert "1, 2, 4, 8 or 16" in lib.fs_last_error().decode()
    assert torch.all(out == 7.0)
