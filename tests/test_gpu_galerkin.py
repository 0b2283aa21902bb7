"""Multigrid on node aggregates with Galerkin coarse operators (needs a B200).

``coarsening="galerkin"`` builds every coarse level as ``P^T A P`` with P
the piecewise-constant map from 2x2x2 node aggregates to their free fine
nodes.  Checks:
* the device's level-1 and level-2 operators equal ``P^T A P`` assembled in
  NumPy from the fine masses (FP64 plan, equilibrated masses to 1e-12) on an
  odd-sized grid with a 1e6 mass contrast and scattered fixed nodes;
* the extraction of the reference's 48x48x24 layered case through it agrees
  with the reference to 1e-9;
* on a copper-in-oxide EQS operator (conductance ratio 1.7e6) it needs far
  fewer iterations than the rediscretised geometric hierarchy, and
  ``coarsening="auto"`` picks it there;
* over-correcting its coarse corrections (``agg_alpha``, default 1.7) cuts
  the iterations further.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _node_masses(shape, rng, contrast):
    """Random positive edge masses in the padded node layout (0 on the last
    plane of each axis), log-uniform over ``contrast``."""
    m = np.exp(rng.uniform(0.0, np.log(contrast), (3,) + shape))
    m[0, -1] = 0.0
    m[1, :, -1] = 0.0
    m[2, :, :, -1] = 0.0
    return m


def _laplacian(m, shape):
    import scipy.sparse as sp
    nx, ny, nz = shape
    N = nx * ny * nz
    idx = np.arange(N).reshape(shape)
    rows, cols, vals = [], [], []
    for a, (sl0, sl1) in enumerate([((slice(0, -1),), (slice(1, None),)),
                                    ((slice(None), slice(0, -1)), (slice(None), slice(1, None))),
                                    ((slice(None), slice(None), slice(0, -1)),
                                     (slice(None), slice(None), slice(1, None)))]):
        i0, i1 = idx[sl0].ravel(), idx[sl1].ravel()
        w = m[a][sl0].ravel()
        rows += [i0, i1]
        cols += [i1, i0]
        vals += [-w, -w]
    off = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                        shape=(N, N))
    return sp.csr_matrix(off - sp.diags(np.asarray(off.sum(axis=1)).ravel()))


def _classify(A, fixed):
    """Free rows of the eliminated operator as the plan classifies them: not
    fixed, a nonzero diagonal and at least one free neighbour."""
    import scipy.sparse as sp
    n = A.shape[0]
    free = ~fixed
    Aff = sp.csr_matrix(sp.diags(free.astype(float)) @ A @ sp.diags(free.astype(float)))
    d = A.diagonal()
    off_free = np.asarray(abs(Aff - sp.diags(Aff.diagonal())).sum(axis=1)).ravel()
    keep = free & (d != 0) & (off_free > 0)
    return keep, np.arange(n)


def _galerkin_chain(m, shape, fixed, levels):
    """Equilibrated masses of each coarse level: A_c = P^T A_ff P on the
    kept rows, equilibrated to unit diagonal."""
    import scipy.sparse as sp
    A = _laplacian(m, shape)
    keep, _ = _classify(A, fixed)
    out = []
    cur_shape, cur_A, cur_keep = shape, A, keep
    for _ in range(levels):
        nx, ny, nz = cur_shape
        cs = tuple((n + 1) // 2 for n in cur_shape)
        agg = (np.arange(nx)[:, None, None] // 2 * cs[1] + np.arange(ny)[None, :, None] // 2) \
            * cs[2] + np.arange(nz)[None, None, :] // 2
        agg = agg.ravel()
        Nc = int(np.prod(cs))
        P = sp.csr_matrix((cur_keep.astype(float), (np.arange(agg.size), agg)),
                          shape=(agg.size, Nc))
        D = sp.diags(cur_keep.astype(float))
        Ac = sp.csr_matrix(P.T @ (D @ cur_A @ D) @ P)
        dc = Ac.diagonal()
        off = Ac - sp.diags(dc)
        off_abs = np.asarray(abs(off).sum(axis=1)).ravel()
        ckeep = (dc > 0) & (off_abs > 0)
        s = np.where(ckeep, 1.0 / np.sqrt(np.where(dc > 0, dc, 1.0)), 0.0)
        Aeq = sp.csr_matrix(sp.diags(s) @ (-off) @ sp.diags(s))
        cidx = np.arange(Nc).reshape(cs)
        em = np.zeros((3,) + cs)
        em[0, :-1] = np.asarray(Aeq[cidx[:-1].ravel(), cidx[1:].ravel()]).reshape(cs[0] - 1, cs[1], cs[2])
        em[1, :, :-1] = np.asarray(Aeq[cidx[:, :-1].ravel(), cidx[:, 1:].ravel()]).reshape(
            cs[0], cs[1] - 1, cs[2])
        em[2, :, :, :-1] = np.asarray(Aeq[cidx[:, :, :-1].ravel(), cidx[:, :, 1:].ravel()]).reshape(
            cs[0], cs[1], cs[2] - 1)
        out.append((cs, em, ckeep))
        # the next level works on the full (unequilibrated) coarse operator
        cur_shape, cur_A, cur_keep = cs, Ac, ckeep
    return out


def test_coarse_levels_are_the_galerkin_products(cuda):
    import torch

    from fieldspice_b200 import _lib as L
    from fieldspice_b200.device import DeviceOperator, EliminatedSystem
    from fieldspice_b200.grid import RectilinearGrid
    rng = np.random.default_rng(11)
    shape = (70, 61, 40)            # three levels above the coarsest-size limit
    m = _node_masses(shape, rng, 1e6)
    fixed = rng.random(shape) < 0.08
    fixed[:, :, 0] = True
    g = RectilinearGrid(*[np.arange(n, dtype=float) for n in shape])
    op = DeviceOperator(g, masses=torch.as_tensor(m.reshape(3, -1), device=cuda).contiguous(),
                        shape=shape)
    label = torch.as_tensor(fixed.ravel().astype(np.uint8) * L.LABEL_FIXED, device=cuda)
    sys_ = EliminatedSystem(op, label, 1, precision="fp64", preconditioner="mg",
                            coarsening="galerkin")
    lib = L.lib()
    nlev = ctypes.c_int()
    dims = (ctypes.c_int * 48)()
    L.check("levels", lib.fs_pcg_plan_levels(sys_.plan, ctypes.byref(nlev), dims))
    assert nlev.value >= 3
    want = _galerkin_chain(m, shape, fixed.ravel(), 2)
    for lev, (cs, em_want, keep) in zip((1, 2), want):
        assert tuple(dims[3 * lev:3 * lev + 3]) == cs
        em = (ctypes.c_void_p * 3)()
        lab = ctypes.c_void_p()
        L.check("level_data", lib.fs_pcg_plan_level_data(sys_.plan, lev, em, ctypes.byref(lab),
                                                         None))
        n = int(np.prod(cs))
        got = np.stack([_read_f64(sys_.workspace, em[a], n) for a in range(3)]).reshape((3,) + cs)
        assert np.abs(got - em_want).max() <= 1e-12 * max(np.abs(em_want).max(), 1e-300), lev
    sys_.close()


def _read_f64(ws, ptr, n):
    """n FP64 values at device address ptr inside the plan workspace ws."""
    import torch
    off = ptr - ws.data_ptr()
    assert 0 <= off and off + 8 * n <= ws.numel()
    return ws[off:off + 8 * n].view(torch.float64).cpu().numpy()


def test_galerkin_extraction_matches_reference(cuda, golden):
    from fieldspice_b200.boundaries import BoundarySpec, Dirichlet
    from fieldspice_b200.grid import RectilinearGrid
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig, Terminal
    from fieldspice_b200.solvers.poisson import PoissonSolver
    d = golden("layered_48x48x24_s1")
    g = RectilinearGrid(d["x"], d["y"], d["z"])
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    terms = [Terminal(f"box{i}", nid[a0:a1 + 1, b0:b1 + 1, c0:c1 + 1].ravel())
             for i, (a0, b0, c0, a1, b1, c1) in enumerate(d["boxes"])]
    for precision in ("mixed", "fp64"):
        rep = {}
        C = PoissonSolver(g, d["eps_cell"], SolverConfig(tol=1e-11),
                          gpu=GPUConfig(precision=precision, preconditioner="mg",
                                        coarsening="galerkin")).capacitance_matrix(
            terms, BoundarySpec(zlo=Dirichlet(0.0)), report=rep)
        assert rep["linear"]["coarsening"] == "galerkin"
        ref = d["C"]
        assert np.abs(C - ref).max() / np.abs(np.diag(ref)).max() <= 1e-9, precision


def _copper_step(shape, coarsening, precision="fp64", mg_params=None):
    """One backward-Euler step operator of the seeded interconnect (copper
    boxes in oxide over doped silicon, dt = 1 ps), one Dirichlet solve."""
    import torch

    from fieldspice_b200 import _lib as L
    from fieldspice_b200 import workloads as W
    from fieldspice_b200.device import DeviceOperator, EliminatedSystem
    w = W.eqs_interconnect(shape, nbox=6, nports=2, seed=0)
    g = w.grid()
    dt = 1e-12
    K = DeviceOperator(g, w.eps_cell).combine(1.0 / dt, DeviceOperator(g, w.sigma_cell), 1.0)
    label = torch.zeros(K.N, dtype=torch.uint8, device=K.dev)
    nid = np.arange(K.N).reshape(shape)
    fixed = np.concatenate([nid[:, :, 0].ravel()] + [np.asarray(t) for t in w.terminals])
    label[torch.as_tensor(fixed, device=K.dev)] = L.LABEL_FIXED
    sys_ = EliminatedSystem(K, label, 1, precision=precision, preconditioner="mg",
                            coarsening=coarsening, mg_params=mg_params)
    sys_.phi.zero_()
    sys_.phi[torch.as_tensor(np.asarray(w.terminals[0]), device=K.dev)] = 1.0
    _, stats = sys_.solve(1e-10)
    used = sys_.coarsening
    sys_.close()
    return stats[0], used


def test_galerkin_beats_geometric_on_copper_in_oxide(cuda):
    shape = (64, 64, 32)
    geo, _ = _copper_step(shape, "geometric")
    gal, _ = _copper_step(shape, "galerkin")
    _, chosen = _copper_step(shape, "auto")
    print(f"copper/oxide step {shape}: geometric {geo['iterations']} iterations, "
          f"galerkin {gal['iterations']}")
    assert gal["relres"] < 1e-10 and geo["relres"] < 1e-10
    assert gal["iterations"] * 3 <= geo["iterations"], (gal["iterations"], geo["iterations"])
    assert chosen == "galerkin"


def test_aggregation_over_correction(cuda):
    """The default over-correction of the aggregation hierarchy (agg_alpha
    1.7) against plain coarse corrections (1.0) on the copper/oxide step:
    the same converged solve in clearly fewer iterations."""
    shape = (96, 96, 48)
    plain, _ = _copper_step(shape, "galerkin", mg_params={"agg_alpha": 1.0})
    over, _ = _copper_step(shape, "galerkin")
    print(f"copper/oxide step {shape}: alpha 1.0 {plain['iterations']} iterations, "
          f"alpha 1.7 {over['iterations']}")
    assert plain["relres"] < 1e-10 and over["relres"] < 1e-10
    assert over["iterations"] * 5 <= plain["iterations"] * 4
