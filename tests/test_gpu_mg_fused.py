"""The fused multigrid smoothing passes equal the two-kernel forms (needs a B200).

The degree-2 pre-smoothing of a V-cycle level (``k_mg_pre0`` then
``k_mg_pre1``: x1 = c0 b, r1 = b - c0 A~b, d1 = cd x1 + cr r1, x2 = x1 + d1,
r2 = r1 - A~d1) runs as one TMA-staged x-march over b (``k_mg_pre_fused``),
and the post-smoothing (``k_mg_residual`` then ``k_mg_post2``: r0 = b - A~x,
x + alpha r0 + beta A~r0) as one over x (``k_mg_post_fused``), wherever the
level's rows allow it (for 32-byte nodes with each node split over two threads,
``k_mg_smooth_split``; ``FS_MG_SPLIT=0`` keeps one thread per node);
``FS_MG_PRE=plain`` and ``FS_MG_POST=plain`` keep the two-kernel forms.  The arithmetic and its order are the same, so one V-cycle applied
through ``fs_pcg_plan_precondition`` to the same vector agrees to round-off
(the compilers of the two kernels may contract different products into
FMAs).  The restriction runs as a TMA-staged x-march (``k_mg_restrict_tma``)
for 16- and 32-byte nodes; ``FS_MG_RESTRICT=plain`` keeps the gather kernel
(``k_mg_restrict``), whose sums run in another order: the V-cycles agree to
FP rounding.  8-byte nodes (one FP64 RHS, two FP32) are staged through a
3-D tensor map whose rows merge the RHS and z.  The grid is ragged on purpose: y and z end inside a tile, x is odd,
and two levels run fused while the coarser ones do not.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _system(precision, nrhs, shape=(37, 45, 48), seed=3):
    import torch

    from fieldspice_b200 import _lib as L
    from fieldspice_b200.device import DeviceOperator, EliminatedSystem
    from fieldspice_b200.grid import RectilinearGrid
    rng = np.random.default_rng(seed)
    axes = [np.concatenate([[0.0], np.cumsum(rng.uniform(0.5, 1.5, n - 1))]) * 1e-6
            for n in shape]
    g = RectilinearGrid(*axes)
    eps = rng.uniform(1.0, 12.0, size=tuple(n - 1 for n in shape))
    op = DeviceOperator(g, eps)
    label = torch.zeros(op.N, dtype=torch.uint8, device=op.dev)
    nid = np.arange(op.N).reshape(shape)
    label[torch.as_tensor(nid[:, :, 0].ravel(), device=op.dev)] = L.LABEL_FIXED
    label[torch.as_tensor(nid[3:9, 10:20, 30:34].ravel(), device=op.dev)] = L.LABEL_FIXED
    return EliminatedSystem(op, label, nrhs, precision=precision, preconditioner="mg")


def _vcycle(sys_, r):
    import torch

    from fieldspice_b200 import _lib as L
    z = torch.empty_like(r)
    L.check("fs_pcg_plan_precondition",
            L.lib().fs_pcg_plan_precondition(sys_.plan, ctypes.c_void_p(r.data_ptr()),
                                             ctypes.c_void_p(z.data_ptr()), L.stream_ptr()))
    torch.cuda.synchronize()
    return z


@pytest.mark.parametrize("split", ["1", "0"])
@pytest.mark.parametrize("which", ["FS_MG_PRE", "FS_MG_POST", "FS_MG_RESTRICT"])
@pytest.mark.parametrize("precision,nrhs", [("mixed", 8), ("mixed", 4), ("fp64", 4),
                                            ("fp64", 1), ("mixed", 2)])
def test_fused_smoothing_equals_two_kernels(cuda, monkeypatch, precision, nrhs, which, split):
    """split "1": 32-byte nodes (8 FP32 / 4 FP64 RHS) run the two-threads-per-node
    pass (k_mg_smooth_split); "0" keeps one thread per node."""
    import torch
    sys_ = _system(precision, nrhs)
    dt = torch.float32 if precision == "mixed" else torch.float64
    gen = torch.Generator(device="cuda").manual_seed(11)
    r = torch.randn(sys_.op.N * sys_.k, dtype=dt, device="cuda", generator=gen)
    monkeypatch.delenv("FS_MG_PRE", raising=False)
    monkeypatch.delenv("FS_MG_POST", raising=False)
    monkeypatch.delenv("FS_MG_RESTRICT", raising=False)
    monkeypatch.setenv("FS_MG_SPLIT", split)
    z_fused = _vcycle(sys_, r)
    monkeypatch.setenv(which, "plain")
    z_plain = _vcycle(sys_, r)
    scale = z_plain.abs().max().item()
    tol = 1e-5 if precision == "mixed" else 1e-12
    assert scale > 0
    assert (z_fused - z_plain).abs().max().item() <= tol * scale
    sys_.close()


def test_fused_smoothing_extraction_iterations(cuda, golden, monkeypatch):
    """The 48x48x24 layered extraction recorded from the reference: the same C
    and the same iteration counts with the fused passes and with the two-kernel
    forms."""
    from fieldspice_b200.boundaries import BoundarySpec, Dirichlet
    from fieldspice_b200.grid import RectilinearGrid
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig, Terminal
    from fieldspice_b200.solvers.poisson import PoissonSolver
    d = golden("layered_48x48x24_s1")
    g = RectilinearGrid(d["x"], d["y"], d["z"])
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    terms = [Terminal(f"box{i}", nid[a0:a1 + 1, b0:b1 + 1, c0:c1 + 1].ravel())
             for i, (a0, b0, c0, a1, b1, c1) in enumerate(d["boxes"])]

    def run():
        ps = PoissonSolver(g, d["eps_cell"], SolverConfig(tol=1e-11),
                           gpu=GPUConfig(precision="mixed", preconditioner="mg"))
        C = ps.capacitance_matrix(terms, BoundarySpec(zlo=Dirichlet(0.0)))
        return C, list(ps.last_capacitance_report["linear"]["iterations"])

    monkeypatch.delenv("FS_MG_PRE", raising=False)
    monkeypatch.delenv("FS_MG_POST", raising=False)
    C_f, it_f = run()
    monkeypatch.setenv("FS_MG_PRE", "plain")
    monkeypatch.setenv("FS_MG_POST", "plain")
    monkeypatch.setenv("FS_MG_RESTRICT", "plain")
    C_p, it_p = run()
    scale = np.abs(np.diag(d["C"])).max()
    assert np.abs(C_f - d["C"]).max() / scale <= 1e-9
    assert np.abs(C_f - C_p).max() / scale <= 1e-9
    assert max(it_f) <= max(it_p) + 1
