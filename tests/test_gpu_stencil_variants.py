"""Every CG stencil kernel gives the reference's capacitance (needs a B200).

``FS_STENCIL`` selects the kernel of ``q = A~ p, p.q`` when a plan is built:
``plain`` (cached loads), ``tma1`` (p staged by TMA), the default (p and the
three mass tiles staged by TMA), ``tmas`` (as the default, with q leaving
through shared memory by TMA stores), ``tma_split`` (as the default, each
32-byte node split over two threads), ``pz`` (the direction update
p = z + beta p_old formed inside the stencil) and ``pz4`` / ``pz16`` (the same
on 32x4 / 32x16 tiles: the tile shapes the autotuner also tries).  Each runs the 48x48x24 layered
extraction recorded from the reference (8 right-hand sides) and, against the
cached-load kernel, the extraction of the first four terminals (4 RHS).
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(golden):
    from fieldspice_b200.grid import RectilinearGrid
    from fieldspice_b200.solvers.base import Terminal
    d = golden("layered_48x48x24_s1")
    g = RectilinearGrid(d["x"], d["y"], d["z"])
    nid = np.arange(g.n_nodes).reshape(g.shape_nodes)
    terms = [Terminal(f"box{i}", nid[a0:a1 + 1, b0:b1 + 1, c0:c1 + 1].ravel())
             for i, (a0, b0, c0, a1, b1, c1) in enumerate(d["boxes"])]
    return d, g, terms


def _extract(g, eps, terms, precision):
    from fieldspice_b200.boundaries import BoundarySpec, Dirichlet
    from fieldspice_b200.solvers.base import GPUConfig, SolverConfig
    from fieldspice_b200.solvers.poisson import PoissonSolver
    ps = PoissonSolver(g, eps, SolverConfig(tol=1e-11),
                       gpu=GPUConfig(precision=precision, preconditioner="mg"))
    return ps.capacitance_matrix(terms, BoundarySpec(zlo=Dirichlet(0.0)))


@pytest.mark.parametrize("variant", ["plain", "tma1", "default", "tmas", "tma_split", "pz",
                                     "pz4", "pz16"])
@pytest.mark.parametrize("precision", ["mixed", "fp64"])
def test_stencil_variant_matches_reference(cuda, golden, monkeypatch, variant, precision):
    d, g, terms = _problem(golden)
    monkeypatch.setenv("FS_STENCIL", "plain")
    C4_plain = _extract(g, d["eps_cell"], terms[:4], precision)
    if variant == "default":
        monkeypatch.delenv("FS_STENCIL", raising=False)
    else:
        monkeypatch.setenv("FS_STENCIL", variant)
    ref = d["C"]
    scale = np.abs(np.diag(ref)).max()
    C = _extract(g, d["eps_cell"], terms, precision)
    assert np.abs(C - ref).max() / scale <= 1e-9
    C4 = _extract(g, d["eps_cell"], terms[:4], precision)
    assert np.abs(C4 - C4_plain).max() / np.abs(np.diag(C4_plain)).max() <= 1e-9


def test_stencil_autotuner_picks_and_caches(cuda, golden, monkeypatch):
    """Without FS_STENCIL the first plan of a shape times the stencil kernels
    and keeps the fastest; the next plan of the same shape reuses it."""
    import torch

    from fieldspice_b200 import _lib as L
    from fieldspice_b200.device import DeviceOperator, EliminatedSystem
    monkeypatch.delenv("FS_STENCIL", raising=False)
    d, g, terms = _problem(golden)
    op = DeviceOperator(g, d["eps_cell"])
    label = torch.zeros(op.N, dtype=torch.uint8, device=op.dev)
    for t in terms:
        label[torch.as_tensor(t.nodes, device=op.dev)] = L.LABEL_FIXED
    kinds = []
    for _ in range(2):
        sys_ = EliminatedSystem(op, label, 8, precision="mixed", preconditioner="mg")
        kinds.append(L.lib().fs_pcg_plan_stencil_kind(sys_.plan))
        sys_.close()
    assert kinds[0] in (0, 2, 3, 4)
    assert kinds[1] == kinds[0]


def _uniform_system(shape, k, precision):
    """A layered grid with its zlo plane fixed, as an eliminated system."""
    import torch

    from fieldspice_b200 import _lib as L
    from fieldspice_b200.device import DeviceOperator, EliminatedSystem
    from fieldspice_b200.grid import RectilinearGrid
    g = RectilinearGrid(*[np.arange(n) * 10e-9 for n in shape])
    eps = np.full(g.shape_cells, 3.9 * 8.854e-12)
    eps[:, :, : shape[2] // 3] *= 2.0
    op = DeviceOperator(g, eps)
    label = torch.zeros(shape, dtype=torch.uint8, device=op.dev)
    label[:, :, 0] = L.LABEL_FIXED
    return EliminatedSystem(op, label.view(-1), k, precision=precision, preconditioner="mg")


def test_stencil_autotuner_times_launches_that_work(cuda, monkeypatch):
    """Each candidate the autotuner times must do the stencil's work: its mean
    launch time is at least the algorithmic bytes over 10 TB/s (more than any
    B200 HBM can move), far above the few microseconds of a launch that
    returns at once.  220x200x100 nodes (2^22 <= N < 2^23, z extent not a
    multiple of 32), 8 FP32 RHS: a shape class no other test uses (the batch
    tests' 8-RHS blocks stop at 2.4 M nodes), so this plan runs the
    autotuner."""
    import ctypes

    from fieldspice_b200 import _lib as L
    monkeypatch.delenv("FS_STENCIL", raising=False)
    shape = (220, 200, 100)
    sys_ = _uniform_system(shape, 8, "mixed")
    ms = (ctypes.c_float * 8)()
    L.check("fs_pcg_plan_stencil_times", L.lib().fs_pcg_plan_stencil_times(sys_.plan, ms))
    kind = L.lib().fs_pcg_plan_stencil_kind(sys_.plan)
    sys_.close()
    N = int(np.prod(shape))
    # at least the stencil's bytes (p, q, masses) over 10 TB/s for every
    # candidate (each is timed with its direction update, whose bytes add)
    floor_ms = N * (2 * 8 * 4 + 3 * 4) / 10e12 * 1e3
    timed = {c: ms[c] for c in range(8) if ms[c] >= 0}
    assert set(timed) == {0, 2, 3, 4, 5, 6, 7}, list(ms)
    for c, t in timed.items():
        assert t >= floor_ms, (c, t, floor_ms)
    assert timed[kind] == min(timed.values())


@pytest.mark.parametrize("precision,k", [("mixed", 8), ("fp64", 4)])
def test_tma_split_selected_for_32_byte_nodes(cuda, monkeypatch, precision, k):
    """FS_STENCIL=tma_split runs the split kernel (kind 4) whenever a node is
    32 bytes (8 FP32 or 4 FP64 values); other widths fall back to kind 2."""
    from fieldspice_b200 import _lib as L
    monkeypatch.setenv("FS_STENCIL", "tma_split")
    sys_ = _uniform_system((48, 40, 32), k, precision)
    assert L.lib().fs_pcg_plan_stencil_kind(sys_.plan) == 4
    sys_.close()
    other = 4 if k == 8 else 8
    sys_ = _uniform_system((48, 40, 32), other, precision)
    assert L.lib().fs_pcg_plan_stencil_kind(sys_.plan) == 2
    sys_.close()
