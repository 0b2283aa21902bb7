"""The learned preconditioner end to end (needs a B200).

A U-Net is trained on the GPU (library kernels only) on residual-to-error
pairs from the path's own Jacobi-PCG iterates on seeded geometries of the
layered-box family, then used as the coarse-level solver of the V-cycle
inside flexible CG on a held-out geometry.  Checks:
* the extraction converges to relres 1e-10 and its C matches an FP64
  multigrid extraction at relres 1e-12 to 1e-9 of max|diag C|;
* what the trained network gains over the method without it, measured
  against both ends: the same flexible CG with the network's output set to
  zero (the V-cycle truncated at the network's level, no coarse correction)
  and the same V-cycle with its own multigrid recursion below that level
  (plain multigrid PCG, the stronger coarse solver).  The trained network
  must recover most of the iterations the recursion saves over no coarse
  correction at all, and do better than an untrained network; it does not
  beat the recursion, which is exact up to smoothing on these levels.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPE = (64, 64, 64)


def _workloads(seeds, shape=SHAPE):
    from fieldspice_b200 import workloads as W
    return [W.layered_boxes(shape, nbox=8, seed=s) for s in seeds]


def _extract(w, gpu, tol=1e-10):
    from fieldspice_b200.solvers.base import SolverConfig
    from fieldspice_b200.solvers.poisson import PoissonSolver
    rep = {}
    C = PoissonSolver(w.grid(), w.eps_cell, SolverConfig(tol=tol), gpu=gpu).capacitance_matrix(
        w.terminal_objects(), w.boundary_spec(), report=rep)
    return C, rep


@pytest.fixture(scope="module")
def trained(cuda):
    from fieldspice_b200.learned import LearnedPreconditioner
    net = LearnedPreconditioner.train(_workloads(range(100, 112)), level=2, epochs=4,
                                      batch=8, lr=1e-3, seed=0)
    return net


def test_training_pairs_are_exact(cuda):
    """b = A~_l x on every pair (recomputed in FP64 from the stored masses)."""
    import torch
    from fieldspice_b200.learned import training_pairs
    data = training_pairs(_workloads([7]), level=2, snapshots=(8, 64))
    d = data["dims"]
    assert d == (16, 16, 16)
    S = data["rhs"].shape[0]
    assert S == 16 and data["em"].shape == (S, 3, 16 ** 3)
    x = data["target"][0].double().reshape(d)
    em = data["em"][0].double().reshape(3, *d)
    free = (data["label"][0] == 0).reshape(d)
    ax = x.clone()
    ax[:-1] -= em[0][:-1] * x[1:]
    ax[1:] -= em[0][:-1] * x[:-1]
    ax[:, :-1] -= em[1][:, :-1] * x[:, 1:]
    ax[:, 1:] -= em[1][:, :-1] * x[:, :-1]
    ax[:, :, :-1] -= em[2][:, :, :-1] * x[:, :, 1:]
    ax[:, :, 1:] -= em[2][:, :, :-1] * x[:, :, :-1]
    ax = torch.where(free, ax, torch.zeros_like(ax))
    b = data["rhs"][0].double().reshape(d)
    assert torch.abs(ax - b).max() <= 1e-5 * torch.abs(b).max()
    assert torch.all(data["target"][0][~free.reshape(-1)] == 0)


def test_training_reduces_the_loss(cuda, trained):
    h = trained.history
    assert len(h) >= 2 and np.all(np.isfinite(h))
    assert h[-1] < 0.5 * h[0], h


@pytest.mark.parametrize("mode", ["replace"])
def test_learned_fcg_matches_fp64_multigrid(cuda, trained, mode):
    from fieldspice_b200.solvers.base import GPUConfig
    w = _workloads([999])[0]                      # held out
    Cref, _ = _extract(w, GPUConfig(precision="fp64", preconditioner="mg"), tol=1e-12)
    C, rep = _extract(w, GPUConfig(preconditioner="learned", learned=trained.with_mode(mode)))
    scale = np.abs(np.diag(Cref)).max()
    assert np.abs(C - Cref).max() / scale <= 1e-9
    assert max(rep["linear"]["relres_fp64"]) < 1e-10
    # with 12 small training geometries FCG may hand a stalled RHS over to
    # multigrid (learned_fallback); the answer is held to the same bar
    assert isinstance(rep["linear"]["learned_fallback"], bool)


def test_hybrid_mode_converges_to_the_same_answer(cuda, trained):
    """The hybrid mode (network guess + V-cycle on its residual) may hand
    over to plain multigrid when FCG stalls; the answer is the same."""
    from fieldspice_b200.solvers.base import GPUConfig
    w = _workloads([999])[0]
    Cref, _ = _extract(w, GPUConfig(precision="fp64", preconditioner="mg"), tol=1e-12)
    C, rep = _extract(w, GPUConfig(preconditioner="learned", learned=trained.with_mode("hybrid")))
    assert np.abs(C - Cref).max() / np.abs(np.diag(Cref)).max() <= 1e-9
    assert max(rep["linear"]["relres_fp64"]) < 1e-10


def test_trained_network_gains_over_the_method_without_it(cuda, trained):
    """The V-cycle with the network as its level-2 correction ('replace'),
    against the same V-cycle with that correction zeroed, with its own
    multigrid recursion (plain multigrid PCG) and with an untrained network."""
    from fieldspice_b200.learned import LearnedPreconditioner
    from fieldspice_b200.solvers.base import GPUConfig
    w = _workloads([999])[0]

    def iters(gpu):
        _, rep = _extract(w, gpu)
        return max(rep["linear"]["iterations"])

    def learned(net):
        return iters(GPUConfig(preconditioner="learned", learned=net))
    rep_net = trained.with_mode("replace")
    it_learned, it_zero = learned(rep_net), learned(rep_net.zero())
    it_rand = learned(LearnedPreconditioner(level=2, seed=5, mode="replace"))
    it_mg = iters(GPUConfig(preconditioner="mg", coarsening="geometric"))
    recovered = (it_zero - it_learned) / max(it_zero - it_mg, 1)
    print(f"iterations: learned {it_learned}, zeroed {it_zero}, untrained {it_rand}, "
          f"multigrid recursion {it_mg}; recovered {recovered:.2f}")
    assert it_mg <= it_learned < it_zero, (it_mg, it_learned, it_zero)
    assert recovered >= 0.5, (it_learned, it_zero, it_mg)
    assert it_learned < it_rand, (it_learned, it_rand)
